// Batched, tick-driven correction engine.
//
// Every job (one field) runs the reference GPU driver's control flow
// (src/ExtreM_cuda.cu main() :5508-5997) as a state machine on the host: one
// state per phase of that flow (c_loops detection and rounds, r_loops, a
// manifold round with the wrong-neighbour arbitration, s_loops, saddle_loops,
// their join variants, the third block's detection, the final join pass).
// A tick runs, in program order, every phase that any job is in: one launch
// per kernel serves all jobs in that phase (kernels take the device array of
// job descriptors and a selection), and a job moves on through phases whose
// successor does not depend on a counter within the same tick.  At the end of
// a tick the counter blocks of all jobs come back in one copy and every job
// that stopped at a branch takes it, with the reference's rules.
//
// The branches read exactly the counters the reference reads at the same
// points, so a job's sequence of kernel launches, and its result, do not
// depend on what else is in the batch.  The plain entry points run a batch of
// one job; the batch and serving entry points admit many.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <string>
#include <unordered_map>
#include <vector>

#include "extremz_encode.cuh"
#include "extremz_kernels.cuh"
#include "extremz_topo.cuh"

namespace extremz {

// Trace phases (the same records as the oracle's trace).
enum Phase : int {
  PH_CLOOP_DETECT = 1, PH_WRONG_NBR = 2, PH_SLOOPS = 3, PH_SADDLE = 4, PH_DETECT3 = 5,
  PH_SLOOPS_JOIN = 6, PH_SADDLE_JOIN = 7, PH_OUTER = 8, PH_CHECKSUM = 9
};

// Kernel classes for the optional per-class timing (extremz_report.prof_*).
enum KClass : int {
  K_SETUP = 0, K_DETECT, K_DIRECTION, K_JUMP, K_PROPOSE, K_APPLY, K_ROWS, K_WRONG_NBR,
  K_FIXPATH, K_OTHER, K_DIRECTION_FIRST, K_JUMP_FIRST, K_NUM
};

// Program counter of a job, in the order phases run within a tick.
enum Pc : int {
  PC_SETUP_A = 0,   // classify f, f's manifolds, CP counts          -> sync
  PC_SETUP_B,       // CP lists, rows, per-extremum saddles             -> CL_DETECT
  PC_CL_DETECT,     // c_loops entry: detection                         -> sync
  PC_CL_ROUND,      // c_loops round: proposals, apply, detection       -> sync
  PC_RLOOPS,        // r_loops (fixpath)                                -> MANIFOLD
  PC_MANIFOLD,      // manifolds, rows, wrong neighbours                -> sync
  PC_SLOOPS,        // s_loops                                          -> sync
  PC_SADDLE,        // saddle_loops
  PC_SLOOPS_J,      // s_loops_join                                     -> sync
  PC_SADDLE_J,      // saddle_loops_join (inside the loop)
  PC_PRE_END,       // counters re-read before the loop (:5589-5599)    -> sync
  PC_DET3,          // third block: wrong max / saddle detection
  PC_DET3J,         // third block: join detection
  PC_FINAL_DETECT,  // end of an outer iteration: detection             -> sync
  PC_FINAL_JOIN,    // unconditional saddle_loops_join (:5997)          -> sync
  PC_DONE,
  PC_COUNT = PC_DONE
};

template <class T>
__global__ void k_checksum(const T* __restrict__ a, int N, unsigned long long* out) {
  unsigned long long acc = 0;
  const int stride = gridDim.x * blockDim.x;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < N; v += stride) {
    unsigned long long bits = 0;
    if (sizeof(T) == 8) bits = (unsigned long long)__double_as_longlong((double)a[v]);
    else bits = (unsigned long long)__float_as_uint((float)a[v]);
    unsigned long long z = bits + 0x9e3779b97f4a7c15ull * (unsigned long long)(v + 1);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    acc += z ^ (z >> 31);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, acc);
}

// Workspace of one job of n voxels, in two parts: the per-voxel arrays, taken
// at admission, and the per-critical-point arrays, taken once the counts are
// known (ns2 2-saddles, ns1 1-saddles, nmax maxima, nmin minima).  ksz is the
// size of an order-preserving key (4 or 8).
constexpr long long arr_bytes(long long count, long long sz) { return (count * sz + 255) & ~255ll; }

// Internal job flag (outside the public EXTREMZ_FLAG_* bits): keep a copy of
// the incoming decompressed field for the edit stream.
constexpr int kFlagKeepInput = 1 << 30;
// Internal job flag: analysis only -- classification, labels and critical-point
// lists of the field (admitted as the original), no correction.
constexpr int kFlagAnalysis = 1 << 29;
// Internal job flag: keep the bitset of voxels whose value changed (Job::edited)
// so that only those travel back to a host buffer.
constexpr int kFlagTrackEdits = 1 << 28;
// Internal job flag: mismatch census -- the loop test's eleven counters
// evaluated once on the decompressed field (detection, one manifold round
// with the wrong-neighbour arbitration, and the wrong-extremum / wrong-saddle
// detection of both trees), no edit.
constexpr int kFlagCensus = 1 << 27;
constexpr int kInternalFlags = kFlagKeepInput | kFlagAnalysis | kFlagTrackEdits | kFlagCensus;

constexpr long long job_bytes_voxels(long long n, long long ksz) {
  return arr_bytes(n, 1) + arr_bytes(n, 2)                          // otype, olm
         + 5 * arr_bytes(n, 4)                                      // ds, as, dds, das, ext
         + arr_bytes(n, ksz) + 3 * arr_bytes(n, 4)                  // delta, counter, touched, mm
         + arr_bytes(n, 4) + arr_bytes(n, 1) + 3 * arr_bytes(n, 4)  // mm_next, mstat, dirty, stamps
         + arr_bytes(n, 8) + 2 * arr_bytes(n, 4)                    // claim, taken, taken1
         + 4 * arr_bytes(n, 4)                                      // cand(_next), flagged(1)
         + arr_bytes(n, 4) + arr_bytes(n, 1)                        // cand_j, mis
         + 2 * arr_bytes(n, 4)                                      // pdd, pda
         + arr_bytes((n + 31) / 32, 4) + arr_bytes(n, 1)            // change bitset, dirtyv
         + 4 * arr_bytes((n + 31) / 32, 4)  // wrong-saddle change bitsets, touched roots
         + 2 * arr_bytes((n + kCpBlock - 1) / kCpBlock, 4)  // dirtyv stamp, seed count per block
         + arr_bytes(6 * ((n + kCpBlock - 1) / kCpBlock), 4)        // CP block counts
         + arr_bytes(6 * ((n + kCpBlock - 1) / kCpBlock / 1024 + 1), 4)  // and their chunk sums
         + 4096;
}

constexpr long long job_bytes_cps(long long ns2, long long ns1, long long nmax, long long nmin,
                                  long long e2, long long e1, long long ksz) {
  return arr_bytes(ns2, 4) + arr_bytes(ns1, 4) + arr_bytes(nmax, 4) + arr_bytes(nmin, 4)
         + arr_bytes(ns2 * kRowStride, 4) + arr_bytes(ns2 * 2, 4) + arr_bytes(ns2, 1)
         + arr_bytes(ns1 * kRowStride, 4) + arr_bytes(ns1 * 2, 4) + arr_bytes(ns1, 1)
         + 2 * arr_bytes(ns2, 16) + 2 * arr_bytes(ns1, 16)  // compact rows (orm, oend)
         + arr_bytes(ns2, 1) + arr_bytes(ns1, 1)                    // seed bits
         + 4 * arr_bytes(nmax, 4) + 4 * arr_bytes(nmin, 4)
         + arr_bytes(nmax > nmin ? nmax : nmin, ksz) + arr_bytes(nmax > nmin ? nmax : nmin, 4)
         + arr_bytes(8, 8)
         // per-extremum row-entry lists: offsets, entries, stamps; queue, chunk sums
         + arr_bytes(nmax + 1, 4) + arr_bytes(e2, 4) + arr_bytes(nmax, 4)
         + arr_bytes(nmin + 1, 4) + arr_bytes(e1, 4) + arr_bytes(nmin, 4)
         + 2 * arr_bytes(nmax > nmin ? nmax : nmin, 4)
         + arr_bytes((nmax > nmin ? nmax : nmin) / 1024 + 2, 4) + 4096;
}

// Per tile: change mark.
constexpr long long job_bytes_tiles(long long nt) { return arr_bytes(nt, 1); }

// Worst case (every voxel a critical point of every kind; a voxel's upper and
// lower neighbours, at most 14, give the row entries of both sides; at most
// one tile per voxel).
constexpr long long job_bytes_sz(long long n, long long ksz) {
  return job_bytes_voxels(n, ksz) + job_bytes_tiles(n) +
         job_bytes_cps(n, n, n, n, 7 * n, 7 * n, ksz);
}
template <class T>
constexpr long long job_bytes(long long n) {
  return job_bytes_sz(n, sizeof(typename KeyOf<T>::K));
}
constexpr long long job_bytes_max(long long n) { return job_bytes_sz(n, 8); }

// One job's host-side state.
template <class T>
struct JobHost {
  using K = typename KeyOf<T>::K;
  bool used = false;
  int pc = PC_DONE;
  int block = 0;          // 0 = before the loop, 1..3 = block of an outer iteration
  bool waiting = false;   // stopped at a branch that needs this tick's counters
  cudaEvent_t input_ready = nullptr;  // the decompressed field is still arriving until this event
  int outer = 0, rounds = 0, cloop_total = 0, manifold_rounds = 0;
  int nfc = 0, nfc1 = 0;
  int c[11] = {0};        // loop-test counters (:5603-5605)
  bool dense_done = false;
  int status = EXTREMZ_OK;
  extremz_params p{};
  Job<T> J{};
  Arena arena, arena2;  // per-voxel part, per-critical-point part
  bool own_arena = false, own_arena2 = false;
  int ntiles = 0, nb = 0;
  int* bcount = nullptr;
  int* chunk = nullptr;  // chunk sums of the CP block counts
  unsigned long long* checksum = nullptr;
  int32_t* trace = nullptr;
  int trace_cap = 0, trace_len = 0;
  std::vector<int> pending;  // trace phases to emit once the tick's counters are back
  int blocks_per_sm = 8;      // grid-stride kernels' blocks per SM (tuning knob)
  long long applied_tick = -1;  // last tick that issued edits for this job
  long long tag = 0;

  void emit(int phase, int a = 0, int b = 0, int c3 = 0) {
    if (!trace || trace_len + 4 > trace_cap) return;
    trace[trace_len++] = phase;
    trace[trace_len++] = a;
    trace[trace_len++] = b;
    trace[trace_len++] = c3;
  }
};

template <class T>
class BatchEngine {
 public:
  using K = typename KeyOf<T>::K;

  explicit BatchEngine(cudaStream_t st) : st_(st) {}
  ~BatchEngine() { release_all(); }

  int init(const DeviceTables* preset_tables, Arena* fixed_storage) {
    if (ready_) return EXTREMZ_OK;
    int dev = 0;
    EZ_CHECK(cudaGetDevice(&dev));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    sms_ = sms;
    grid_ = sms * 8;
    if (preset_tables) tb_ = *preset_tables;
    else if (int rc = device_tables(&tb_)) return rc;
    const size_t desc_bytes = sizeof(Job<T>) * kMaxSel;
    const size_t map_bytes = sizeof(CUtensorMap) * 2 * kMaxSel;
    const size_t ctr_bytes = sizeof(int) * C_COUNT * kMaxSel;
    if (fixed_storage) {  // borrowed: carve the engine's arrays from it
      jobs_dev_ = fixed_storage->template take<Job<T>>(kMaxSel);
      maps_dev_ = fixed_storage->template take<CUtensorMap>(2 * kMaxSel);
      ctr_dev_ = fixed_storage->template take<int>(C_COUNT * kMaxSel);
      if (!jobs_dev_ || !maps_dev_ || !ctr_dev_) return EXTREMZ_OOM;
      borrowed_ = true;
      ctr_host_ = static_ctr_host_;
    } else {
      if (cudaMalloc(&jobs_dev_, desc_bytes) != cudaSuccess ||
          cudaMalloc(&maps_dev_, map_bytes) != cudaSuccess ||
          cudaMalloc(&ctr_dev_, ctr_bytes) != cudaSuccess ||
          cudaMallocHost(&ctr_host_, ctr_bytes) != cudaSuccess) {
        cudaGetLastError();
        return EXTREMZ_OOM;
      }
    }
    slots_.assign(kMaxSel, JobHost<T>());
    ready_ = true;
    return EXTREMZ_OK;
  }

  void release_all() {
    drop_graphs();
    for (auto& j : slots_) free_job(j);
    if (!borrowed_) {
      if (jobs_dev_) cudaFree(jobs_dev_);
      if (maps_dev_) cudaFree(maps_dev_);
      if (ctr_dev_) cudaFree(ctr_dev_);
      if (ctr_host_) cudaFreeHost(ctr_host_);
    }
    jobs_dev_ = nullptr;
    maps_dev_ = nullptr;
    ctr_dev_ = nullptr;
    ctr_host_ = nullptr;
    ready_ = false;
  }

  int free_slots() const {
    int n = 0;
    for (const auto& j : slots_) n += !j.used;
    return n;
  }
  int active() const {
    int n = 0;
    for (const auto& j : slots_) n += j.used && j.pc != PC_DONE;
    return n;
  }
  long long launches() const { return launches_; }
  long long graph_replays() const { return graph_replays_; }
  long long graph_captures() const { return graph_captures_; }
  void set_graphs(bool on) {
    graphs_on_ = on;
    if (!on) drop_graphs();
  }
  void set_stream(cudaStream_t st) { st_ = st; }
  cudaStream_t stream() const { return st_; }
  // Stream-ordered pool the job workspaces come from (nullptr: the device's
  // default pool).
  void set_pool(cudaMemPool_t pool) { pool_mem_ = pool; }
  void set_profile(bool on, int mask) {
    profile_ = on;
    profile_mask_ = mask;
  }

  // Admits a job.  storage: borrowed workspace (nullptr = allocate).
  int admit(const T* f, T* g, int W, int H, int D, const extremz_params& p, int32_t* trace,
            int trace_cap, Arena* storage, long long tag, int* slot_out) {
    int slot = -1;
    for (int i = 0; i < kMaxSel; ++i)
      if (!slots_[i].used) {
        slot = i;
        break;
      }
    if (slot < 0) return EXTREMZ_OOM;
    JobHost<T>& jh = slots_[slot];
    jh = JobHost<T>();
    jh.used = true;
    jh.p = p;
    jh.tag = tag;
    jh.trace = trace;
    jh.trace_cap = trace_cap;
    Job<T>& J = jh.J;
    std::memset(&J, 0, sizeof(J));
    J.dim = Dims{W, H, D, W * H * D};
    J.f = f;
    J.g = g;
    J.bound = (T)p.bound;
    J.thr = (T)p.thr;
    J.sentinel = T(-4.0) * J.bound;  // init_delta (:2572)
    J.sentinel_key = KeyOf<T>::enc(J.sentinel);
    J.q = p.q;
    J.edit_type = p.edit_type;
    J.iter_cap = p.device_iter_cap > 0 ? p.device_iter_cap : J.dim.N + 1;
    J.pass_chunk = p.tune_pass_chunk > 0 ? p.tune_pass_chunk : 4;
    J.wn_lockstep = (p.flags & EXTREMZ_FLAG_WN_ASCENDING) == 0;
    jh.blocks_per_sm = p.tune_blocks_per_sm > 0 ? p.tune_blocks_per_sm : 8;
    J.tb = tb_;
    J.ctr = ctr_dev_ + (size_t)slot * C_COUNT;
    const int N = J.dim.N;
    // Borrowed storage holds both parts; an allocation holds the first (and a
    // copy of the incoming field when an edit stream will be encoded).
    const bool keep_input = (p.flags & kFlagKeepInput) != 0;
    const bool track_edits = (p.flags & kFlagTrackEdits) != 0;
    const long long ntiles = (long long)((W + TX - 1) / TX) * ((H + TY - 1) / TY) * ((D + TZ - 1) / TZ);
    const long long need = (storage ? job_bytes<T>(N)
                                    : job_bytes_voxels(N, sizeof(K)) + job_bytes_tiles(ntiles)) +
                           (keep_input ? arr_bytes(N, sizeof(T)) : 0) +
                           (track_edits ? arr_bytes((N + 31) / 32, 4) : 0);
    if (storage) {
      jh.arena = *storage;
      jh.arena.used = 0;
      if ((long long)jh.arena.cap < need) {
        jh.used = false;
        return EXTREMZ_OOM;
      }
    } else {
      void* base = nullptr;
      const cudaError_t e = pool_mem_ ? cudaMallocFromPoolAsync(&base, (size_t)need, pool_mem_, st_)
                                      : cudaMallocAsync(&base, (size_t)need, st_);
      if (e != cudaSuccess) {
        cudaGetLastError();
        jh.used = false;
        return EXTREMZ_OOM;
      }
      jh.arena.base = static_cast<char*>(base);
      jh.arena.cap = (size_t)need;
      jh.arena.fixed = true;
      jh.own_arena = true;
    }
    Arena& A = jh.arena;
    J.otype = A.take<int8_t>(N);
    J.olm = A.take<uint16_t>(N);
    J.ds = A.take<int>(N);
    J.as = A.take<int>(N);
    J.dds = A.take<int>(N);
    J.das = A.take<int>(N);
    J.ext = A.take<int>(N);
    J.delta = A.take<K>(N);
    J.counter = A.take<int>(N);
    J.touched = A.take<int>(N);
    J.mm = A.take<int>(N);
    J.mm_next = A.take<int>(N);
    J.mstat = A.take<uint8_t>(N);
    J.dirty = A.take<int>(N);
    J.dstamp = A.take<int>(N);
    J.rstamp = A.take<int>(N);
    J.claim = A.take<unsigned long long>(N);
    J.taken = A.take<int>(N);
    J.taken1 = A.take<int>(N);
    J.cand = A.take<int>(N);
    J.cand_next = A.take<int>(N);
    J.flagged = A.take<int>(N);
    J.flagged1 = A.take<int>(N);
    J.cand_j = A.take<int>(N);
    J.mis = A.take<uint8_t>(N);
    J.pdd = A.take<int>(N);
    J.pda = A.take<int>(N);
    J.vchg = A.take<unsigned>((N + 31) / 32);
    J.rtouch2 = A.take<unsigned>((N + 31) / 32);
    J.rtouch1 = A.take<unsigned>((N + 31) / 32);
    J.wchg2 = A.take<unsigned>((N + 31) / 32);
    J.wchg1 = A.take<unsigned>((N + 31) / 32);
    J.dirtyv = A.take<uint8_t>(N);
    jh.nb = (N + kCpBlock - 1) / kCpBlock;
    J.bdirty = A.take<int>(jh.nb);
    J.hcnt = A.take<int>(jh.nb);
    jh.bcount = A.take<int>(6ll * jh.nb);
    jh.chunk = A.take<int>(6ll * ((jh.nb + 1023) / 1024));
    J.cpoff = jh.bcount;
    jh.ntiles = ((W + TX - 1) / TX) * ((H + TY - 1) / TY) * ((D + TZ - 1) / TZ);
    J.tdirty = A.take<uint8_t>(jh.ntiles);

    J.g0 = keep_input ? A.take<T>(N) : nullptr;
    J.edited = track_edits ? A.take<unsigned>((N + 31) / 32) : nullptr;
    if (!J.tdirty || (keep_input && !J.g0) || (track_edits && !J.edited)) {
      free_job(jh);
      return EXTREMZ_OOM;
    }
    if (track_edits)
      EZ_CHECK(cudaMemsetAsync(J.edited, 0, (size_t)((N + 31) / 32) * 4, st_));
    if (keep_input)
      EZ_CHECK(cudaMemcpyAsync(J.g0, g, (size_t)N * sizeof(T), cudaMemcpyDeviceToDevice, st_));
    // Tile maps of both fields (TMA when the stride allows).
    CUtensorMap mf, mg;
    const bool tma_ok = (p.flags & EXTREMZ_FLAG_NO_TMA) == 0;
    J.tma_f = tma_ok && make_tile_map(&mf, f, J.dim);
    J.tma_g = tma_ok && make_tile_map(&mg, (const T*)g, J.dim);
    EZ_CHECK(cudaMemcpyAsync(maps_dev_ + 2 * slot, &mf, sizeof(mf), cudaMemcpyHostToDevice, st_));
    EZ_CHECK(cudaMemcpyAsync(maps_dev_ + 2 * slot + 1, &mg, sizeof(mg), cudaMemcpyHostToDevice, st_));
    J.map_f = maps_dev_ + 2 * slot;
    J.map_g = maps_dev_ + 2 * slot + 1;
    EZ_CHECK(cudaMemsetAsync(J.ctr, 0, C_COUNT * sizeof(int), st_));
    EZ_CHECK(cudaMemcpyAsync(jobs_dev_ + slot, &J, sizeof(J), cudaMemcpyHostToDevice, st_));
    jh.pc = PC_SETUP_A;
    if (slot_out) *slot_out = slot;
    return EXTREMZ_OK;
  }

  const JobHost<T>& job(int slot) const { return slots_[slot]; }

  void fill_report(int slot, extremz_report* r) const {
    const JobHost<T>& j = slots_[slot];
    if (!r) return;
    r->status = j.status;
    r->outer_iters = j.outer;
    r->cloop_rounds = j.cloop_total;
    r->manifold_rounds = j.manifold_rounds;
    std::memcpy(r->counters, j.c, sizeof(j.c));
    r->error_bits = ctr_host_ ? ctr_host_[(size_t)slot * C_COUNT + C_ERROR] : 0;
    r->manifold_reused = ctr_host_ ? ctr_host_[(size_t)slot * C_COUNT + C_MFREUSED] : 0;
    for (int k = 0; k < 4; ++k)
      r->cp_counts[k] = ctr_host_ ? ctr_host_[(size_t)slot * C_COUNT + C_NS2 + k] : 0;
  }

  // Edit stream of a finished job admitted with kFlagKeepInput, into the
  // caller's device buffers es->index / es->edits (see extremz_encode.cuh).
  // Synchronises the stream.  BAD_ARG when a buffer is too small (the sizes
  // needed are filled in) or a counter does not fit three bits.
  int encode(int slot, extremz_edit_stream* es) {
    JobHost<T>& jh = slots_[slot];
    const Job<T>& J = jh.J;
    if (!J.g0 || !es) return EXTREMZ_BAD_ARG;
    const int N = J.dim.N, nb = jh.nb, et = jh.p.edit_type, q = jh.p.q;
    if (et == 0 && q > 7) return EXTREMZ_BAD_ARG;  // counters up to q: three bits
    unsigned long long* acc = jh.checksum;         // 8 words of scratch
    unsigned long long init[8] = {0, 0, KeyOf<double>::enc((double)INFINITY),
                                  KeyOf<double>::enc(-(double)INFINITY), 0, 0, 0, 0};
    EZ_CHECK(cudaMemcpyAsync(acc, init, sizeof(init), cudaMemcpyHostToDevice, st_));
    int* bc = jh.bcount;  // 4 x nb ints, free once the correction is over
    launch(K_OTHER, k_enc_count<T>, nb, kCpBlock, (const T*)J.g0, (const T*)J.g,
           (const int*)J.counter, N, q, et, bc);
    launch(K_OTHER, k_scan_lists, 1, 1024, bc, nb, 2, reinterpret_cast<int*>(acc + 4));
    launch(K_OTHER, k_enc_stats<T>, grid_, 256, J.f, (const T*)J.g0, (const T*)J.g, N, acc);
    unsigned long long h[8];
    EZ_CHECK(cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, st_));
    EZ_CHECK(cudaStreamSynchronize(st_));
    int tot[2];
    std::memcpy(tot, &h[4], sizeof(tot));
    const long long index_bytes = et == 0 ? (3ll * N + 7) / 8 : 4ll * tot[0];
    const long long edit_bytes = (long long)tot[1] * (long long)sizeof(T);
    es->edited = tot[0];
    es->n_edits = tot[1];
    es->index_bytes = index_bytes;
    es->edit_bytes = edit_bytes;
    double s0, s1;
    std::memcpy(&s0, &h[0], 8);
    std::memcpy(&s1, &h[1], 8);
    const double range = KeyOf<double>::dec(h[3]) - KeyOf<double>::dec(h[2]);
    auto psnr = [&](double sse) {
      const double mse = sse / (double)N;
      return mse == 0 ? (double)INFINITY : -20.0 * std::log10(std::sqrt(mse) / range);
    };
    es->psnr_before = psnr(s0);
    es->psnr_after = psnr(s1);
    if (index_bytes > es->index_cap || edit_bytes > es->edits_cap ||
        (index_bytes && !es->index) || (edit_bytes && !es->edits))
      return EXTREMZ_BAD_ARG;
    launch(K_OTHER, k_enc_write<T>, nb, kCpBlock, J.f, (const T*)J.g0, (const T*)J.g,
           (const int*)J.counter, N, J.bound, q, et, (const int*)bc, J.touched,
           static_cast<T*>(es->edits));
    if (et == 1) {
      launch(K_OTHER, k_enc_diff, grid_, 256, (const int*)J.touched, tot[0],
             static_cast<int*>(es->index));
    } else {
      launch(K_OTHER, k_enc_pack3<T>, grid_, 256, (const T*)J.g0, (const T*)J.g,
             (const int*)J.counter, (long long)N, static_cast<uint8_t*>(es->index), index_bytes,
             acc + 5);
    }
    unsigned long long bad = 0;
    EZ_CHECK(cudaMemcpyAsync(&bad, acc + 5, 8, cudaMemcpyDeviceToHost, st_));
    EZ_CHECK(cudaStreamSynchronize(st_));
    return bad ? EXTREMZ_BAD_ARG : EXTREMZ_OK;
  }

  // Voxels of a finished job admitted with kFlagTrackEdits whose value
  // changed: ids (ascending) into the job's `touched` array and their
  // corrected values into its proposal buffer, both free once the correction
  // is over.  Returns the count; edited_ids / edited_vals give the arrays.
  int edited_list(int slot, int* count) {
    JobHost<T>& jh = slots_[slot];
    const Job<T>& J = jh.J;
    static_assert(sizeof(K) == sizeof(T), "values are written over the proposal keys");
    if (!J.edited) return EXTREMZ_BAD_ARG;
    const int N = J.dim.N, nb = jh.nb;
    int* tot = reinterpret_cast<int*>(jh.checksum);
    launch(K_OTHER, k_edit_count, nb, 32, (const unsigned*)J.edited, N, jh.bcount);
    launch(K_OTHER, k_scan_lists, 1, 1024, jh.bcount, nb, 1, tot);
    launch(K_OTHER, k_edit_write<T>, nb, 32, (const unsigned*)J.edited, (const T*)J.g, N,
           (const int*)jh.bcount, J.touched, reinterpret_cast<T*>(J.delta));
    EZ_CHECK(cudaMemcpyAsync(count, tot, sizeof(int), cudaMemcpyDeviceToHost, st_));
    EZ_CHECK(cudaStreamSynchronize(st_));
    return EXTREMZ_OK;
  }
  const int* edited_ids(int slot) const { return slots_[slot].J.touched; }
  const T* edited_vals(int slot) const { return reinterpret_cast<const T*>(slots_[slot].J.delta); }

  // Stream-ordered scratch from the engine's pool (or the device's default).
  void* scratch(size_t bytes) {
    void* p = nullptr;
    const cudaError_t e = pool_mem_ ? cudaMallocFromPoolAsync(&p, bytes, pool_mem_, st_)
                                    : cudaMallocAsync(&p, bytes, st_);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    return p;
  }

  // Merge-tree persistence pairs of a finished analysis job (see
  // extremz_topo.cuh): split tree into max_pairs (2 ints per maximum), join
  // tree into min_pairs (2 per minimum), device buffers of the caller.
  // counts (host) receives the numbers of maxima and minima.  Synchronises.
  int persistence(int slot, int* max_pairs, long long max_cap, int* min_pairs, long long min_cap,
                  long long* counts, int* max_parent = nullptr, int* min_parent = nullptr) {
    JobHost<T>& jh = slots_[slot];
    const Job<T>& J = jh.J;
    const int ne[2] = {h(slot, C_NMAX), h(slot, C_NMIN)};
    counts[0] = ne[0];
    counts[1] = ne[1];
    if (2ll * ne[0] > max_cap || 2ll * ne[1] > min_cap || (ne[0] && !max_pairs) ||
        (ne[1] && !min_pairs))
      return EXTREMZ_BAD_ARG;
    // Merge vertices of both trees, ascending id (the job's CP-block scratch
    // is free once the analysis is done).
    const int N = J.dim.N;
    int* cand = static_cast<int*>(scratch((size_t)2 * N * sizeof(int) + 256));
    if (!cand) return EXTREMZ_OOM;
    int* ctot = J.ctr + C_CAND;  // two free counter slots of the finished job
    launch(K_OTHER, k_pp_cand_count<T>, jh.nb, kCpBlock, J.f, J.dim, jh.bcount);
    launch(K_OTHER, k_scan_lists, 1, 1024, jh.bcount, jh.nb, 2, ctot);
    launch(K_OTHER, k_pp_cand_write<T>, jh.nb, kCpBlock, J.f, J.dim, (const int*)jh.bcount, cand,
           cand + N);
    int ns[2];
    EZ_CHECK(cudaMemcpyAsync(ns, ctot, sizeof(ns), cudaMemcpyDeviceToHost, st_));
    EZ_CHECK(cudaStreamSynchronize(st_));
    const int nmaxall = std::max(std::max(ns[0], ns[1]), std::max(ne[0], ne[1])) + 1;
    // Scratch: sort keys and values (in and out), ranks, rows and counts,
    // largest / pointer / pair per extremum, sorted list indices of both
    // sides' extrema, and the round flag.
    size_t cub_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, cub_bytes, (unsigned long long*)nullptr,
                                    (unsigned long long*)nullptr, (int*)nullptr, (int*)nullptr,
                                    nmaxall, 0, 64, st_);
    const size_t a = ((size_t)nmaxall * 8 + 255) & ~size_t(255);
    const size_t b = ((size_t)nmaxall * 4 + 255) & ~size_t(255);
    const size_t rows_bytes = (((size_t)std::max(ns[0], ns[1]) + 1) * kPpRow * 4 + 255) & ~size_t(255);
    const size_t total = 2 * a + 10 * b + rows_bytes + ((cub_bytes + 255) & ~size_t(255)) + 256;
    char* base = static_cast<char*>(scratch(total));
    if (!base) {
      cudaFreeAsync(cand, st_);
      return EXTREMZ_OOM;
    }
    char* q = base;
    auto take = [&](size_t n) { char* r = q; q += n; return r; };
    auto* kin = reinterpret_cast<unsigned long long*>(take(a));
    auto* kout = reinterpret_cast<unsigned long long*>(take(a));
    int* vin = reinterpret_cast<int*>(take(b));
    int* ext_li[2] = {reinterpret_cast<int*>(take(b)), reinterpret_cast<int*>(take(b))};
    int* sad_li = reinterpret_cast<int*>(take(b));
    int* erank = reinterpret_cast<int*>(take(b));
    int* largest = reinterpret_cast<int*>(take(b));
    int* ptr = reinterpret_cast<int*>(take(b));
    int* pair = reinterpret_cast<int*>(take(b));
    int* lmax = reinterpret_cast<int*>(take(b));
    int* cnt = reinterpret_cast<int*>(take(b));
    int* rows = reinterpret_cast<int*>(take(rows_bytes));
    void* cub_tmp = take((cub_bytes + 255) & ~size_t(255));
    int* flag = reinterpret_cast<int*>(take(256));  // [0] round paired, [1] jump limit hit
    EZ_CHECK(cudaMemsetAsync(flag, 0, 8, st_));
    const int* elist[2] = {J.maxima, J.minima};
    const int* slist[2] = {cand, cand + N};
    int rc = EXTREMZ_OK;
    auto sort = [&](const int* list, int n, bool reverse, bool complement, int* out_li) {
      launch(K_OTHER, k_pp_keys<T>, grid_, 256, J.f, list, n, reverse, complement, kin, vin);
      size_t tb = cub_bytes;
      if (cub::DeviceRadixSort::SortPairs(cub_tmp, tb, kin, kout, vin, out_li, n, 0, 64, st_) !=
          cudaSuccess)
        rc = EXTREMZ_CUDA_ERR;
    };
    // Extrema ascending in each tree's order: maxima by (value, id), minima by
    // the reverse of it.
    if (ne[0]) sort(elist[0], ne[0], false, false, ext_li[0]);
    if (ne[1]) sort(elist[1], ne[1], true, true, ext_li[1]);
    int glob[2] = {-1, -1};  // global maximum, global minimum (vertex ids)
    if (ne[0] && ne[1] && rc == EXTREMZ_OK) {
      int li[2];
      EZ_CHECK(cudaMemcpyAsync(&li[0], ext_li[0] + ne[0] - 1, 4, cudaMemcpyDeviceToHost, st_));
      EZ_CHECK(cudaMemcpyAsync(&li[1], ext_li[1] + ne[1] - 1, 4, cudaMemcpyDeviceToHost, st_));
      EZ_CHECK(cudaStreamSynchronize(st_));
      EZ_CHECK(cudaMemcpyAsync(&glob[0], elist[0] + li[0], 4, cudaMemcpyDeviceToHost, st_));
      EZ_CHECK(cudaMemcpyAsync(&glob[1], elist[1] + li[1], 4, cudaMemcpyDeviceToHost, st_));
      EZ_CHECK(cudaStreamSynchronize(st_));
    }
    for (int side = 0; side < 2 && rc == EXTREMZ_OK; ++side) {
      const bool kmax = side == 0;
      const int n_e = ne[side], n_s = ns[side];
      if (n_e == 0) continue;
      launch(K_OTHER, k_pp_rank, grid_, 256, (const int*)ext_li[side], n_e, erank);
      // Saddles descending in the tree's order.
      if (n_s) sort(slist[side], n_s, kmax, kmax, sad_li);
      if (kmax)
        launch(K_OTHER, k_pp_rows<T, true>, grid_, 256, J.f, J.dim, slist[0], (const int*)sad_li,
               n_s, (const int*)J.ds, (const int*)J.ext, (const int*)erank, rows, cnt);
      else
        launch(K_OTHER, k_pp_rows<T, false>, grid_, 256, J.f, J.dim, slist[1], (const int*)sad_li,
               n_s, (const int*)J.as, (const int*)J.ext, (const int*)erank, rows, cnt);
      launch(K_OTHER, k_fill<int>, grid_, 256, largest, kInf, (long long)n_e);
      launch(K_OTHER, k_fill<int>, grid_, 256, pair, -1, (long long)n_e);
      launch(K_OTHER, k_iota, grid_, 256, ptr, n_e);
      for (int round = 0; round <= n_e; ++round) {  // every round but the last pairs one
        EZ_CHECK(cudaMemsetAsync(flag, 0, 4, st_));
        if (n_s) launch(K_OTHER, k_pp_largest, grid_, 256, (const int*)rows, (const int*)cnt, n_s,
                        n_e - 1, largest);
        launch(K_OTHER, k_pp_pair, grid_, 256, (const int*)rows, (const int*)cnt, n_e, n_s,
               largest, ptr, pair, lmax, flag);
        int changed = 0;
        EZ_CHECK(cudaMemcpyAsync(&changed, flag, 4, cudaMemcpyDeviceToHost, st_));
        EZ_CHECK(cudaStreamSynchronize(st_));
        if (!changed) break;
        launch(K_OTHER, k_pp_jump, grid_, 256, ptr, n_e, n_e + 1, flag + 1);
        if (n_s) launch(K_OTHER, k_pp_remap, grid_, 256, rows, cnt, n_s, (const int*)ptr);
      }
      launch(K_OTHER, k_pp_out, grid_, 256, (const int*)pair, n_e, (const int*)ext_li[side],
             elist[side], (const int*)sad_li, slist[side], glob[1 - side],
             kmax ? max_pairs : min_pairs, (const int*)lmax, kmax ? max_parent : min_parent);
    }
    int jump_err = 0;
    cudaMemcpyAsync(&jump_err, flag + 1, 4, cudaMemcpyDeviceToHost, st_);
    cudaFreeAsync(base, st_);
    cudaFreeAsync(cand, st_);
    EZ_CHECK(cudaStreamSynchronize(st_));
    if (rc == EXTREMZ_OK && jump_err) rc = EXTREMZ_DEVICE_TIMEOUT;
    return rc;
  }

  // Releases a finished job's slot and (stream-ordered) its workspace.
  void release(int slot) {
    slots_[slot].input_ready = nullptr;
    free_job(slots_[slot]);
  }
  // The job's decompressed field is still being copied in until `ev` (on
  // another stream): setup, which reads only the original field, runs
  // meanwhile, and the first tick that reads the decompressed field waits.
  void set_input_event(int slot, cudaEvent_t ev) { slots_[slot].input_ready = ev; }
  // Releases every job (after an error that ends a batch).
  void release_jobs() {
    for (auto& j : slots_) free_job(j);
  }

  // One tick: every phase any job is in, in program order; then one copy of
  // all counter blocks and the branches.  Returns a status (the jobs keep
  // their own statuses).
  int tick() {
    EZ_RUN(tick_issue());
    return tick_complete();
  }

  // First half of a tick: the launches and the asynchronous copy of the
  // counter blocks.  Engines on different streams issue, then complete, so
  // their ticks overlap on the device.
  int tick_issue() {
    issued_ = false;
    ++tick_id_;
    // A tick whose launches repeat an earlier tick's exactly (kernels, launch
    // shapes and arguments; per-job state is read from device memory) runs as
    // one CUDA graph: recorded, captured the third time its signature is
    // seen, replayed from then on.  Ticks that allocate (setup) launch
    // directly.  Timed launches (EXTREMZ_FLAG_PROFILE) keep their events
    // inside the graph, so profiling does not change how a tick launches.
    bool graph = graphs_on_;
    for (const auto& j : slots_)
      if (j.used && !j.waiting && j.pc == PC_SETUP_B) graph = false;
    if (graph) {
      recording_ = true;
      sig_.clear();
      pending_.clear();
      pending_timed_.clear();
      sig_append(profile_ ? profile_mask_ | (1 << 30) : 0);
    }
    int rc = EXTREMZ_OK;
    for (int ph = 0; ph < PC_COUNT && rc == EXTREMZ_OK; ++ph) {
      std::vector<int> sel;
      for (int i = 0; i < kMaxSel; ++i)
        if (slots_[i].used && !slots_[i].waiting && slots_[i].pc == ph) sel.push_back(i);
      if (sel.empty()) continue;
      issued_ = true;
      // A job can reach its first phase that reads the decompressed field in
      // the same tick as its setup, so the wait goes right before that phase.
      if (ph >= PC_CL_DETECT)
        for (int i : sel)
          if (slots_[i].input_ready) {
            EZ_CHECK(cudaStreamWaitEvent(st_, slots_[i].input_ready, 0));
            slots_[i].input_ready = nullptr;
          }
      rc = run_phase(ph, sel);
    }
    recording_ = false;
    if (rc != EXTREMZ_OK) return rc;
    if (graph && !pending_.empty()) EZ_RUN(run_recorded());
    if (!issued_) return EXTREMZ_OK;
    EZ_CHECK(cudaGetLastError());
    // The counter blocks up to the last slot in use (the host reads no other).
    int hi = 0;
    for (int i = 0; i < kMaxSel; ++i)
      if (slots_[i].used) hi = i + 1;
    EZ_CHECK(cudaMemcpyAsync(ctr_host_, ctr_dev_, sizeof(int) * C_COUNT * (size_t)hi,
                             cudaMemcpyDeviceToHost, st_));
    return EXTREMZ_OK;
  }

  // Second half: wait for the counters, then every job's branches.
  int tick_complete() {
    if (!issued_) return EXTREMZ_OK;
    issued_ = false;
    EZ_CHECK(cudaStreamSynchronize(st_));
    fold_timings();
    for (int i = 0; i < kMaxSel; ++i) {
      JobHost<T>& j = slots_[i];
      if (!j.used || j.pc == PC_DONE) continue;
      flush_pending(i);
      if (h(i, C_ERROR)) {
        finish(i, EXTREMZ_DEVICE_TIMEOUT);
        continue;
      }
      if (j.waiting) {
        j.waiting = false;
        EZ_RUN(decide(i));
      }
    }
    return EXTREMZ_OK;
  }

  // Per-class timing of the launches since set_profile(true, ...).
  void collect_profile(extremz_report* rep) {
    if (!recs_.empty()) {
      cudaStreamSynchronize(st_);
      fold_timings();
    }
    if (rep)
      for (int c = 0; c < K_NUM; ++c) {
        rep->prof_ms[c] += prof_ms_[c];
        rep->prof_launches[c] += prof_n_[c];
      }
    reset_timings();
  }
  void drop_profile_events() {
    for (const Rec& r : recs_)
      if (r.owned) {
        pool_.push_back(r.a);
        pool_.push_back(r.b);
      }
    recs_.clear();
    reset_timings();
    for (cudaEvent_t e : pool_) cudaEventDestroy(e);
    pool_.clear();
  }

 private:
  cudaStream_t st_;
  struct Rec { int cls; cudaEvent_t a, b; bool owned; };
  // Tick graphs (see tick_issue).
  bool graphs_on_ = true, recording_ = false, capturing_ = false;
  std::string sig_;
  std::vector<std::function<void(cudaStream_t)>> pending_;
  // Timed launches of the tick being recorded: class, and the event pair the
  // launch records around itself (filled in just before the launches run).
  std::vector<Rec> pending_timed_;
  struct GraphEntry {
    cudaGraphExec_t exec = nullptr;
    unsigned long long last = 0;
    std::vector<Rec> timed;  // events recorded by the graph's timed launches
  };
  std::unordered_map<std::string, GraphEntry> graphs_;
  std::unordered_map<std::string, int> seen_;
  unsigned long long graph_clock_ = 0;
  long long graph_replays_ = 0, graph_captures_ = 0;
  static constexpr size_t kMaxGraphs = 256;
  // A signature is captured at its third sighting: ticks of a single
  // correction repeat many times, while a batch's changing selections often
  // repeat once or twice, where a capture would not pay for itself.
  static constexpr int kCaptureAt = 3;
  cudaStream_t cap_ = nullptr;  // capture stream
  cudaMemPool_t pool_mem_ = nullptr;
  bool ready_ = false, borrowed_ = false, issued_ = false;
  long long tick_id_ = 0;
  int grid_ = 1184;  // grid of the grid-stride kernels for the phase being issued
  int sms_ = 148;
  DeviceTables tb_{};
  Job<T>* jobs_dev_ = nullptr;
  CUtensorMap* maps_dev_ = nullptr;
  int* ctr_dev_ = nullptr;
  int* ctr_host_ = nullptr;
  int static_ctr_host_[C_COUNT * kMaxSel];
  std::vector<JobHost<T>> slots_;
  long long launches_ = 0;
  bool profile_ = false;
  int profile_mask_ = 0;
  // A timed launch: events around it.  Events of a launch inside a captured
  // tick graph belong to the graph (recorded again at every replay, read after
  // the tick's synchronisation); the others return to the pool.
  std::vector<Rec> recs_;
  float prof_ms_[K_NUM] = {};
  int prof_n_[K_NUM] = {};
  void fold_timings() {
    for (const Rec& r : recs_) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, r.a, r.b) != cudaSuccess) {
        cudaGetLastError();
        ms = 0.f;
      }
      prof_ms_[r.cls] += ms;
      prof_n_[r.cls] += 1;
      if (r.owned) {
        pool_.push_back(r.a);
        pool_.push_back(r.b);
      }
    }
    recs_.clear();
  }
  void reset_timings() {
    for (int c = 0; c < K_NUM; ++c) {
      prof_ms_[c] = 0.f;
      prof_n_[c] = 0;
    }
  }
  std::vector<cudaEvent_t> pool_;

  int h(int slot, int c) const { return ctr_host_[(size_t)slot * C_COUNT + c]; }

  cudaEvent_t event() {
    if (!pool_.empty()) {
      cudaEvent_t e = pool_.back();
      pool_.pop_back();
      return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
  }

  template <class A>
  void sig_append(const A& a) {
    sig_.append(reinterpret_cast<const char*>(&a), sizeof(A));
  }
  // A job selection by its used part (kernels read no entry past n): the
  // signature of a one-job tick stays a few hundred bytes to hash.
  void sig_append(const Sel& s) {
    sig_.append(reinterpret_cast<const char*>(&s.n), sizeof(int));
    sig_.append(reinterpret_cast<const char*>(s.idx), sizeof(int) * (size_t)s.n);
    sig_.append(reinterpret_cast<const char*>(s.off), sizeof(int) * (size_t)(s.n + 1));
  }

  template <class... KArgs, class... Args>
  void launch(int cls, void (*kern)(KArgs...), dim3 grid, dim3 block, Args... args) {
    const bool timed = profile_ && (profile_mask_ == 0 || (profile_mask_ >> cls & 1));
    if (recording_) {  // tick graphs: record, launch later as one graph
      sig_append(reinterpret_cast<const void*>(kern));
      sig_append(grid);
      sig_append(block);
      (sig_append(args), ...);
      if (timed) {
        const size_t k = pending_timed_.size();
        pending_timed_.push_back({cls, nullptr, nullptr, false});
        pending_.push_back([=](cudaStream_t s) {
          // In a capture the events become event-record nodes of the graph.
          const Rec& r = pending_timed_[k];
          const unsigned fl = capturing_ ? cudaEventRecordExternal : cudaEventRecordDefault;
          if (r.a) cudaEventRecordWithFlags(r.a, s, fl);
          kern<<<grid, block, 0, s>>>(args...);
          if (r.b) cudaEventRecordWithFlags(r.b, s, fl);
        });
      } else {
        pending_.push_back([=](cudaStream_t s) { kern<<<grid, block, 0, s>>>(args...); });
      }
      ++launches_;
      return;
    }
    cudaEvent_t a = nullptr, b = nullptr;
    if (timed) {
      a = event();
      b = event();
      cudaEventRecord(a, st_);
    }
    kern<<<grid, block, 0, st_>>>(args...);
    ++launches_;
    if (timed) {
      cudaEventRecord(b, st_);
      recs_.push_back({cls, a, b, true});
    }
  }

  // Event pairs for the recorded tick's timed launches, from the pool.
  void arm_timed() {
    for (Rec& r : pending_timed_) {
      r.a = event();
      r.b = event();
      r.owned = true;
    }
  }

  void run_direct(bool timing = true) {
    if (timing) arm_timed();
    for (auto& go : pending_) go(st_);
    pending_.clear();
    for (const Rec& r : pending_timed_)
      if (r.a) recs_.push_back(r);
    pending_timed_.clear();
  }

  // (cudaEventDestroy of an event still pending releases it once it completes.)
  static void release_graph_events(GraphEntry& e) {
    for (const Rec& r : e.timed) {
      cudaEventDestroy(r.a);
      cudaEventDestroy(r.b);
    }
    e.timed.clear();
  }

  void drop_graphs() {
    for (auto& kv : graphs_) {
      if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
      release_graph_events(kv.second);
    }
    graphs_.clear();
    seen_.clear();
    if (cap_) cudaStreamDestroy(cap_);
    cap_ = nullptr;
  }

  // Launches the recorded tick: replays its graph, captures it on the third
  // sighting of its signature, or launches directly.
  int run_recorded() {
    ++graph_clock_;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st_, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
      cudaGetLastError();  // the caller is capturing this stream: launch into it directly
      run_direct(false);   // (untimed: the events would not have run when read)
      return EXTREMZ_OK;
    }
    auto it = graphs_.find(sig_);
    if (it != graphs_.end()) {
      it->second.last = graph_clock_;
      pending_.clear();
      pending_timed_.clear();
      ++graph_replays_;
      EZ_CHECK(cudaGraphLaunch(it->second.exec, st_));
      for (Rec r : it->second.timed) {
        r.owned = false;
        recs_.push_back(r);
      }
      return EXTREMZ_OK;
    }
    if (seen_.size() > 4 * kMaxGraphs) seen_.clear();
    if (++seen_[sig_] < kCaptureAt) {
      run_direct();
      return EXTREMZ_OK;
    }
    if (graphs_.size() >= kMaxGraphs) {  // evict the least recently used
      auto old = graphs_.begin();
      for (auto g = graphs_.begin(); g != graphs_.end(); ++g)
        if (g->second.last < old->second.last) old = g;
      cudaGraphExecDestroy(old->second.exec);
      release_graph_events(old->second);
      graphs_.erase(old);
    }
    // Captured on a private stream (the caller's may be the legacy stream,
    // which cannot be captured), launched on the caller's.
    if (!cap_ && cudaStreamCreateWithFlags(&cap_, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      graphs_on_ = false;
      run_direct();
      return EXTREMZ_OK;
    }
    cudaGraph_t g = nullptr;
    cudaGraphExec_t exec = nullptr;
    if (cudaStreamBeginCapture(cap_, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      cudaGetLastError();
      graphs_on_ = false;
      run_direct();
      return EXTREMZ_OK;
    }
    arm_timed();
    capturing_ = true;
    for (auto& go : pending_) go(cap_);
    capturing_ = false;
    const cudaError_t ec = cudaStreamEndCapture(cap_, &g);
    if (ec != cudaSuccess || !g || cudaGraphInstantiate(&exec, g, 0) != cudaSuccess) {
      cudaGetLastError();
      if (g) cudaGraphDestroy(g);
      graphs_on_ = false;  // capture unavailable here: launch directly from now on
      for (const Rec& r : pending_timed_) {
        pool_.push_back(r.a);
        pool_.push_back(r.b);
      }
      run_direct();
      return EXTREMZ_OK;
    }
    cudaGraphDestroy(g);
    pending_.clear();
    GraphEntry ge{exec, graph_clock_};
    ge.timed = pending_timed_;
    pending_timed_.clear();
    ++graph_captures_;
    EZ_CHECK(cudaGraphLaunch(exec, st_));
    for (Rec r : ge.timed) {
      r.owned = false;
      recs_.push_back(r);
    }
    graphs_[sig_] = std::move(ge);
    return EXTREMZ_OK;
  }

  void free_job(JobHost<T>& j) {
    if (j.used && j.own_arena && j.arena.base) cudaFreeAsync(j.arena.base, st_);
    if (j.used && j.own_arena2 && j.arena2.base) cudaFreeAsync(j.arena2.base, st_);
    j = JobHost<T>();
  }

  // The per-critical-point part of a job's workspace: exact size from the
  // counts, or the rest of borrowed storage.
  int take_cp_storage(JobHost<T>& jh, int ns2, int ns1, int nmax, int nmin, int e2, int e1) {
    if (!jh.own_arena) return EXTREMZ_OK;  // borrowed: carve from the same arena
    const long long need = job_bytes_cps(ns2, ns1, nmax, nmin, e2, e1, sizeof(K));
    void* base = nullptr;
    const cudaError_t e = pool_mem_ ? cudaMallocFromPoolAsync(&base, (size_t)need, pool_mem_, st_)
                                    : cudaMallocAsync(&base, (size_t)need, st_);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return EXTREMZ_OOM;
    }
    jh.arena2.base = static_cast<char*>(base);
    jh.arena2.cap = (size_t)need;
    jh.arena2.used = 0;
    jh.arena2.fixed = true;
    jh.own_arena2 = true;
    return EXTREMZ_OK;
  }

  Sel make_sel(const std::vector<int>& slots, bool tiles) const {
    Sel s;
    std::memset(&s, 0, sizeof(s));
    s.n = (int)slots.size();
    int off = 0;
    for (int k = 0; k < s.n; ++k) {
      s.idx[k] = slots[k];
      s.off[k] = off;
      if (tiles) off += slots_[slots[k]].ntiles;
    }
    s.off[s.n] = off;
    return s;
  }

  void ctl(const Sel& s, int op) { launch(K_OTHER, k_ctl<T>, 1, 64, jobs_dev_, s, op); }

  // ------------------------------------------------------------- phases --
  int run_phase(int ph, const std::vector<int>& sel) {
    int bps = 1;  // jobs share launches: the largest knob of the selection
    for (int i : sel) bps = std::max(bps, slots_[i].blocks_per_sm);
    grid_ = sms_ * bps;
    if (ph == PC_CL_ROUND || ph == PC_RLOOPS || ph == PC_SLOOPS || ph == PC_SADDLE ||
        ph == PC_SLOOPS_J || ph == PC_SADDLE_J || ph == PC_FINAL_JOIN)
      for (int i : sel) slots_[i].applied_tick = tick_id_;  // phases that apply edits
    const Sel s = make_sel(sel, false);
    const Sel st = make_sel(sel, true);
    const Job<T>* jobs = jobs_dev_;
    switch (ph) {
      case PC_SETUP_A:
        launch(K_SETUP, k_direction<T, false>, st.off[st.n], 256, jobs, st);
        launch(K_SETUP, k_jump2<T, false>, grid_, 256, jobs, s);
        for (int i : sel) {
          JobHost<T>& j = slots_[i];
          launch(K_OTHER, k_cp_count, (j.nb + kCpWarps - 1) / kCpWarps, 32 * kCpWarps,
                 (const int8_t*)j.J.otype, (const uint16_t*)j.J.olm, j.J.dim, j.nb, j.bcount);
          EZ_RUN(scan_counts(j.bcount, j.nb, 6, j.J.ctr + C_NS2, j.chunk));
          j.waiting = true;
        }
        return EXTREMZ_OK;
      case PC_SETUP_B:
        for (int i : sel) {
          const int rc = setup_b(i);
          if (rc == EXTREMZ_OOM) {  // this job ends; the others go on
            finish(i, EXTREMZ_OOM);
            continue;
          }
          if (rc != EXTREMZ_OK) return rc;
          if (slots_[i].p.flags & kFlagAnalysis) finish(i, EXTREMZ_OK);
          else slots_[i].pc = PC_CL_DETECT;
        }
        return EXTREMZ_OK;
      case PC_CL_DETECT:
        detect(sel);
        for (int i : sel) slots_[i].waiting = true;
        return EXTREMZ_OK;
      case PC_CL_ROUND:
        ctl(s, OP_ZERO_TOUCHED);
        launch(K_PROPOSE, k_propose_cp<T>, grid_, 256, jobs, s);
        launch(K_APPLY, k_apply<T>, grid_, 256, jobs, s);
        detect(sel);
        for (int i : sel) slots_[i].waiting = true;
        return EXTREMZ_OK;
      case PC_RLOOPS:
        ctl(s, OP_ZERO_TOUCHED);
        launch(K_FIXPATH, k_fixpath<T, true>, grid_, 256, jobs, s);
        launch(K_FIXPATH, k_fixpath<T, false>, grid_, 256, jobs, s);
        launch(K_APPLY, k_apply<T>, grid_, 256, jobs, s);
        for (int i : sel) slots_[i].pc = PC_MANIFOLD;
        return EXTREMZ_OK;
      case PC_MANIFOLD: {
        // Jobs known on the host to have no value change since their last
        // manifold round began (no edit in the counters of the last tick, none
        // issued in this one) get only the round's bookkeeping; their kernels
        // would return at once.  The others run the round (whose kernels
        // check again on the device).
        std::vector<int> quiet, busy;
        for (int i : sel) {
          const JobHost<T>& j = slots_[i];
          const bool known_clean =
              j.manifold_rounds > 0 && j.applied_tick != tick_id_ && h(i, C_CHANGED) == 0;
          (known_clean ? quiet : busy).push_back(i);
        }
        if (!quiet.empty()) ctl(make_sel(quiet, false), OP_MF_BEGIN);
        if (!busy.empty()) {
          const Sel bs = make_sel(busy, false), bt = make_sel(busy, true);
          ctl(bs, OP_MF_BEGIN);
          // Steepest pointers: every tile in a job's first round, one block
          // per tile; in later rounds the tiles that changed, listed first,
          // then taken by a fixed grid (a launch of one block per tile of
          // the field costs more than the few changed tiles).
          std::vector<int> fresh, later;
          for (int i : busy) (slots_[i].manifold_rounds == 0 ? fresh : later).push_back(i);
          if (!fresh.empty()) {
            const Sel ft = make_sel(fresh, true);
            launch(K_DIRECTION_FIRST, k_direction<T, true>, ft.off[ft.n], 256, jobs, ft);
          }
          if (!later.empty()) {
            const Sel ls = make_sel(later, false), lt = make_sel(later, true);
            const int ntiles = lt.off[lt.n];
            launch(K_DIRECTION, k_tile_list<T>,
                   std::max(1, std::min((ntiles + 255) / 256, 2 * sms_)), 256, jobs, ls);
            launch(K_DIRECTION, k_direction_list<T>, std::max(1, std::min(ntiles, 4 * sms_)),
                   256, jobs, ls);
          }
          if (!fresh.empty())
            launch(K_JUMP_FIRST, k_jump2<T, true, false>, grid_, 256, jobs, make_sel(fresh, false));
          if (!later.empty())
            launch(K_JUMP, k_jump2<T, true, true>, grid_, 256, jobs, make_sel(later, false));
          launch(K_OTHER, k_clear_changed<T>, grid_, 256, jobs, bs);
          launch(K_ROWS, k_saddle_pass<T>, grid_, 256, jobs, bs);
          bool vote = false;
          // Lockstep jobs: the fourteen steps in one block per job when the
          // job's previous round had short candidate lists (the counts of
          // that round are still in the host copy of its counters), else one
          // grid launch per step.  Either is exact for any list length.
          std::vector<int> lock_small, lock_large;
          for (int i : busy) {
            if (!slots_[i].J.wn_lockstep) {
              vote = true;
              continue;
            }
            const bool small = slots_[i].manifold_rounds > 0 &&
                               h(i, C_CAND) + h(i, C_CANDJ) <= kWnBlockMax;
            (small ? lock_small : lock_large).push_back(i);
          }
          if (vote) {
            wn_rounds<true>(bs);  // its completion brings in the join side's list
            wn_rounds<false>(bs);
          }
          if (!lock_small.empty()) {
            const Sel ss = make_sel(lock_small, false);
            launch(K_WRONG_NBR, k_wn_steps_block<T>, ss.n, 1024, jobs, ss);
          }
          if (!lock_large.empty()) {
            const Sel sl = make_sel(lock_large, false);
            const int grid = std::min(grid_, 2 * sms_);
            for (int d = 0; d < kNumDirs; ++d)
              launch(K_WRONG_NBR, k_wn_step<T>, grid, 256, jobs, sl, d);
          }
        }
        for (int i : sel) {
          slots_[i].manifold_rounds++;
          slots_[i].waiting = true;
        }
        return EXTREMZ_OK;
      }
      case PC_SLOOPS:
        ctl(s, OP_SLOOPS_BEGIN);
        launch(K_OTHER, k_wim_scan<T, true>, grid_, 256, jobs, s);
        launch(K_OTHER, k_wim_collect<T, true>, grid_, 256, jobs, s, 1);
        launch(K_APPLY, k_apply<T>, grid_, 256, jobs, s);
        for (int i : sel) slots_[i].waiting = true;
        return EXTREMZ_OK;
      case PC_SADDLE:
        ctl(s, OP_SADDLE_BEGIN);
        launch(K_OTHER, k_wis_mark<T, true>, grid_, 256, jobs, s);
        launch(K_OTHER, k_wis_update<T, true>, grid_, 256, jobs, s);
        launch(K_OTHER, k_wis_long<T, true>, 2 * sms_, 256, jobs, s);
        launch(K_OTHER, k_wis_collect<T, true>, grid_, 256, jobs, s, 1);
        launch(K_APPLY, k_apply<T>, grid_, 256, jobs, s);
        for (int i : sel) {
          slots_[i].pending.push_back(PH_SADDLE);
          slots_[i].pc = joinb(slots_[i]);
        }
        return EXTREMZ_OK;
      case PC_SLOOPS_J:
        ctl(s, OP_SLOOPS_JOIN_BEGIN);
        launch(K_OTHER, k_wim_scan<T, false>, grid_, 256, jobs, s);
        launch(K_OTHER, k_wim_collect<T, false>, grid_, 256, jobs, s, 1);
        launch(K_OTHER, k_wim_min2_scan<T>, grid_, 256, jobs, s);
        launch(K_OTHER, k_wim_min2_collect<T>, grid_, 256, jobs, s);
        launch(K_APPLY, k_apply<T>, grid_, 256, jobs, s);
        for (int i : sel) slots_[i].waiting = true;
        return EXTREMZ_OK;
      case PC_SADDLE_J:
      case PC_FINAL_JOIN:
        ctl(s, OP_SADDLE_JOIN_BEGIN);
        launch(K_OTHER, k_wis_mark<T, false>, grid_, 256, jobs, s);
        launch(K_OTHER, k_wis_update<T, false>, grid_, 256, jobs, s);
        launch(K_OTHER, k_wis_long<T, false>, 2 * sms_, 256, jobs, s);
        launch(K_OTHER, k_wis_collect<T, false>, grid_, 256, jobs, s, 1);
        launch(K_APPLY, k_apply<T>, grid_, 256, jobs, s);
        for (int i : sel) {
          slots_[i].pending.push_back(PH_SADDLE_JOIN);
          if (ph == PC_SADDLE_J) slots_[i].pc = endb(slots_[i]);
          else slots_[i].waiting = true;
        }
        return EXTREMZ_OK;
      case PC_PRE_END:
        for (int i : sel) slots_[i].waiting = true;
        return EXTREMZ_OK;
      case PC_DET3:
        ctl(s, OP_DETECT3_BEGIN);
        launch(K_OTHER, k_wim_scan<T, true>, grid_, 256, jobs, s);
        launch(K_OTHER, k_wim_collect<T, true>, grid_, 256, jobs, s, 0);
        launch(K_OTHER, k_wis_mark<T, true>, grid_, 256, jobs, s);
        launch(K_OTHER, k_wis_update<T, true>, grid_, 256, jobs, s);
        launch(K_OTHER, k_wis_long<T, true>, 2 * sms_, 256, jobs, s);
        launch(K_OTHER, k_wis_collect<T, true>, grid_, 256, jobs, s, 0);
        for (int i : sel) {
          slots_[i].pending.push_back(PH_DETECT3);
          slots_[i].pc = (slots_[i].p.flags & kFlagCensus) ? PC_DET3J : join3(slots_[i]);
        }
        return EXTREMZ_OK;
      case PC_DET3J:
        ctl(s, OP_DETECT3_JOIN_BEGIN);
        launch(K_OTHER, k_wim_scan<T, false>, grid_, 256, jobs, s);
        launch(K_OTHER, k_wim_collect<T, false>, grid_, 256, jobs, s, 0);
        launch(K_OTHER, k_wis_mark<T, false>, grid_, 256, jobs, s);
        launch(K_OTHER, k_wis_update<T, false>, grid_, 256, jobs, s);
        launch(K_OTHER, k_wis_long<T, false>, 2 * sms_, 256, jobs, s);
        launch(K_OTHER, k_wis_collect<T, false>, grid_, 256, jobs, s, 0);
        for (int i : sel) slots_[i].pc = PC_FINAL_DETECT;
        return EXTREMZ_OK;
      case PC_FINAL_DETECT:
        detect(sel);
        for (int i : sel) slots_[i].waiting = true;
        return EXTREMZ_OK;
      default:
        return EXTREMZ_OK;
    }
  }

  // Mismatch detection: dense the first time a job detects, then incremental
  // over the neighbourhoods of the vertices changed since.
  void detect(const std::vector<int>& sel) {
    std::vector<int> dense, incr;
    for (int i : sel) (slots_[i].dense_done ? incr : dense).push_back(i);
    if (!dense.empty()) {
      const Sel s = make_sel(dense, false), st = make_sel(dense, true);
      ctl(s, OP_DETECT_DENSE_BEGIN);
      launch(K_DETECT, k_classify<T, true>, st.off[st.n], 256, (const Job<T>*)jobs_dev_, st);
      ctl(s, OP_DETECT_END_DENSE);
      for (int i : dense) slots_[i].dense_done = true;
    }
    if (!incr.empty()) {
      const Sel s = make_sel(incr, false);
      ctl(s, OP_DETECT_BEGIN);
      launch(K_DETECT, k_redetect<T>, grid_, 256, (const Job<T>*)jobs_dev_, s);
      launch(K_DETECT, k_keep<T>, grid_, 256, (const Job<T>*)jobs_dev_, s);
      ctl(s, OP_DETECT_END);
    }
  }

  // Three grid-wide arbitration rounds and the per-job completion rounds of
  // the candidate list being resolved (one side).
  template <bool kSplit>
  void wn_rounds(const Sel& s) {
    const Job<T>* jobs = jobs_dev_;
    // Candidate lists are short next to the field (a few per cent of the
    // saddles at most), so two blocks per SM cover them.
    const int grid = std::min(grid_, 2 * sms_);
    for (int r = 0; r < kWnGridRounds; ++r) {
      launch(K_WRONG_NBR, k_wn_vote<T, kSplit>, grid, 256, jobs, s, r);
      launch(K_WRONG_NBR, k_wn_commit<T, kSplit>, grid, 256, jobs, s, r);
    }
    launch(K_WRONG_NBR, k_wn_resolve<T, kSplit>, s.n, 1024, jobs_dev_, s);
  }

  // Exclusive scan of nl lists of n counts each (list l at c + l * n), the
  // list totals into totals[0 .. nl); chunk holds nl * ceil(n / 1024) sums.
  int scan_counts(int* c, int n, int nl, int* totals, int* chunk) {
    const int nc = (n + 1023) / 1024;
    launch(K_OTHER, k_chunk_sums, dim3(nc, nl), 1024, (const int*)c, n, chunk);
    launch(K_OTHER, k_scan_lists, 1, 1024, chunk, nc, nl, totals);
    launch(K_OTHER, k_chunk_scan, dim3(nc, nl), 1024, c, n, (const int*)chunk);
    return EXTREMZ_OK;
  }

  // Per-extremum entry counts cnt[0 .. n) into offsets (the total into cnt[n])
  // and a copy of the offsets into cur, the fill cursors.
  int entry_lists(int* cnt, int* cur, int n, int* chunk) {
    EZ_RUN(scan_counts(cnt, n, 1, cnt + n, chunk));
    EZ_CHECK(cudaMemcpyAsync(cur, cnt, (size_t)n * 4, cudaMemcpyDeviceToDevice, st_));
    return EXTREMZ_OK;
  }

  int setup_b(int slot) {
    JobHost<T>& jh = slots_[slot];
    Job<T>& J = jh.J;
    const int N = J.dim.N;
    const int ns2 = h(slot, C_NS2), ns1 = h(slot, C_NS1), nmax = h(slot, C_NMAX),
              nmin = h(slot, C_NMIN), e2 = h(slot, C_E2), e1 = h(slot, C_E1);
    EZ_RUN(take_cp_storage(jh, ns2, ns1, nmax, nmin, e2, e1));
    Arena& A = jh.own_arena2 ? jh.arena2 : jh.arena;
    J.sad2 = A.take<int>(ns2);
    J.sad1 = A.take<int>(ns1);
    J.maxima = A.take<int>(nmax);
    J.minima = A.take<int>(nmin);
    J.orow2 = A.take<int>((long long)ns2 * kRowStride);
    J.orm2 = A.take<int4>(ns2);
    J.oend2 = A.take<int4>(ns2);
    J.drow2 = A.take<int>((long long)ns2 * 2);
    J.ocnt2 = A.take<uint8_t>(ns2);
    J.orow1 = A.take<int>((long long)ns1 * kRowStride);
    J.orm1 = A.take<int4>(ns1);
    J.oend1 = A.take<int4>(ns1);
    J.drow1 = A.take<int>((long long)ns1 * 2);
    J.ocnt1 = A.take<uint8_t>(ns1);
    J.has2 = A.take<uint8_t>(ns2);
    J.has1 = A.take<uint8_t>(ns1);
    J.largest = A.take<int>(nmax);
    J.first1 = A.take<int>(nmax);
    J.flag2 = A.take<int>(nmax);
    J.first_s = A.take<int>(nmax);
    J.smallest = A.take<int>(nmin);
    J.first_min1 = A.take<int>(nmin);
    J.flag_min2 = A.take<int>(nmin);
    J.first_sj = A.take<int>(nmin);
    const int ne = std::max(nmax, nmin);
    J.ext_key = A.take<K>(ne);
    J.ext_id = A.take<int>(ne);
    jh.checksum = A.take<unsigned long long>(8);
    J.moff2 = A.take<int>(nmax + 1);
    J.ment2 = A.take<int>(e2);
    J.wstamp2 = A.take<int>(nmax);
    J.moff1 = A.take<int>(nmin + 1);
    J.ment1 = A.take<int>(e1);
    J.wstamp1 = A.take<int>(nmin);
    J.aff = A.take<int>(ne);
    J.wlong = A.take<int>(ne);
    int* chunk = A.take<int>(ne / 1024 + 2);
    if (!jh.checksum || !J.ext_id || !J.ocnt1 || !J.first_sj || !chunk) return EXTREMZ_OOM;
    launch(K_OTHER, k_cp_write, (jh.nb + kCpWarps - 1) / kCpWarps, 32 * kCpWarps,
           (const int8_t*)J.otype, N, jh.nb, (const int*)jh.bcount,
           J.sad2, J.sad1, J.maxima, J.minima);
    launch(K_OTHER, k_ext_index<T>, grid_, 256, J);
    // Per side: the rows (with their compact copies, each named extremum's
    // extreme saddle key and entry count), the entry lists' offsets, then the
    // extreme saddle ids and the entries.  The sides share the selection
    // scratch (ext_key, ext_id), so they go one after the other.  Rows name
    // only extrema, so a side with rows has extrema.
    if (nmax) {
      launch(K_OTHER, k_fill<K>, grid_, 256, J.ext_key, K(0), (long long)nmax);
      launch(K_OTHER, k_fill<int>, grid_, 256, J.ext_id, -1, (long long)nmax);
      EZ_CHECK(cudaMemsetAsync(J.moff2, 0, (size_t)(nmax + 1) * 4, st_));
    }
    launch(K_SETUP, k_rows<T, true>, grid_, 256, J, J.f, (const int*)J.ds, (const int*)J.sad2,
           (int)C_NS2, J.orow2, J.ocnt2, J.orm2, J.oend2);
    if (nmax) {
      EZ_RUN(entry_lists(J.moff2, J.wstamp2, nmax, chunk));
      launch(K_OTHER, k_extreme_saddle<T, true>, grid_, 256, J);
      EZ_CHECK(cudaMemsetAsync(J.wstamp2, 0, (size_t)nmax * 4, st_));
      EZ_CHECK(cudaMemcpyAsync(J.largest, J.ext_id, nmax * 4, cudaMemcpyDeviceToDevice, st_));
      launch(K_OTHER, k_fill<int>, grid_, 256, J.first1, kInf, (long long)nmax);
      launch(K_OTHER, k_fill<int>, grid_, 256, J.first_s, kInf, (long long)nmax);
      EZ_CHECK(cudaMemsetAsync(J.flag2, 0, nmax * 4, st_));
    }
    if (nmin) {
      launch(K_OTHER, k_fill<K>, grid_, 256, J.ext_key, ~K(0), (long long)nmin);
      launch(K_OTHER, k_fill<int>, grid_, 256, J.ext_id, kInf, (long long)nmin);
      EZ_CHECK(cudaMemsetAsync(J.moff1, 0, (size_t)(nmin + 1) * 4, st_));
    }
    launch(K_SETUP, k_rows<T, false>, grid_, 256, J, J.f, (const int*)J.as, (const int*)J.sad1,
           (int)C_NS1, J.orow1, J.ocnt1, J.orm1, J.oend1);
    if (nmin) {
      EZ_RUN(entry_lists(J.moff1, J.wstamp1, nmin, chunk));
      launch(K_OTHER, k_extreme_saddle<T, false>, grid_, 256, J);
      EZ_CHECK(cudaMemsetAsync(J.wstamp1, 0, (size_t)nmin * 4, st_));
      EZ_CHECK(cudaMemcpyAsync(J.smallest, J.ext_id, nmin * 4, cudaMemcpyDeviceToDevice, st_));
      launch(K_OTHER, k_fill<int>, grid_, 256, J.ext_id, kInf, (long long)nmin);
      launch(K_OTHER, k_fill<int>, grid_, 256, J.first_min1, kInf, (long long)nmin);
      launch(K_OTHER, k_fill<int>, grid_, 256, J.first_sj, kInf, (long long)nmin);
      EZ_CHECK(cudaMemsetAsync(J.flag_min2, 0, nmin * 4, st_));
    }
    // Decompressed row slots start at zero: the reference's rows are fresh
    // cudaMalloc memory read before first written (:5338-5341, :3128-3130).
    if (ns2) EZ_CHECK(cudaMemsetAsync(J.drow2, 0, (size_t)ns2 * 2 * 4, st_));
    if (ns1) EZ_CHECK(cudaMemsetAsync(J.drow1, 0, (size_t)ns1 * 2 * 4, st_));
    // Every tile's pointers are computed in the first manifold round.
    EZ_CHECK(cudaMemsetAsync(J.tdirty, 1, (size_t)jh.ntiles, st_));
    // Block stamps start below the first round's; no root is touched.
    EZ_CHECK(cudaMemsetAsync(J.bdirty, 0, (size_t)jh.nb * 4, st_));
    EZ_CHECK(cudaMemsetAsync(J.rtouch2, 0, (size_t)((N + 31) / 32) * 4, st_));
    EZ_CHECK(cudaMemsetAsync(J.rtouch1, 0, (size_t)((N + 31) / 32) * 4, st_));
    // Proposal buffer at the sentinel, edit counters at -1 (:5082), stamps 0.
    launch(K_OTHER, k_fill<K>, grid_, 256, J.delta, J.sentinel_key, (long long)N);
    launch(K_OTHER, k_fill<int>, grid_, 256, J.counter, -1, (long long)N);
    EZ_CHECK(cudaMemsetAsync(J.claim, 0, (size_t)N * 8, st_));
    EZ_CHECK(cudaMemsetAsync(J.taken, 0, (size_t)N * 4, st_));
    EZ_CHECK(cudaMemsetAsync(J.taken1, 0, (size_t)N * 4, st_));
    EZ_CHECK(cudaMemsetAsync(J.dstamp, 0, (size_t)N * 4, st_));
    EZ_CHECK(cudaMemsetAsync(J.rstamp, 0, (size_t)N * 4, st_));
    EZ_CHECK(cudaMemsetAsync(J.vchg, 0xff, (size_t)((N + 31) / 32) * 4, st_));
    EZ_CHECK(cudaMemsetAsync(J.wchg2, 0, (size_t)((N + 31) / 32) * 4, st_));
    EZ_CHECK(cudaMemsetAsync(J.wchg1, 0, (size_t)((N + 31) / 32) * 4, st_));
    EZ_CHECK(cudaMemcpyAsync(jobs_dev_ + slot, &J, sizeof(J), cudaMemcpyHostToDevice, st_));
    return EXTREMZ_OK;
  }

  // ----------------------------------------------------------- branches --
  // Immediate successors (no counter needed).
  int after_cl(JobHost<T>& j) {
    if (j.block == 1) return PC_RLOOPS;
    return PC_MANIFOLD;
  }
  int joinb(JobHost<T>& j) {
    if (j.nfc1 == 0 && j.p.preserve_join) return PC_SLOOPS_J;
    return endb(j);
  }
  int endb(JobHost<T>& j) {
    if (j.block == 0) return PC_PRE_END;
    j.block += 1;  // block 1 -> 2, 2 -> 3
    j.rounds = 0;
    return PC_CL_DETECT;
  }
  int join3(JobHost<T>& j) {
    if (j.nfc1 == 0 && j.p.preserve_join) return PC_DET3J;
    return PC_FINAL_DETECT;
  }

  void finish(int slot, int status) {
    JobHost<T>& j = slots_[slot];
    j.status = status;
    j.pc = PC_DONE;
  }

  void flush_pending(int slot) {
    JobHost<T>& j = slots_[slot];
    for (int ph : j.pending) {
      if (ph == PH_SADDLE) j.emit(PH_SADDLE, h(slot, C_WSC));
      else if (ph == PH_SADDLE_JOIN) j.emit(PH_SADDLE_JOIN, h(slot, C_WSCJ));
      else if (ph == PH_DETECT3) j.emit(PH_DETECT3, h(slot, C_WSC), h(slot, C_WMC), h(slot, C_WMC2));
    }
    j.pending.clear();
  }

  void snapshot(int slot) {
    JobHost<T>& j = slots_[slot];
    const int v[11] = {j.nfc, j.nfc1, h(slot, C_CMAX), h(slot, C_CMIN), h(slot, C_CSAD),
                       h(slot, C_WMC), h(slot, C_WMC2), h(slot, C_WSC), h(slot, C_WMIN),
                       h(slot, C_WMIN2), h(slot, C_WSCJ)};
    std::memcpy(j.c, v, sizeof(v));
  }

  int loop_test(int slot) {
    JobHost<T>& j = slots_[slot];
    bool any = false;
    for (int i = 0; i < 11; ++i) any |= j.c[i] > 0;
    if (!any) {
      if (j.p.final_join) j.pc = PC_FINAL_JOIN;
      else finish(slot, EXTREMZ_OK);
      return EXTREMZ_OK;
    }
    if (j.outer >= j.p.max_outer) {
      finish(slot, EXTREMZ_ROUND_CAP);
      return EXTREMZ_OK;
    }
    j.outer += 1;
    j.block = 1;
    j.rounds = 0;
    j.pc = PC_CL_DETECT;
    return EXTREMZ_OK;
  }

  int checksum_emit(int slot) {
    JobHost<T>& j = slots_[slot];
    if (!j.trace) return EXTREMZ_OK;
    EZ_CHECK(cudaMemsetAsync(j.checksum, 0, 8, st_));
    launch(K_OTHER, k_checksum<T>, grid_, 256, (const T*)j.J.g, j.J.dim.N, j.checksum);
    unsigned long long hsum = 0;
    EZ_CHECK(cudaMemcpyAsync(&hsum, j.checksum, 8, cudaMemcpyDeviceToHost, st_));
    EZ_CHECK(cudaStreamSynchronize(st_));
    j.emit(PH_CHECKSUM, (int)(hsum & 0x7fffffff), (int)((hsum >> 31) & 0x7fffffff));
    return EXTREMZ_OK;
  }

  // Branch of a job that stopped at a counter-dependent point.
  int decide(int slot) {
    JobHost<T>& j = slots_[slot];
    switch (j.pc) {
      case PC_SETUP_A:
        j.pc = PC_SETUP_B;
        return EXTREMZ_OK;
      case PC_CL_DETECT:
      case PC_CL_ROUND:
        j.emit(PH_CLOOP_DETECT, h(slot, C_CMAX), h(slot, C_CMIN), h(slot, C_CSAD));
        if (j.p.flags & kFlagCensus) {  // no edit: on to the third block's checks
          j.block = 3;
          j.pc = PC_MANIFOLD;
          return EXTREMZ_OK;
        }
        if (h(slot, C_MM) > 0) {
          if (j.rounds >= j.p.max_cloop_rounds) {
            finish(slot, EXTREMZ_ROUND_CAP);
            return EXTREMZ_OK;
          }
          j.rounds += 1;
          j.cloop_total += 1;
          j.pc = PC_CL_ROUND;
        } else {
          j.pc = after_cl(j);
        }
        return EXTREMZ_OK;
      case PC_MANIFOLD:
        j.nfc = h(slot, C_NFC);
        j.nfc1 = h(slot, C_NFC1);
        j.emit(PH_WRONG_NBR, j.nfc, j.nfc1);
        if (j.p.flags & kFlagCensus) j.pc = PC_DET3;
        else if (j.block == 3) j.pc = j.nfc == 0 ? PC_DET3 : join3(j);
        else j.pc = j.nfc == 0 ? PC_SLOOPS : joinb(j);
        return EXTREMZ_OK;
      case PC_SLOOPS:
        // s_loops refreshes the file-scope host copies (:3473-3476).
        j.emit(PH_SLOOPS, h(slot, C_WMC), h(slot, C_WMC2));
        j.pc = h(slot, C_WMC) == 0 ? PC_SADDLE : joinb(j);
        return EXTREMZ_OK;
      case PC_SLOOPS_J:
        j.emit(PH_SLOOPS_JOIN, h(slot, C_WMIN), h(slot, C_WMIN2));
        j.pc = h(slot, C_WMIN) == 0 ? PC_SADDLE_J : endb(j);
        return EXTREMZ_OK;
      case PC_PRE_END:  // :5589-5599
        snapshot(slot);
        return loop_test(slot);
      case PC_FINAL_DETECT:
        j.emit(PH_CLOOP_DETECT, h(slot, C_CMAX), h(slot, C_CMIN), h(slot, C_CSAD));
        snapshot(slot);
        if (j.p.flags & kFlagCensus) {
          finish(slot, EXTREMZ_OK);
          return EXTREMZ_OK;
        }
        j.emit(PH_OUTER, j.outer);
        EZ_RUN(checksum_emit(slot));
        return loop_test(slot);
      case PC_FINAL_JOIN:
        finish(slot, EXTREMZ_OK);
        return EXTREMZ_OK;
      default:
        return EXTREMZ_OK;
    }
  }
};

}  // namespace extremz

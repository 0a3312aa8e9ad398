// Host engine of the ExtreM correction and its C ABI (include/extremz.h).
//
// The engine runs the reference GPU driver's control flow (src/ExtreM_cuda.cu
// main() :5508-5997) on one CUDA stream: setup, hot loop #1 (c_loops), the
// outer loop of three blocks and the final join-saddle pass.  Every kernel is a
// grid-stride loop over a device-resident count, so no launch shape depends on
// a host copy of a counter; the host reads the counter block only where the
// reference's control flow branches on it.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/extremz.h"
#include "extremz_kernels.cuh"
#include "extremz_lut.h"

namespace extremz {

#define EZ_CHECK(call)                                  \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) {                            \
      last_cuda_error() = e_;                           \
      return EXTREMZ_CUDA_ERR;                          \
    }                                                   \
  } while (0)

cudaError_t& last_cuda_error() {
  static thread_local cudaError_t e = cudaSuccess;
  return e;
}

// Device copies of the lookup tables, one per device, built on first use.
struct DeviceLut {
  int8_t* lut = nullptr;
  int* key_offset = nullptr;
  bool ready = false;
};

static std::mutex g_lut_mu;
static DeviceLut g_lut[64];

static int device_tables(DeviceTables* out) {
  int dev = 0;
  EZ_CHECK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return EXTREMZ_BAD_ARG;
  std::lock_guard<std::mutex> lk(g_lut_mu);
  DeviceLut& d = g_lut[dev];
  if (!d.ready) {
    static HostTables* host = [] {
      HostTables* t = new HostTables;
      build_tables(*t);
      return t;
    }();
    EZ_CHECK(cudaMalloc(&d.lut, kLutSize));
    EZ_CHECK(cudaMalloc(&d.key_offset, 64 * sizeof(int)));
    EZ_CHECK(cudaMemcpy(d.lut, host->lut, kLutSize, cudaMemcpyHostToDevice));
    EZ_CHECK(cudaMemcpy(d.key_offset, host->key_offset, 64 * sizeof(int), cudaMemcpyHostToDevice));
    d.ready = true;
  }
  out->lut = d.lut;
  out->key_offset = d.key_offset;
  return EXTREMZ_OK;
}

const HostTables& host_tables() {
  static HostTables* t = [] {
    HostTables* p = new HostTables;
    build_tables(*p);
    return p;
  }();
  return *t;
}

// ---------------------------------------------------------------------------
// Tensor maps for the TMA halo tiles.  The encoder comes from the driver
// through the runtime, so the library does not link libcuda directly.
// ---------------------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
    }
    return (PFN_cuTensorMapEncodeTiled_v12000)p;
  }();
  return fn;
}

// A 3-D map of the field with the halo-tile box; false when TMA cannot be
// used (base not 16-byte aligned, or a row stride that is not a multiple of
// 16 bytes), in which case the kernels load tiles with plain loads.
template <class T>
static bool make_tile_map(CUtensorMap* m, const T* ptr, const Dims& g) {
  std::memset(m, 0, sizeof(*m));
  if ((reinterpret_cast<uintptr_t>(ptr) & 15) || ((size_t)g.W * sizeof(T)) % 16) return false;
  auto fn = tensor_map_encoder();
  if (!fn) return false;
  cuuint64_t dims[3] = {(cuuint64_t)g.W, (cuuint64_t)g.H, (cuuint64_t)g.D};
  cuuint64_t strides[2] = {(cuuint64_t)g.W * sizeof(T), (cuuint64_t)g.W * g.H * sizeof(T)};
  cuuint32_t box[3] = {(cuuint32_t)SX, (cuuint32_t)SY, (cuuint32_t)SZ};
  cuuint32_t es[3] = {1, 1, 1};
  CUresult r = fn(m, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                  3, const_cast<T*>(ptr), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// ---------------------------------------------------------------------------
// Workspace: one device arena per context, grown on demand.
// ---------------------------------------------------------------------------
struct Arena {
  char* base = nullptr;
  size_t cap = 0, used = 0;
  bool fixed = false;  // borrowed storage: never freed or grown
  int reserve(size_t bytes) {
    if (bytes <= cap) return EXTREMZ_OK;
    if (fixed) return EXTREMZ_OOM;
    if (base) cudaFree(base);
    base = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&base, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return EXTREMZ_OOM;
    }
    cap = bytes;
    return EXTREMZ_OK;
  }
  template <class P>
  P* take(size_t count) {
    size_t bytes = (count * sizeof(P) + 255) & ~size_t(255);
    if (used + bytes > cap) return nullptr;
    P* p = reinterpret_cast<P*>(base + used);
    used += bytes;
    return p;
  }
};

struct Context {
  int device = 0;
  bool has_tables = false;  // tables given by the owner instead of device_tables()
  DeviceTables tables{};
  Arena arena;
  Arena stage;           // device copies of host fields (extremz_correct_host)
  int* h_ctr = nullptr;  // pinned copy of the counter block
  unsigned long long wn_round = 0;
  int wn_stamp = 0;
  ~Context() {
    if (arena.base && !arena.fixed) cudaFree(arena.base);
    if (stage.base) cudaFree(stage.base);
    if (h_ctr) cudaFreeHost(h_ctr);
  }
};

// Kernel classes for the optional per-class timing (extremz_report.prof_*).
enum KClass : int {
  K_SETUP = 0, K_DETECT, K_DIRECTION, K_JUMP, K_PROPOSE, K_APPLY, K_ROWS, K_WRONG_NBR,
  K_FIXPATH, K_OTHER, K_NUM
};

// Phases of the trace (same records as the oracle's trace).
enum Phase : int {
  PH_CLOOP_DETECT = 1, PH_WRONG_NBR = 2, PH_SLOOPS = 3, PH_SADDLE = 4, PH_DETECT3 = 5,
  PH_SLOOPS_JOIN = 6, PH_SADDLE_JOIN = 7, PH_OUTER = 8, PH_CHECKSUM = 9
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

template <class T>
class Corrector {
 public:
  using K = typename KeyOf<T>::K;

  Corrector(Context& ctx, const T* f, T* g, int W, int H, int D, const extremz_params& p,
            cudaStream_t st, int32_t* trace, int trace_cap)
      : ctx_(ctx), p_(p), st_(st), trace_(trace), trace_cap_(trace_cap) {
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
    profile_ = (p.flags & EXTREMZ_FLAG_PROFILE) != 0;
    const bool tma_ok = (p.flags & EXTREMZ_FLAG_NO_TMA) == 0;
    tma_f_ = tma_ok && make_tile_map(&map_f_, f, J.dim);
    tma_g_ = tma_ok && make_tile_map(&map_g_, (const T*)g, J.dim);
    profile_mask_ = (p.flags >> EXTREMZ_PROFILE_CLASS_SHIFT) & ((1 << K_NUM) - 1);
  }

  int run(extremz_report* rep) {
    int rc = setup();
    if (rc != EXTREMZ_OK) return rc;
    rc = main_loop();
    if (rep) {
      rep->status = rc;
      rep->outer_iters = outer_;
      rep->cloop_rounds = cloop_rounds_;
      rep->manifold_rounds = manifold_rounds_;
      std::memcpy(rep->counters, hc_, sizeof(hc_));
      rep->error_bits = ctx_.h_ctr[C_ERROR];
      rep->kernel_launches = launches_;
    }
    finish_profile(rep);
    return rc;
  }

 private:
  Context& ctx_;
  extremz_params p_;
  cudaStream_t st_;
  int32_t* trace_;
  int trace_cap_, trace_len_ = 0;
  Job<T> J;
  int grid_ = 0;
  int outer_ = 0, cloop_rounds_ = 0, manifold_rounds_ = 0;
  bool capped_ = false;
  int hc_[11] = {0};
  int* ctr_ = nullptr;

  CUtensorMap map_f_, map_g_;
  bool tma_f_ = false, tma_g_ = false;
  // The job descriptor lives in device memory; every per-round kernel takes
  // the descriptor array and a selection (here: the one job).
  Job<T>* jobs_dev_ = nullptr;
  CUtensorMap* maps_dev_ = nullptr;
  Sel sel1_;

  const Job<T>* jobs() const { return jobs_dev_; }
  int ntiles() const {
    return ((J.dim.W + TX - 1) / TX) * ((J.dim.H + TY - 1) / TY) * ((J.dim.D + TZ - 1) / TZ);
  }
  int upload_job() {
    EZ_CHECK(cudaMemcpyAsync(jobs_dev_, &J, sizeof(J), cudaMemcpyHostToDevice, st_));
    return EXTREMZ_OK;
  }
  void swap_lists(int which) { launch(K_OTHER, k_swap_lists<T>, 1, 32, jobs_dev_, sel1_, which); }

  long long launches_ = 0;
  bool profile_ = false;
  int profile_mask_ = 0;
  struct Rec { int cls; cudaEvent_t a, b; };
  std::vector<Rec> recs_;
  std::vector<cudaEvent_t> pool_;

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

  // Every kernel goes through here: counted, and bracketed by events when
  // per-class timing is on.
  template <class... KArgs, class... Args>
  void launch(int cls, void (*kern)(KArgs...), dim3 grid, dim3 block, Args... args) {
    cudaEvent_t a = nullptr, b = nullptr;
    const bool timed = profile_ && (profile_mask_ == 0 || (profile_mask_ >> cls & 1));
    if (timed) {
      a = event();
      b = event();
      cudaEventRecord(a, st_);
    }
    kern<<<grid, block, 0, st_>>>(args...);
    ++launches_;
    if (timed) {
      cudaEventRecord(b, st_);
      recs_.push_back({cls, a, b});
    }
  }

  void finish_profile(extremz_report* rep) {
    if (!profile_) return;
    cudaStreamSynchronize(st_);
    for (const Rec& r : recs_) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, r.a, r.b);
      if (rep) {
        rep->prof_ms[r.cls] += ms;
        rep->prof_launches[r.cls] += 1;
      }
      pool_.push_back(r.a);
      pool_.push_back(r.b);
    }
    recs_.clear();
    for (cudaEvent_t e : pool_) cudaEventDestroy(e);
    pool_.clear();
  }

  int iter_cap() const { return p_.device_iter_cap > 0 ? p_.device_iter_cap : J.dim.N + 1; }

  int sm_count() {
    int dev = 0, n = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n;
  }

  void emit(int phase, int a = 0, int b = 0, int c = 0) {
    if (!trace_ || trace_len_ + 4 > trace_cap_) return;
    trace_[trace_len_++] = phase;
    trace_[trace_len_++] = a;
    trace_[trace_len_++] = b;
    trace_[trace_len_++] = c;
  }

  int zero(int slot, int n = 1) {
    EZ_CHECK(cudaMemsetAsync(ctr_ + slot, 0, n * sizeof(int), st_));
    return EXTREMZ_OK;
  }
  int read_ctr() {
    EZ_CHECK(cudaMemcpyAsync(ctx_.h_ctr, ctr_, C_COUNT * sizeof(int), cudaMemcpyDeviceToHost, st_));
    EZ_CHECK(cudaStreamSynchronize(st_));
    if (ctx_.h_ctr[C_ERROR]) return EXTREMZ_DEVICE_TIMEOUT;
    return EXTREMZ_OK;
  }
  int h(int slot) const { return ctx_.h_ctr[slot]; }
  int launched() {
    EZ_CHECK(cudaGetLastError());
    return EXTREMZ_OK;
  }
  dim3 tile_grid() const {
    return dim3((J.dim.W + TX - 1) / TX, (J.dim.H + TY - 1) / TY, (J.dim.D + TZ - 1) / TZ);
  }

#define EZ_RUN(expr)               \
  do {                             \
    int rc_ = (expr);              \
    if (rc_ != EXTREMZ_OK) return rc_; \
  } while (0)

  // ---------------------------------------------------------------- setup --
  int setup() {
    const int N = J.dim.N;
    if (ctx_.has_tables) J.tb = ctx_.tables;
    else EZ_RUN(device_tables(&J.tb));
    if (!ctx_.h_ctr) EZ_CHECK(cudaMallocHost(&ctx_.h_ctr, C_COUNT * sizeof(int)));
    grid_ = sm_count() * 8;
    const int nb = (N + kCpBlock - 1) / kCpBlock;
    // Phase-1 arena: per-voxel arrays and the CP block counts.  The per-CP
    // arrays are carved after the counts are known.
    auto bytes_for = [&](long long ns2, long long ns1, long long nmax, long long nmin) {
      long long b = 0;
      auto add = [&](long long count, long long sz) { b += (count * sz + 255) & ~255ll; };
      add(C_COUNT, 4);
      add(N, 1); add(N, 2);                    // otype, olm
      for (int i = 0; i < 5; ++i) add(N, 4);   // ds, as, dds, das, ext
      add(N, sizeof(K)); add(N, 4); add(N, 4); add(N, 4);  // delta, counter, touched, mm
      add(N, 4); add(N, 1); add(N, 4); add(N, 4); add(N, 4);  // mm_next, mstat, dirty, dstamp, rstamp
      add(N, 8); add(N, 4); add(N, 4);         // claim, taken, taken1
      for (int i = 0; i < 4; ++i) add(N, 4);   // cand, cand_next, flagged, flagged1
      add(4ll * nb, 4);                        // cp block counts
      add(ns2, 4); add(ns1, 4); add(nmax, 4); add(nmin, 4);
      add(ns2 * kRowStride, 4); add(ns2 * 2, 4); add(ns2, 1);
      add(ns1 * kRowStride, 4); add(ns1 * 2, 4); add(ns1, 1);
      for (int i = 0; i < 4; ++i) add(nmax, 4);  // largest, first1, flag2, first_s
      for (int i = 0; i < 4; ++i) add(nmin, 4);  // smallest, first_min1, flag_min2, first_sj
      long long ne = std::max(nmax, nmin);
      add(ne, sizeof(K)); add(ne, 4);
      add(8, 8);  // checksum
      return b;
    };
    // Worst case for the CP lists is N each; reserve that up front so the
    // arena is never re-allocated between the two phases.
    long long worst = bytes_for(N, N, N, N);
    int rc = ctx_.arena.reserve((size_t)worst);
    if (rc != EXTREMZ_OK) return rc;
    Arena& A = ctx_.arena;
    A.used = 0;
    ctr_ = J.ctr = A.take<int>(C_COUNT);
    J.otype = A.take<int8_t>(N);
    J.olm = A.take<uint16_t>(N);
    J.ds = A.take<int>(N); J.as = A.take<int>(N);
    J.dds = A.take<int>(N); J.das = A.take<int>(N);
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
    J.taken = A.take<int>(N); J.taken1 = A.take<int>(N);
    J.cand = A.take<int>(N); J.cand_next = A.take<int>(N);
    J.flagged = A.take<int>(N); J.flagged1 = A.take<int>(N);
    int* bcount = A.take<int>(4ll * nb);
    jobs_dev_ = A.take<Job<T>>(1);
    maps_dev_ = A.take<CUtensorMap>(2);
    if (!jobs_dev_ || !maps_dev_) return EXTREMZ_OOM;
    EZ_CHECK(cudaMemcpyAsync(maps_dev_, &map_f_, sizeof(CUtensorMap), cudaMemcpyHostToDevice, st_));
    EZ_CHECK(cudaMemcpyAsync(maps_dev_ + 1, &map_g_, sizeof(CUtensorMap), cudaMemcpyHostToDevice, st_));
    J.map_f = maps_dev_;
    J.map_g = maps_dev_ + 1;
    J.tma_f = tma_f_;
    J.tma_g = tma_g_;
    std::memset(&sel1_, 0, sizeof(sel1_));
    sel1_.n = 1;
    sel1_.idx[0] = 0;
    sel1_.off[0] = 0;
    sel1_.off[1] = ntiles();
    EZ_RUN(upload_job());
    EZ_CHECK(cudaMemsetAsync(ctr_, 0, C_COUNT * sizeof(int), st_));

    // Original classification and manifolds.
    launch(K_SETUP, k_classify<T, false>, ntiles(), 256, jobs(), sel1_);
    launch(K_DIRECTION, k_direction<T, false>, ntiles(), 256, jobs(), sel1_);
    launch(K_JUMP, k_jump2<T, false>, grid_, 256, jobs(), sel1_, iter_cap());
    EZ_RUN(launched());
    // Critical-point lists in ascending id.
    launch(K_OTHER, k_cp_count, nb, kCpBlock, J.otype, N, bcount);
    launch(K_OTHER, k_cp_scan, 1, 1024, bcount, nb, ctr_);
    EZ_RUN(launched());
    EZ_RUN(read_ctr());
    const int ns2 = h(C_NS2), ns1 = h(C_NS1), nmax = h(C_NMAX), nmin = h(C_NMIN);
    J.sad2 = A.take<int>(ns2); J.sad1 = A.take<int>(ns1);
    J.maxima = A.take<int>(nmax); J.minima = A.take<int>(nmin);
    J.orow2 = A.take<int>((long long)ns2 * kRowStride);
    J.drow2 = A.take<int>((long long)ns2 * 2);
    J.ocnt2 = A.take<uint8_t>(ns2);
    J.orow1 = A.take<int>((long long)ns1 * kRowStride);
    J.drow1 = A.take<int>((long long)ns1 * 2);
    J.ocnt1 = A.take<uint8_t>(ns1);
    J.largest = A.take<int>(nmax); J.first1 = A.take<int>(nmax);
    J.flag2 = A.take<int>(nmax); J.first_s = A.take<int>(nmax);
    J.smallest = A.take<int>(nmin); J.first_min1 = A.take<int>(nmin);
    J.flag_min2 = A.take<int>(nmin); J.first_sj = A.take<int>(nmin);
    const int ne = std::max(nmax, nmin);
    J.ext_key = A.take<K>(ne);
    J.ext_id = A.take<int>(ne);
    checksum_ = A.take<unsigned long long>(8);
    EZ_RUN(upload_job());
    launch(K_OTHER, k_cp_write, nb, kCpBlock, J.otype, N, bcount, J.sad2, J.sad1, J.maxima, J.minima);
    launch(K_OTHER, k_ext_index<T>, grid_, 256, J);
    launch(K_ROWS, k_rows<T, true>, grid_, 256, J, J.f, J.ds, J.sad2, C_NS2, J.orow2);
    launch(K_ROWS, k_rows<T, false>, grid_, 256, J, J.f, J.as, J.sad1, C_NS1, J.orow1);
    launch(K_SETUP, k_row_counts<T>, grid_, 256, J);
    EZ_RUN(launched());
    // Decompressed row slots start at zero: the reference's rows are fresh
    // cudaMalloc memory read before first written (:5338-5341, :3128-3130).
    if (ns2) EZ_CHECK(cudaMemsetAsync(J.drow2, 0, (size_t)ns2 * 2 * 4, st_));
    if (ns1) EZ_CHECK(cudaMemsetAsync(J.drow1, 0, (size_t)ns1 * 2 * 4, st_));
    // Largest saddle per maximum, smallest per minimum (original field).
    if (nmax) {
      launch(K_OTHER, k_fill<K>, grid_, 256, J.ext_key, K(0), nmax);
      launch(K_OTHER, k_fill<int>, grid_, 256, J.ext_id, -1, nmax);
      launch(K_OTHER, k_extreme_saddle<T, true>, grid_, 256, J, 0);
      launch(K_OTHER, k_extreme_saddle<T, true>, grid_, 256, J, 1);
      EZ_CHECK(cudaMemcpyAsync(J.largest, J.ext_id, nmax * 4, cudaMemcpyDeviceToDevice, st_));
      launch(K_OTHER, k_fill<int>, grid_, 256, J.first1, kInf, nmax);
      launch(K_OTHER, k_fill<int>, grid_, 256, J.first_s, kInf, nmax);
      EZ_CHECK(cudaMemsetAsync(J.flag2, 0, nmax * 4, st_));
    }
    if (nmin) {
      launch(K_OTHER, k_fill<K>, grid_, 256, J.ext_key, ~K(0), nmin);
      launch(K_OTHER, k_fill<int>, grid_, 256, J.ext_id, kInf, nmin);
      launch(K_OTHER, k_extreme_saddle<T, false>, grid_, 256, J, 0);
      launch(K_OTHER, k_extreme_saddle<T, false>, grid_, 256, J, 1);
      EZ_CHECK(cudaMemcpyAsync(J.smallest, J.ext_id, nmin * 4, cudaMemcpyDeviceToDevice, st_));
      launch(K_OTHER, k_fill<int>, grid_, 256, J.first_min1, kInf, nmin);
      launch(K_OTHER, k_fill<int>, grid_, 256, J.first_sj, kInf, nmin);
      EZ_CHECK(cudaMemsetAsync(J.flag_min2, 0, nmin * 4, st_));
    }
    // Proposal buffer at the sentinel, counters at -1 (:5082), stamps at 0.
    launch(K_OTHER, k_fill<K>, grid_, 256, J.delta, J.sentinel_key, N);
    launch(K_OTHER, k_fill<int>, grid_, 256, J.counter, -1, N);
    EZ_CHECK(cudaMemsetAsync(J.claim, 0, (size_t)N * 8, st_));
    EZ_CHECK(cudaMemsetAsync(J.taken, 0, (size_t)N * 4, st_));
    EZ_CHECK(cudaMemsetAsync(J.taken1, 0, (size_t)N * 4, st_));
    EZ_CHECK(cudaMemsetAsync(J.dstamp, 0, (size_t)N * 4, st_));
    EZ_CHECK(cudaMemsetAsync(J.rstamp, 0, (size_t)N * 4, st_));
    EZ_RUN(launched());
    return EXTREMZ_OK;
  }

  int dirty_epoch_ = 1, detect_epoch_ = 0;
  bool dense_done_ = false;

  unsigned long long* checksum_ = nullptr;

  int checksum_emit() {
    if (!trace_) return EXTREMZ_OK;
    EZ_CHECK(cudaMemsetAsync(checksum_, 0, 8, st_));
    launch(K_OTHER, k_checksum<T>, grid_, 256, J.g, J.dim.N, checksum_);
    unsigned long long hsum = 0;
    EZ_CHECK(cudaMemcpyAsync(&hsum, checksum_, 8, cudaMemcpyDeviceToHost, st_));
    EZ_CHECK(cudaStreamSynchronize(st_));
    emit(PH_CHECKSUM, (int)(hsum & 0x7fffffff), (int)((hsum >> 31) & 0x7fffffff));
    return EXTREMZ_OK;
  }

  // ------------------------------------------------------------- c_loops --
  // Mismatch detection: dense the first time, then incremental over the
  // neighbourhoods of the vertices changed since the previous detection.
  int detect() {
    if (!dense_done_) {
      EZ_RUN(zero(C_MM, 4));
      launch(K_DETECT, k_classify<T, true>, ntiles(), 256, jobs(), sel1_);
      dense_done_ = true;
    } else {
      ++detect_epoch_;
      EZ_RUN(zero(C_MM_NEXT));
      EZ_RUN(zero(C_CMAX, 3));
      launch(K_DETECT, k_redetect<T>, grid_, 256, jobs(), sel1_, detect_epoch_);
      launch(K_DETECT, k_keep<T>, grid_, 256, jobs(), sel1_, detect_epoch_);
      swap_lists(0);
    }
    EZ_RUN(zero(C_DIRTY));
    ++dirty_epoch_;
    EZ_RUN(launched());
    EZ_RUN(read_ctr());
    emit(PH_CLOOP_DETECT, h(C_CMAX), h(C_CMIN), h(C_CSAD));
    return EXTREMZ_OK;
  }

  int apply() {
    launch(K_APPLY, k_apply<T>, grid_, 256, jobs(), sel1_, dirty_epoch_);
    return launched();
  }

  // c_loops (:3913-4044).
  int c_loops() {
    EZ_RUN(detect());
    int rounds = 0;
    while (h(C_MM) > 0) {
      if (rounds >= p_.max_cloop_rounds) {
        capped_ = true;
        return EXTREMZ_OK;
      }
      ++rounds;
      ++cloop_rounds_;
      EZ_RUN(zero(C_TOUCHED));
      launch(K_PROPOSE, k_propose_cp<T>, grid_, 256, jobs(), sel1_);
      EZ_RUN(launched());
      EZ_RUN(apply());
      EZ_RUN(detect());
    }
    return EXTREMZ_OK;
  }

  // ----------------------------------------------------------- manifolds --
  // One manifold round: decompressed steepest roots, then per saddle side the
  // fused row-slot / candidate pass and the wrong-neighbour arbitration
  // (ComputeDirection + Compute*Manifold, findAscPaths / findDescPaths,
  // get_wrong_split_neighbors / get_wrong_join_neighbors).
  int manifold_block() {
    ++manifold_rounds_;
    const int N = J.dim.N;
    launch(K_DIRECTION, k_direction<T, true>, ntiles(), 256, jobs(), sel1_);
    launch(K_JUMP, k_jump2<T, true>, grid_, 256, jobs(), sel1_, iter_cap());
    const int stamp = ++ctx_.wn_stamp;
    EZ_RUN(zero(C_NFC, 2));
    EZ_RUN(resolve_side<true>(stamp));
    EZ_RUN(resolve_side<false>(stamp));
    EZ_RUN(read_ctr());
    emit(PH_WRONG_NBR, h(C_NFC), h(C_NFC1));
    return EXTREMZ_OK;
  }

  // Bounded device rounds of vote / commit, then the sequential completion
  // for whatever is left; no host round trip.
  template <bool kSplit>
  int resolve_side(int stamp) {
    EZ_RUN(zero(C_CAND));
    launch(K_ROWS, k_saddle_pass<T, kSplit>, grid_, 256, jobs(), sel1_);
    const int kRounds = 3;
    for (int r = 0; r < kRounds; ++r) {
      const unsigned long long round = ++ctx_.wn_round;
      EZ_RUN(zero(C_CAND_NEXT));
      launch(K_WRONG_NBR, k_wn_vote<T, kSplit>, grid_, 256, jobs(), sel1_, round, stamp);
      launch(K_WRONG_NBR, k_wn_commit<T, kSplit>, grid_, 256, jobs(), sel1_, round, stamp);
      swap_lists(1);
    }
    launch(K_WRONG_NBR, k_wn_sequential<T, kSplit>, 1, 1, jobs(), sel1_, stamp);
    return launched();
  }

  // r_loops (:4210-4227).
  int r_loops() {
    EZ_RUN(zero(C_TOUCHED));
    launch(K_FIXPATH, k_fixpath<T, true>, grid_, 256, jobs(), sel1_, iter_cap());
    launch(K_FIXPATH, k_fixpath<T, false>, grid_, 256, jobs(), sel1_, iter_cap());
    EZ_RUN(launched());
    return apply();
  }

  // s_loops (:3465-3487).
  int s_loops() {
    EZ_RUN(zero(C_WMC, 2));
    EZ_RUN(zero(C_TOUCHED));
    launch(K_OTHER, k_wim_scan<T, true>, grid_, 256, jobs(), sel1_);
    launch(K_OTHER, k_wim_collect<T, true>, grid_, 256, jobs(), sel1_, 1);
    EZ_RUN(launched());
    EZ_RUN(apply());
    // s_loops refreshes the reference's file-scope host copies (:3473-3476);
    // the first block branches on them right away.
    EZ_RUN(read_ctr());
    emit(PH_SLOOPS, h(C_WMC), h(C_WMC2));
    return EXTREMZ_OK;
  }

  // saddle_loops (:4229-4243).
  int saddle_loops() {
    EZ_RUN(zero(C_WSC));
    EZ_RUN(zero(C_TOUCHED));
    launch(K_OTHER, k_wis_scan<T, true>, grid_, 256, jobs(), sel1_);
    launch(K_OTHER, k_wis_collect<T, true>, grid_, 256, jobs(), sel1_, 1);
    EZ_RUN(launched());
    EZ_RUN(apply());
    if (trace_) {
      EZ_RUN(read_ctr());
      emit(PH_SADDLE, h(C_WSC));
    }
    return EXTREMZ_OK;
  }

  // s_loops_join (:3489-3512).
  int s_loops_join() {
    EZ_RUN(zero(C_WMIN, 2));
    EZ_RUN(zero(C_TOUCHED));
    launch(K_OTHER, k_wim_scan<T, false>, grid_, 256, jobs(), sel1_);
    launch(K_OTHER, k_wim_collect<T, false>, grid_, 256, jobs(), sel1_, 1);
    launch(K_OTHER, k_wim_min2_scan<T>, grid_, 256, jobs(), sel1_);
    launch(K_OTHER, k_wim_min2_collect<T>, grid_, 256, jobs(), sel1_);
    EZ_RUN(launched());
    EZ_RUN(apply());
    if (trace_) {
      EZ_RUN(read_ctr());
      emit(PH_SLOOPS_JOIN, h(C_WMIN), h(C_WMIN2));
    }
    return EXTREMZ_OK;
  }

  // saddle_loops_join (:4245-4261).
  int saddle_loops_join() {
    EZ_RUN(zero(C_WSCJ));
    EZ_RUN(zero(C_TOUCHED));
    launch(K_OTHER, k_wis_scan<T, false>, grid_, 256, jobs(), sel1_);
    launch(K_OTHER, k_wis_collect<T, false>, grid_, 256, jobs(), sel1_, 1);
    EZ_RUN(launched());
    EZ_RUN(apply());
    if (trace_) {
      EZ_RUN(read_ctr());
      emit(PH_SADDLE_JOIN, h(C_WSCJ));
    }
    return EXTREMZ_OK;
  }

  // --------------------------------------------------------------- main --
  // main() (:5508-5997).  The reference's host counters: c_loops and r_loops
  // take them by value (main's copies unchanged); s_loops, saddle_loops and
  // the join variants refresh the file-scope copies of wrong_max(_2),
  // wrong_saddle, wrong_min(_2) and wrong_saddle_join (:62, :3473-3476,
  // :4236, :3498-3501, :4252).  Each device counter changes only in the call
  // that refreshes its host copy, so reading the counter block at the end of
  // an iteration yields exactly those copies.
  int main_loop() {
    const bool join = p_.preserve_join != 0;
    EZ_RUN(c_loops());
    if (capped_) return EXTREMZ_ROUND_CAP;
    EZ_RUN(manifold_block());
    int nfc = h(C_NFC), nfc1 = h(C_NFC1);
    if (nfc == 0) {
      EZ_RUN(s_loops());
      if (h(C_WMC) == 0) EZ_RUN(saddle_loops());
    }
    if (nfc1 == 0 && join) {
      EZ_RUN(s_loops_join());
      EZ_RUN(read_ctr());
      if (h(C_WMIN) == 0) EZ_RUN(saddle_loops_join());
    }
    EZ_RUN(read_ctr());  // :5589-5599
    auto snapshot = [&](int* c) {
      const int v[11] = {nfc, nfc1, h(C_CMAX), h(C_CMIN), h(C_CSAD), h(C_WMC),
                         h(C_WMC2), h(C_WSC), h(C_WMIN), h(C_WMIN2), h(C_WSCJ)};
      std::memcpy(c, v, sizeof(v));
    };
    nfc = h(C_NFC);
    nfc1 = h(C_NFC1);
    int c[11];
    snapshot(c);
    auto any = [&] {
      for (int i = 0; i < 11; ++i)
        if (c[i] > 0) return true;
      return false;
    };
    while (any()) {
      if (outer_ >= p_.max_outer) {
        capped_ = true;
        break;
      }
      ++outer_;
      // Block 1 (:5622-5747).
      EZ_RUN(c_loops());
      if (capped_) break;
      EZ_RUN(r_loops());
      EZ_RUN(manifold_block());
      nfc = h(C_NFC);
      nfc1 = h(C_NFC1);
      if (nfc == 0) {
        EZ_RUN(s_loops());
        if (h(C_WMC) == 0) EZ_RUN(saddle_loops());
      }
      if (nfc1 == 0 && join) {
        EZ_RUN(s_loops_join());
        EZ_RUN(read_ctr());
        if (h(C_WMIN) == 0) EZ_RUN(saddle_loops_join());
      }
      // Block 2 (:5749-5870).
      EZ_RUN(c_loops());
      if (capped_) break;
      EZ_RUN(manifold_block());
      nfc = h(C_NFC);
      nfc1 = h(C_NFC1);
      if (nfc == 0) {
        EZ_RUN(s_loops());
        if (h(C_WMC) == 0) EZ_RUN(saddle_loops());
      }
      if (nfc1 == 0 && join) {
        EZ_RUN(s_loops_join());
        EZ_RUN(read_ctr());
        if (h(C_WMIN) == 0) EZ_RUN(saddle_loops_join());
      }
      // Block 3 (:5872-5979): detection only.
      EZ_RUN(c_loops());
      if (capped_) break;
      EZ_RUN(manifold_block());
      nfc = h(C_NFC);
      nfc1 = h(C_NFC1);
      if (nfc == 0) {
        EZ_RUN(zero(C_WMC, 2));
        EZ_RUN(zero(C_WSC));
        launch(K_OTHER, k_wim_scan<T, true>, grid_, 256, jobs(), sel1_);
        launch(K_OTHER, k_wim_collect<T, true>, grid_, 256, jobs(), sel1_, 0);
        launch(K_OTHER, k_wis_scan<T, true>, grid_, 256, jobs(), sel1_);
        launch(K_OTHER, k_wis_collect<T, true>, grid_, 256, jobs(), sel1_, 0);
        EZ_RUN(launched());
        if (trace_) {
          EZ_RUN(read_ctr());
          emit(PH_DETECT3, h(C_WSC), h(C_WMC), h(C_WMC2));
        }
      }
      if (nfc1 == 0 && join) {
        EZ_RUN(zero(C_WMIN, 2));
        EZ_RUN(zero(C_WSCJ));
        launch(K_OTHER, k_wim_scan<T, false>, grid_, 256, jobs(), sel1_);
        launch(K_OTHER, k_wim_collect<T, false>, grid_, 256, jobs(), sel1_, 0);
        launch(K_OTHER, k_wis_scan<T, false>, grid_, 256, jobs(), sel1_);
        launch(K_OTHER, k_wis_collect<T, false>, grid_, 256, jobs(), sel1_, 0);
        EZ_RUN(launched());
      }
      EZ_RUN(detect());  // reads the whole counter block
      snapshot(c);
      emit(PH_OUTER, outer_);
      EZ_RUN(checksum_emit());
    }
    std::memcpy(hc_, c, sizeof(c));  // counters at loop exit
    if (!capped_ && p_.final_join) EZ_RUN(saddle_loops_join());  // unconditional (:5997)
    EZ_RUN(read_ctr());
    return capped_ ? EXTREMZ_ROUND_CAP : EXTREMZ_OK;
  }
#undef EZ_RUN
};

static int check_args(int dtype, long long W, long long H, long long D, const extremz_params* p) {
  if (!p || (dtype != EXTREMZ_F32 && dtype != EXTREMZ_F64)) return EXTREMZ_BAD_ARG;
  if (W <= 0 || H <= 0 || D <= 0) return EXTREMZ_BAD_ARG;
  if (W * H * D >= (1ll << kCatShift)) return EXTREMZ_BAD_ARG;
  if (p->q <= 0 || (p->edit_type != 0 && p->edit_type != 1)) return EXTREMZ_BAD_ARG;
  if (p->max_outer < 0 || p->max_cloop_rounds < 0 || p->device_iter_cap < 0) return EXTREMZ_BAD_ARG;
  return EXTREMZ_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free correction (extremz_correct_device_noalloc).
//
// Some callers cannot allocate device memory at the time they correct a
// field: code that runs while a CUDA graph is being captured, allocators
// that own all of the device's memory, or real-time paths that forbid
// allocation after start-up.  For them the whole workspace of one correction
// lives in a fixed-size static device array, and the lookup table in static
// device arrays, so a call allocates nothing.  The array is sized for the
// worst case of EXTREMZ_NOALLOC_MAX_VOXELS voxels and every GPU that loads
// the library keeps it until the process exits.
// ---------------------------------------------------------------------------
constexpr long long kNoAllocMaxVoxels = EXTREMZ_NOALLOC_MAX_VOXELS;
// Worst case of the workspace layout (every voxel a critical point of every
// kind, 8-byte values): 297 bytes per voxel plus per-array alignment.
constexpr size_t kNoAllocScratchBytes = (size_t)kNoAllocMaxVoxels * 320 + (1u << 20);
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];
static __device__ int8_t g_noalloc_lut[kLutSize];
static __device__ int g_noalloc_key_offset[64];

struct NoAllocDevice {
  bool ready = false;
  Context ctx;
  int host_ctr[C_COUNT];  // pageable host copy of the counter block
};
static std::mutex g_noalloc_mu;
static NoAllocDevice g_noalloc[64];

// Once per device, with that device current: the device addresses of the
// static arrays (a host-side name of a __device__ array is not a device
// address) and the lookup table upload.
static int noalloc_setup(int dev) {
  NoAllocDevice& d = g_noalloc[dev];
  if (d.ready) return EXTREMZ_OK;
  void* scratch = nullptr;
  void* lut = nullptr;
  void* keys = nullptr;
  EZ_CHECK(cudaGetSymbolAddress(&scratch, g_noalloc_scratch));
  EZ_CHECK(cudaGetSymbolAddress(&lut, g_noalloc_lut));
  EZ_CHECK(cudaGetSymbolAddress(&keys, g_noalloc_key_offset));
  const HostTables& t = host_tables();
  EZ_CHECK(cudaMemcpyToSymbol(g_noalloc_lut, t.lut, kLutSize));
  EZ_CHECK(cudaMemcpyToSymbol(g_noalloc_key_offset, t.key_offset, 64 * sizeof(int)));
  d.ctx.device = dev;
  d.ctx.has_tables = true;
  d.ctx.tables.lut = static_cast<const int8_t*>(lut);
  d.ctx.tables.key_offset = static_cast<const int*>(keys);
  d.ctx.arena.base = static_cast<char*>(scratch);
  d.ctx.arena.cap = kNoAllocScratchBytes;
  d.ctx.arena.fixed = true;
  d.ctx.h_ctr = d.host_ctr;
  d.ready = true;
  return EXTREMZ_OK;
}

static int correct_noalloc(const void* d_orig, void* d_decp, int dtype, int width, int height,
                           int depth, const extremz_params* params, extremz_report* report,
                           void* stream) {
  if (!d_orig || !d_decp || !params) return EXTREMZ_BAD_ARG;
  int rc = check_args(dtype, width, height, depth, params);
  if (rc != EXTREMZ_OK) return rc;
  if ((long long)width * height * depth > kNoAllocMaxVoxels) return EXTREMZ_TOO_LARGE;
  int dev = 0;
  EZ_CHECK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return EXTREMZ_BAD_ARG;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  rc = noalloc_setup(dev);
  if (rc != EXTREMZ_OK) return rc;
  if (report) std::memset(report, 0, sizeof(*report));
  extremz_params p = *params;
  p.flags &= ~EXTREMZ_FLAG_PROFILE;  // no timing events in this mode
  cudaStream_t st = (cudaStream_t)stream;
  Context& ctx = g_noalloc[dev].ctx;
  if (dtype == EXTREMZ_F32) {
    Corrector<float> c(ctx, (const float*)d_orig, (float*)d_decp, width, height, depth, p, st,
                       nullptr, 0);
    rc = c.run(report);
  } else {
    Corrector<double> c(ctx, (const double*)d_orig, (double*)d_decp, width, height, depth, p, st,
                        nullptr, 0);
    rc = c.run(report);
  }
  if (report) report->status = rc;
  return rc;
}

}  // namespace extremz

using namespace extremz;

struct extremz_ctx_s {
  Context c;
};

extern "C" {

int extremz_version(void) { return EXTREMZ_ABI_VERSION; }

void extremz_default_params(extremz_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->bound = 0.0;
  p->thr = 0.0;
  p->q = 4;
  p->edit_type = 1;
  p->max_outer = 1000;
  p->max_cloop_rounds = 100000;
  p->final_join = 1;
  p->preserve_join = 0;
  p->flags = 0;
  p->device_iter_cap = 0;
}

extremz_status extremz_ctx_create(int device, extremz_ctx** out) {
  if (!out) return EXTREMZ_BAD_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return EXTREMZ_NO_DEVICE;
  }
  if (device < 0 || device >= n) return EXTREMZ_BAD_ARG;
  extremz_ctx* c = new (std::nothrow) extremz_ctx;
  if (!c) return EXTREMZ_OOM;
  c->c.device = device;
  *out = c;
  return EXTREMZ_OK;
}

void extremz_ctx_destroy(extremz_ctx* ctx) {
  if (!ctx) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(ctx->c.device);
  delete ctx;
  cudaSetDevice(prev);
}

extremz_status extremz_correct_device(extremz_ctx* ctx, const void* d_orig, void* d_decp, int dtype,
                                      int width, int height, int depth, const extremz_params* params,
                                      extremz_report* report, void* stream, int32_t* trace,
                                      int trace_cap) {
  if (!ctx || !d_orig || !d_decp) return EXTREMZ_BAD_ARG;
  int rc = check_args(dtype, width, height, depth, params);
  if (rc != EXTREMZ_OK) return (extremz_status)rc;
  if (report) std::memset(report, 0, sizeof(*report));
  int prev = 0;
  cudaGetDevice(&prev);
  if (prev != ctx->c.device) cudaSetDevice(ctx->c.device);
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == EXTREMZ_F32) {
    Corrector<float> c(ctx->c, (const float*)d_orig, (float*)d_decp, width, height, depth, *params,
                       st, trace, trace_cap);
    rc = c.run(report);
  } else {
    Corrector<double> c(ctx->c, (const double*)d_orig, (double*)d_decp, width, height, depth,
                        *params, st, trace, trace_cap);
    rc = c.run(report);
  }
  if (report) report->status = rc;
  if (prev != ctx->c.device) cudaSetDevice(prev);
  return (extremz_status)rc;
}

extremz_status extremz_correct_host(extremz_ctx* ctx, const void* h_orig, void* h_decp, int dtype,
                                    int width, int height, int depth, const extremz_params* params,
                                    extremz_report* report, void* stream) {
  if (!ctx || !h_orig || !h_decp) return EXTREMZ_BAD_ARG;
  int rc = check_args(dtype, width, height, depth, params);
  if (rc != EXTREMZ_OK) return (extremz_status)rc;
  int prev = 0;
  cudaGetDevice(&prev);
  if (prev != ctx->c.device) cudaSetDevice(ctx->c.device);
  const size_t bytes = (size_t)width * height * depth * (dtype == EXTREMZ_F32 ? 4 : 8);
  cudaStream_t st = (cudaStream_t)stream;
  rc = ctx->c.stage.reserve(2 * bytes + 512);
  if (rc != EXTREMZ_OK) {
    if (prev != ctx->c.device) cudaSetDevice(prev);
    return (extremz_status)rc;
  }
  ctx->c.stage.used = 0;
  char* df = ctx->c.stage.take<char>(bytes);
  char* dg = ctx->c.stage.take<char>(bytes);
  if (cudaMemcpyAsync(df, h_orig, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(dg, h_decp, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess)
    rc = EXTREMZ_CUDA_ERR;
  if (rc == EXTREMZ_OK)
    rc = extremz_correct_device(ctx, df, dg, dtype, width, height, depth, params, report, stream,
                                nullptr, 0);
  if (rc == EXTREMZ_OK || rc == EXTREMZ_ROUND_CAP) {
    if (cudaMemcpyAsync(h_decp, dg, bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      rc = EXTREMZ_CUDA_ERR;
  }
  if (prev != ctx->c.device) cudaSetDevice(prev);
  return (extremz_status)rc;
}

extremz_status extremz_correct_device_noalloc(const void* d_orig, void* d_decp, int dtype,
                                              int width, int height, int depth,
                                              const extremz_params* params,
                                              extremz_report* report, void* stream) {
  return (extremz_status)correct_noalloc(d_orig, d_decp, dtype, width, height, depth, params,
                                         report, stream);
}

long long extremz_noalloc_max_voxels(void) { return kNoAllocMaxVoxels; }

int extremz_lut(int32_t* out, int n) {
  if (!out || n < kLutSize) return -1;
  const HostTables& t = host_tables();
  for (int i = 0; i < kLutSize; ++i) out[i] = t.lut[i];
  return kLutSize;
}

const char* extremz_status_string(int status) {
  switch (status) {
    case EXTREMZ_OK: return "ok";
    case EXTREMZ_ROUND_CAP: return "round cap reached before zero mismatch";
    case EXTREMZ_BAD_ARG: return "bad argument";
    case EXTREMZ_OOM: return "out of device memory";
    case EXTREMZ_CUDA_ERR: return "CUDA error";
    case EXTREMZ_DEVICE_TIMEOUT: return "device-side iteration limit reached";
    case EXTREMZ_NO_DEVICE: return "no CUDA device";
    case EXTREMZ_TOO_LARGE:
      return "field larger than the static workspace of the allocation-free entry point";
    default: return "unknown status";
  }
}

const char* extremz_last_cuda_error(void) { return cudaGetErrorString(last_cuda_error()); }

}  // extern "C"

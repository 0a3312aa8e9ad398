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
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <dlfcn.h>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
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

#define EZ_RUN(expr)                   \
  do {                                 \
    int rc_ = (expr);                  \
    if (rc_ != EXTREMZ_OK) return rc_; \
  } while (0)

}  // namespace extremz

#include "extremz_batch.cuh"

namespace extremz {

// A stream-ordered pool that keeps what it has grown to: workspaces of
// successive corrections reuse the same memory without returning it to the
// driver at every synchronisation.
static cudaMemPool_t make_pool(int dev) {
  cudaMemPoolProps props;
  std::memset(&props, 0, sizeof(props));
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  cudaMemPool_t pool = nullptr;
  if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  uint64_t keep = ~uint64_t(0);
  cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  return pool;
}

struct Context {
  int device = 0;
  Arena stage;  // device copies of host fields (extremz_correct_host)
  char* hstage = nullptr;  // pinned host staging of edited-voxel lists
  size_t hstage_cap = 0;
  int ensure_hstage(size_t bytes) {
    if (bytes <= hstage_cap) return EXTREMZ_OK;
    if (hstage) cudaFreeHost(hstage);
    hstage = nullptr;
    hstage_cap = 0;
    EZ_CHECK(cudaHostAlloc(reinterpret_cast<void**>(&hstage), bytes, cudaHostAllocDefault));
    hstage_cap = bytes;
    return EXTREMZ_OK;
  }
  cudaMemPool_t pool = nullptr;
  cudaStream_t aux = nullptr;  // second stream of batches (the double engine) and
                               // of the decompressed field's copy in (host entry)
  cudaEvent_t join = nullptr;
  cudaEvent_t orig_in = nullptr, decp_in = nullptr;  // host entry: copies in have ended
  BatchEngine<float> e32{nullptr};
  BatchEngine<double> e64{nullptr};
  int ensure_aux() {
    if (aux) return EXTREMZ_OK;
    EZ_CHECK(cudaStreamCreateWithFlags(&aux, cudaStreamNonBlocking));
    EZ_CHECK(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
    EZ_CHECK(cudaEventCreateWithFlags(&orig_in, cudaEventDisableTiming));
    EZ_CHECK(cudaEventCreateWithFlags(&decp_in, cudaEventDisableTiming));
    return EXTREMZ_OK;
  }
  int ensure_pool() {
    if (pool) return EXTREMZ_OK;
    pool = make_pool(device);
    if (!pool) return EXTREMZ_OOM;
    e32.set_pool(pool);
    e64.set_pool(pool);
    return EXTREMZ_OK;
  }
  ~Context() {
    e32.release_all();
    e64.release_all();
    if (pool) {
      cudaDeviceSynchronize();
      cudaMemPoolDestroy(pool);
    }
    if (stage.base) cudaFree(stage.base);
    if (hstage) cudaFreeHost(hstage);
    if (join) cudaEventDestroy(join);
    if (orig_in) cudaEventDestroy(orig_in);
    if (decp_in) cudaEventDestroy(decp_in);
    if (aux) cudaStreamDestroy(aux);
  }
};

static int check_args(int dtype, long long W, long long H, long long D, const extremz_params* p) {
  if (!p || (dtype != EXTREMZ_F32 && dtype != EXTREMZ_F64)) return EXTREMZ_BAD_ARG;
  if (W <= 0 || H <= 0 || D <= 0) return EXTREMZ_BAD_ARG;
  if (W * H * D >= (1ll << kCatShift)) return EXTREMZ_BAD_ARG;
  if (p->q <= 0 || (p->edit_type != 0 && p->edit_type != 1)) return EXTREMZ_BAD_ARG;
  if (p->max_outer < 0 || p->max_cloop_rounds < 0 || p->device_iter_cap < 0) return EXTREMZ_BAD_ARG;
  if (p->tune_blocks_per_sm < 0 || p->tune_blocks_per_sm > 32 || p->tune_pass_chunk < 0 ||
      p->tune_pass_chunk > 64)
    return EXTREMZ_BAD_ARG;
  return EXTREMZ_OK;
}

// Copy-back of a corrected field into the caller's host buffer, which still
// holds the decompressed field: only the voxels whose value changed travel
// (ids and values, then a scatter on the host) unless they are so many that
// the whole field is cheaper.
template <class T>
struct HostWriteBack {
  Context* c;
  T* h_decp;
  cudaEvent_t input_ready = nullptr;  // the decompressed field's copy in has ended
  long long moved = 0;                // bytes copied device -> host
};

// out[ids[k]] = vals[k]: scattered stores into a large host buffer, bound by
// the latency of their cache misses, so large lists are split over threads
// and each thread prefetches ahead.
template <class T>
static void scatter_host(T* out, const int* ids, const T* vals, int n) {
  auto part = [=](int lo, int hi) {
    for (int k = lo; k < hi; ++k) {
      if (k + 16 < hi) __builtin_prefetch(out + ids[k + 16], 1, 0);
      out[ids[k]] = vals[k];
    }
  };
  const unsigned hc = std::thread::hardware_concurrency();
  const int nt = n < (1 << 15) ? 1 : (int)std::min(8u, std::max(1u, hc));
  if (nt == 1) {
    part(0, n);
    return;
  }
  std::vector<std::thread> th;
  int done = 1;  // parts [0, done) are handed out; a thread that cannot start leaves its part here
  try {
    for (int t = 1; t < nt; ++t, ++done)
      th.emplace_back(part, (int)((long long)n * t / nt), (int)((long long)n * (t + 1) / nt));
  } catch (...) {
  }
  part(0, (int)((long long)n / nt));
  if (done < nt) part((int)((long long)n * done / nt), n);
  for (auto& x : th) x.join();
}

template <class T>
static int write_back(BatchEngine<T>& e, int slot, const T* d_decp, long long N,
                      HostWriteBack<T>& wb) {
  cudaStream_t st = e.stream();
  int n = 0;
  EZ_RUN(e.edited_list(slot, &n));
  // A list entry costs (4 + sizeof(T)) bytes on the bus plus a scattered
  // store on the host; past 1/16 of the voxels the plain copy is faster.
  if ((long long)n * 16 > N) {
    EZ_CHECK(cudaMemcpyAsync(wb.h_decp, d_decp, (size_t)N * sizeof(T), cudaMemcpyDeviceToHost, st));
    EZ_CHECK(cudaStreamSynchronize(st));
    wb.moved = N * (long long)sizeof(T) + 4;
    return EXTREMZ_OK;
  }
  const size_t id_bytes = ((size_t)n * 4 + 255) & ~size_t(255);
  EZ_RUN(wb.c->ensure_hstage(id_bytes + (size_t)n * sizeof(T) + 256));
  int* hid = reinterpret_cast<int*>(wb.c->hstage);
  T* hv = reinterpret_cast<T*>(wb.c->hstage + id_bytes);
  if (n) {
    EZ_CHECK(cudaMemcpyAsync(hid, e.edited_ids(slot), (size_t)n * 4, cudaMemcpyDeviceToHost, st));
    EZ_CHECK(cudaMemcpyAsync(hv, e.edited_vals(slot), (size_t)n * sizeof(T), cudaMemcpyDeviceToHost, st));
    EZ_CHECK(cudaStreamSynchronize(st));
  }
  scatter_host(wb.h_decp, hid, hv, n);
  wb.moved = (long long)n * (4 + (long long)sizeof(T)) + 4;
  return EXTREMZ_OK;
}

// Runs one job to completion on an engine.
template <class T>
static int run_one(BatchEngine<T>& e, cudaStream_t st, const DeviceTables* tables, Arena* engine_store,
                   Arena* job_store, const T* f, T* g, int W, int H, int D, const extremz_params& p0,
                   extremz_report* rep, int32_t* trace, int trace_cap,
                   extremz_edit_stream* es = nullptr, HostWriteBack<T>* wb = nullptr,
                   bool census = false) {
  extremz_params p = p0;
  p.flags &= ~kInternalFlags;
  if (es) p.flags |= kFlagKeepInput;
  if (wb) p.flags |= kFlagTrackEdits;
  if (census) p.flags |= kFlagCensus;
  e.set_stream(st);
  EZ_RUN(e.init(tables, engine_store));
  const bool prof = (p.flags & EXTREMZ_FLAG_PROFILE) != 0;
  e.set_profile(prof, (p.flags >> EXTREMZ_PROFILE_CLASS_SHIFT) & ((1 << K_NUM) - 1));
  const long long l0 = e.launches();
  const long long g0 = e.graph_replays() + e.graph_captures();
  int slot = -1;
  EZ_RUN(e.admit(f, g, W, H, D, p, trace, trace_cap, job_store, 0, &slot));
  if (wb && wb->input_ready) e.set_input_event(slot, wb->input_ready);
  int rc = EXTREMZ_OK;
  while (e.job(slot).pc != PC_DONE) {
    rc = e.tick();
    if (rc != EXTREMZ_OK) break;
  }
  if (rc == EXTREMZ_OK) {
    cudaError_t ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) {
      last_cuda_error() = ce;
      rc = EXTREMZ_CUDA_ERR;
    }
  }
  if (rep) {
    e.fill_report(slot, rep);
    rep->kernel_launches = e.launches() - l0;
    rep->graph_launches = (int)(e.graph_replays() + e.graph_captures() - g0);
    if (prof) e.collect_profile(rep);
    if (rc != EXTREMZ_OK) rep->status = rc;
  }
  if (prof) e.drop_profile_events();
  e.set_profile(false, 0);
  if (rc == EXTREMZ_OK) rc = e.job(slot).status;
  if (es && (rc == EXTREMZ_OK || rc == EXTREMZ_ROUND_CAP)) {
    const int erc = e.encode(slot, es);
    if (erc != EXTREMZ_OK) rc = erc;
  }
  if (wb && (rc == EXTREMZ_OK || rc == EXTREMZ_ROUND_CAP)) {
    const int wrc = write_back(e, slot, g, (long long)W * H * D, *wb);
    if (wrc != EXTREMZ_OK) rc = wrc;
  }
  e.release(slot);
  return rc;
}

// Persistence pairs of one field: an analysis job (classification, labels and
// critical-point lists of the field), then the pairing rounds.
template <class T>
static int analyze_one(BatchEngine<T>& e, cudaStream_t st, const T* field, int W, int H, int D,
                       int* max_pairs, long long max_cap, int* min_pairs, long long min_cap,
                       long long* counts, int* max_parent = nullptr, int* min_parent = nullptr) {
  e.set_stream(st);
  EZ_RUN(e.init(nullptr, nullptr));
  extremz_params p;
  extremz_default_params(&p);
  p.flags = kFlagAnalysis;
  int slot = -1;
  EZ_RUN(e.admit(field, const_cast<T*>(field), W, H, D, p, nullptr, 0, nullptr, 0, &slot));
  int rc = EXTREMZ_OK;
  while (e.job(slot).pc != PC_DONE && rc == EXTREMZ_OK) rc = e.tick();
  if (rc == EXTREMZ_OK) rc = e.job(slot).status;
  if (rc == EXTREMZ_OK)
    rc = e.persistence(slot, max_pairs, max_cap, min_pairs, min_cap, counts, max_parent,
                       min_parent);
  e.release(slot);
  return rc;
}

// Vertex types and steepest-ascent / steepest-descent roots of one field: an
// analysis job, whose arrays are copied out before its workspace goes back.
template <class T>
static int classify_one(BatchEngine<T>& e, cudaStream_t st, const T* field, int W, int H, int D,
                        int8_t* d_type, int32_t* d_ds, int32_t* d_as) {
  e.set_stream(st);
  EZ_RUN(e.init(nullptr, nullptr));
  extremz_params p;
  extremz_default_params(&p);
  p.flags = kFlagAnalysis;
  int slot = -1;
  EZ_RUN(e.admit(field, const_cast<T*>(field), W, H, D, p, nullptr, 0, nullptr, 0, &slot));
  int rc = EXTREMZ_OK;
  while (e.job(slot).pc != PC_DONE && rc == EXTREMZ_OK) rc = e.tick();
  if (rc == EXTREMZ_OK) rc = e.job(slot).status;
  const Job<T>& J = e.job(slot).J;
  const size_t n = (size_t)W * H * D;
  if (rc == EXTREMZ_OK && d_type &&
      cudaMemcpyAsync(d_type, J.otype, n, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    rc = EXTREMZ_CUDA_ERR;
  if (rc == EXTREMZ_OK && d_ds &&
      cudaMemcpyAsync(d_ds, J.ds, n * 4, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    rc = EXTREMZ_CUDA_ERR;
  if (rc == EXTREMZ_OK && d_as &&
      cudaMemcpyAsync(d_as, J.as, n * 4, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    rc = EXTREMZ_CUDA_ERR;
  if (rc == EXTREMZ_OK && cudaStreamSynchronize(st) != cudaSuccess) rc = EXTREMZ_CUDA_ERR;
  if (rc == EXTREMZ_CUDA_ERR) last_cuda_error() = cudaGetLastError();
  e.release(slot);
  return rc;
}

// ---------------------------------------------------------------------------
// Allocation-free correction (extremz_correct_device_noalloc).
//
// Some callers cannot allocate device memory at the time they correct a
// field: applications whose allocator owns all of the device's memory, or
// real-time paths that forbid allocation after start-up because an
// allocation can block.  For them the whole workspace of one correction
// lives in a fixed-size static device array, and the lookup table in static
// device arrays, so a call allocates nothing.  The array is sized for the
// worst case of EXTREMZ_NOALLOC_MAX_VOXELS voxels and every GPU that loads
// the library keeps it until the process exits.
// ---------------------------------------------------------------------------
constexpr long long kNoAllocMaxVoxels = EXTREMZ_NOALLOC_MAX_VOXELS;
static_assert(K_NUM == EXTREMZ_NUM_KCLASS, "the report has one timing slot per kernel class");
// Engine arrays (descriptors, tile maps, counters) first, then one job's
// worst-case workspace (every voxel a critical point of every kind, 8-byte
// values: 443 bytes per voxel plus per-array alignment).
constexpr size_t kNoAllocEngineBytes = 1u << 18;
constexpr size_t kNoAllocScratchBytes = kNoAllocEngineBytes + (size_t)kNoAllocMaxVoxels * 448 + (1u << 20);
// Both engines (float and double) carve their descriptor, tile-map and
// counter arrays from the first part.
constexpr size_t kEngineArrayBytes(size_t job) {
  return ((job * kMaxSel + 255) & ~size_t(255)) + ((sizeof(CUtensorMap) * 2 * kMaxSel + 255) & ~size_t(255)) +
         ((sizeof(int) * C_COUNT * kMaxSel + 255) & ~size_t(255));
}
static_assert(kEngineArrayBytes(sizeof(Job<float>)) + kEngineArrayBytes(sizeof(Job<double>)) <=
                  kNoAllocEngineBytes,
              "engine arrays exceed the static workspace");
static_assert(job_bytes_max(kNoAllocMaxVoxels) <= (long long)(kNoAllocScratchBytes - kNoAllocEngineBytes),
              "job workspace exceeds the static workspace");
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];
static __device__ int8_t g_noalloc_lut[kLutSize];
static __device__ int g_noalloc_key_offset[64];

struct NoAllocDevice {
  bool ready = false;
  DeviceTables tables{};
  Arena engine_store, job_store;
  BatchEngine<float> e32{nullptr};
  BatchEngine<double> e64{nullptr};
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
  d.tables.lut = static_cast<const int8_t*>(lut);
  d.tables.key_offset = static_cast<const int*>(keys);
  d.engine_store.base = static_cast<char*>(scratch);
  d.engine_store.cap = kNoAllocEngineBytes;
  d.engine_store.fixed = true;
  d.job_store.base = static_cast<char*>(scratch) + kNoAllocEngineBytes;
  d.job_store.cap = kNoAllocScratchBytes - kNoAllocEngineBytes;
  d.job_store.fixed = true;
  // Graph instantiation may allocate: this mode launches directly.
  d.e32.set_graphs(false);
  d.e64.set_graphs(false);
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
  NoAllocDevice& d = g_noalloc[dev];
  cudaStream_t st = (cudaStream_t)stream;
  if (dtype == EXTREMZ_F32)
    rc = run_one(d.e32, st, &d.tables, &d.engine_store, &d.job_store, (const float*)d_orig,
                 (float*)d_decp, width, height, depth, p, report, nullptr, 0);
  else
    rc = run_one(d.e64, st, &d.tables, &d.engine_store, &d.job_store, (const double*)d_orig,
                 (double*)d_decp, width, height, depth, p, report, nullptr, 0);
  // run_one can leave early on an error with kernels still writing the shared
  // workspace; wait for them before the lock is released, so that the next
  // call (perhaps on another stream) does not race with them.
  if (cudaStreamSynchronize(st) != cudaSuccess) cudaGetLastError();
  if (report) report->status = rc;
  return rc;
}

// ---------------------------------------------------------------------------
// Batches: many fields, each with its own dtype, shape and parameters.  The
// float and double jobs run on two engines; a tick of each serves all of its
// jobs.  More than kMaxSel jobs of one dtype are admitted as slots free up.
// ---------------------------------------------------------------------------
template <class T>
struct BatchDriver {
  BatchEngine<T>* e;
  std::vector<int> todo;   // field indices not yet admitted
  std::vector<int> slot_of;
  size_t next = 0;
};

static int correct_batch_run(Context& C, const extremz_field* fields, int n,
                             extremz_report* reports, cudaStream_t st);

static int correct_batch(Context& C, const extremz_field* fields, int n, extremz_report* reports,
                         cudaStream_t st) {
  const int rc = correct_batch_run(C, fields, n, reports, st);
  if (rc != EXTREMZ_OK) {  // leave no job behind in the context's engines
    C.e32.release_jobs();
    C.e64.release_jobs();
  }
  return rc;
}

static int correct_batch_run(Context& C, const extremz_field* fields, int n,
                             extremz_report* reports, cudaStream_t st) {
  for (int i = 0; i < n; ++i) {
    EZ_RUN(check_args(fields[i].dtype, fields[i].width, fields[i].height, fields[i].depth,
                      &fields[i].params));
    if (!fields[i].orig || !fields[i].decp) return EXTREMZ_BAD_ARG;
  }
  EZ_RUN(C.ensure_pool());
  EZ_RUN(C.ensure_aux());
  // The double engine runs on the auxiliary stream, after what the caller
  // queued on st; the caller's stream is synchronised with it at the end.
  EZ_CHECK(cudaEventRecord(C.join, st));
  EZ_CHECK(cudaStreamWaitEvent(C.aux, C.join, 0));
  C.e32.set_stream(st);
  C.e64.set_stream(C.aux);
  EZ_RUN(C.e32.init(nullptr, nullptr));
  EZ_RUN(C.e64.init(nullptr, nullptr));
  std::vector<int> slot(n, -1), done(n, 0);
  std::vector<int> which(n);  // 0 float, 1 double
  int remaining = n;
  size_t next = 0;
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  const long long l0 = C.e32.launches() + C.e64.launches();
  // Per-class timing of the whole batch into reports[0] when the first
  // field asks for it.
  const bool prof = n > 0 && reports && (fields[0].params.flags & EXTREMZ_FLAG_PROFILE);
  const int pmask = n > 0 ? (fields[0].params.flags >> EXTREMZ_PROFILE_CLASS_SHIFT) & ((1 << K_NUM) - 1) : 0;
  C.e32.set_profile(prof, pmask);
  C.e64.set_profile(prof, pmask);
  while (remaining > 0) {
    // Admit while slots are free.
    while (next < order.size()) {
      const int i = order[next];
      const extremz_field& fd = fields[i];
      int rc, s = -1;
      if (fd.dtype == EXTREMZ_F32) {
        if (C.e32.free_slots() == 0) break;
        rc = C.e32.admit((const float*)fd.orig, (float*)fd.decp, fd.width, fd.height, fd.depth,
                         fd.params, nullptr, 0, nullptr, i, &s);
      } else {
        if (C.e64.free_slots() == 0) break;
        rc = C.e64.admit((const double*)fd.orig, (double*)fd.decp, fd.width, fd.height, fd.depth,
                         fd.params, nullptr, 0, nullptr, i, &s);
      }
      if (rc == EXTREMZ_OOM && (C.e32.active() + C.e64.active()) > 0) break;  // wait for memory
      if (rc != EXTREMZ_OK) return rc;
      slot[i] = s;
      which[i] = fd.dtype == EXTREMZ_F32 ? 0 : 1;
      ++next;
    }
    const bool a32 = C.e32.active() > 0, a64 = C.e64.active() > 0;
    if (a32) EZ_RUN(C.e32.tick_issue());
    if (a64) EZ_RUN(C.e64.tick_issue());
    if (a32) EZ_RUN(C.e32.tick_complete());
    if (a64) EZ_RUN(C.e64.tick_complete());
    for (int i = 0; i < n; ++i) {
      if (slot[i] < 0 || done[i]) continue;
      const bool fin = which[i] == 0 ? C.e32.job(slot[i]).pc == PC_DONE
                                     : C.e64.job(slot[i]).pc == PC_DONE;
      if (!fin) continue;
      if (reports) {
        if (which[i] == 0) C.e32.fill_report(slot[i], &reports[i]);
        else C.e64.fill_report(slot[i], &reports[i]);
      }
      if (which[i] == 0) C.e32.release(slot[i]);
      else C.e64.release(slot[i]);
      done[i] = 1;
      --remaining;
    }
  }
  EZ_CHECK(cudaStreamSynchronize(C.aux));
  EZ_CHECK(cudaStreamSynchronize(st));
  if (reports && n > 0) reports[0].kernel_launches = C.e32.launches() + C.e64.launches() - l0;
  if (prof) {
    std::memset(reports[0].prof_ms, 0, sizeof(reports[0].prof_ms));
    std::memset(reports[0].prof_launches, 0, sizeof(reports[0].prof_launches));
    C.e32.collect_profile(&reports[0]);
    C.e64.collect_profile(&reports[0]);
    C.e32.drop_profile_events();
    C.e64.drop_profile_events();
    C.e32.set_profile(false, 0);
    C.e64.set_profile(false, 0);
  }
  return EXTREMZ_OK;
}


// ---------------------------------------------------------------------------
// Serving: request loops ("lanes"), each on its own thread with a stream per
// dtype.  Between ticks a lane admits queued requests in arrival order while
// their footprint fits the shared HBM budget and a slot is free; every tick
// serves all of the lane's admitted jobs.  Requests up to split_voxels go to
// lane 0, whose streams have the higher priority, larger ones to lane 1, so a
// small request does not wait behind the long ticks of a large one.
// ---------------------------------------------------------------------------
using Clock = std::chrono::steady_clock;

struct ServerReq {
  long long ticket = 0;
  extremz_field field{};
  cudaEvent_t ready = nullptr;  // recorded on the caller's stream at submission
  long long footprint = 0;
  Clock::time_point t0;
};

struct ServerResult {
  bool done = false;
  int status = EXTREMZ_PENDING;
  extremz_report rep{};
  double latency_ms = 0.0;
};

struct ServerRunning {
  long long ticket;
  long long footprint;
  Clock::time_point t0;
  int dtype;
  int slot;
};

struct ServerLane {
  cudaStream_t st32 = nullptr, st64 = nullptr;
  BatchEngine<float> e32{nullptr};
  BatchEngine<double> e64{nullptr};
  std::thread th;
  std::deque<ServerReq> queue;      // guarded by the server's mutex
  std::vector<ServerRunning> running;  // the lane thread's own
};

static long long field_footprint(const extremz_field& f) {
  const long long n = (long long)f.width * f.height * f.depth;
  const long long vb = f.dtype == EXTREMZ_F32 ? 4 : 8;
  return job_bytes_max(n) + 2 * n * vb;
}

constexpr int kServerLanes = 2;

}  // namespace extremz

struct extremz_server_s {
  int device = 0;
  long long budget = 0;
  long long split = 0;
  int max_jobs = extremz::kMaxSel;
  int nlanes = extremz::kServerLanes;
  cudaMemPool_t pool = nullptr;
  extremz::ServerLane lane[extremz::kServerLanes];
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  int broken = EXTREMZ_OK;  // a CUDA error ends the loops; later requests fail with it
  std::unordered_map<long long, extremz::ServerResult> results;
  long long next_ticket = 1;
  extremz_server_stats stats{};
};

namespace extremz {

static void server_finish(extremz_server* s, const ServerRunning& r, int status,
                          const extremz_report* rep) {
  const double ms =
      std::chrono::duration<double, std::milli>(Clock::now() - r.t0).count();
  std::lock_guard<std::mutex> lk(s->mu);
  ServerResult& res = s->results[r.ticket];
  res.done = true;
  res.status = status;
  if (rep) res.rep = *rep;
  res.rep.status = status;
  res.latency_ms = ms;
  s->stats.bytes_in_use -= r.footprint;
  s->stats.completed += 1;
  s->stats.running -= 1;
  s->cv_work.notify_all();  // budget released: a blocked lane may admit
}

// Marks every queued request of every lane failed with rc (under the lock).
static void server_fail_queued(extremz_server* s, int rc) {
  for (int l = 0; l < s->nlanes; ++l) {
    for (ServerReq& q : s->lane[l].queue) {
      cudaEventDestroy(q.ready);
      ServerResult& res = s->results[q.ticket];
      res.done = true;
      res.status = rc;
      res.rep.status = rc;
    }
    s->lane[l].queue.clear();
  }
  s->stats.queued = 0;
}

static void server_loop(extremz_server* s, int li) {
  cudaSetDevice(s->device);
  ServerLane& L = s->lane[li];
  for (;;) {
    std::vector<ServerReq> admit_now;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      if (L.running.empty())
        s->cv_work.wait(lk, [&] { return s->stop || s->broken || !L.queue.empty(); });
      if ((s->stop || s->broken) && L.running.empty()) break;
      int n32 = 0, n64 = 0;
      for (const auto& r : L.running) (r.dtype == EXTREMZ_F32 ? n32 : n64)++;
      while (!s->stop && !s->broken && !L.queue.empty()) {
        const ServerReq& r = L.queue.front();
        int& n = r.field.dtype == EXTREMZ_F32 ? n32 : n64;
        if (n >= s->max_jobs) break;
        if (s->stats.bytes_in_use + r.footprint > s->budget) break;
        s->stats.bytes_in_use += r.footprint;
        s->stats.peak_bytes_in_use = std::max(s->stats.peak_bytes_in_use, s->stats.bytes_in_use);
        s->stats.queued -= 1;
        s->stats.running += 1;
        s->stats.peak_running = std::max<int>(s->stats.peak_running, (int)s->stats.running);
        ++n;
        admit_now.push_back(r);
        L.queue.pop_front();
      }
    }
    for (ServerReq& r : admit_now) {
      cudaStreamWaitEvent(r.field.dtype == EXTREMZ_F32 ? L.st32 : L.st64, r.ready, 0);
      cudaEventDestroy(r.ready);
      const extremz_field& f = r.field;
      int slot = -1;
      int rc = f.dtype == EXTREMZ_F32
                   ? L.e32.admit((const float*)f.orig, (float*)f.decp, f.width, f.height, f.depth,
                                 f.params, nullptr, 0, nullptr, r.ticket, &slot)
                   : L.e64.admit((const double*)f.orig, (double*)f.decp, f.width, f.height,
                                 f.depth, f.params, nullptr, 0, nullptr, r.ticket, &slot);
      ServerRunning run{r.ticket, r.footprint, r.t0, f.dtype, slot};
      if (rc != EXTREMZ_OK) {
        server_finish(s, run, rc, nullptr);
        continue;
      }
      L.running.push_back(run);
    }
    if (L.running.empty()) {
      // Blocked by the budget the other lane holds: wait for a release.
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_work.wait_for(lk, std::chrono::milliseconds(5));
      continue;
    }
    int rc = EXTREMZ_OK;
    const bool a32 = L.e32.active() > 0, a64 = L.e64.active() > 0;
    if (a32) rc = L.e32.tick_issue();
    if (rc == EXTREMZ_OK && a64) rc = L.e64.tick_issue();
    if (rc == EXTREMZ_OK && a32) rc = L.e32.tick_complete();
    if (rc == EXTREMZ_OK && a64) rc = L.e64.tick_complete();
    std::vector<ServerRunning> still;
    for (const ServerRunning& r : L.running) {
      const bool f32 = r.dtype == EXTREMZ_F32;
      const int pc = f32 ? L.e32.job(r.slot).pc : L.e64.job(r.slot).pc;
      if (rc == EXTREMZ_OK && pc != PC_DONE) {
        still.push_back(r);
        continue;
      }
      extremz_report rep;
      std::memset(&rep, 0, sizeof(rep));
      int status = rc;
      if (rc == EXTREMZ_OK) {
        if (f32) L.e32.fill_report(r.slot, &rep);
        else L.e64.fill_report(r.slot, &rep);
        status = rep.status;
      }
      if (f32) L.e32.release(r.slot);
      else L.e64.release(r.slot);
      server_finish(s, r, status, &rep);
    }
    L.running.swap(still);
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->stats.ticks += 1;
      if (rc != EXTREMZ_OK) {
        s->broken = rc;
        server_fail_queued(s, rc);
      }
    }
    s->cv_done.notify_all();
    if (rc != EXTREMZ_OK) {
      s->cv_work.notify_all();
      break;
    }
  }
  cudaStreamSynchronize(L.st32);
  cudaStreamSynchronize(L.st64);
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
  rc = ctx->c.ensure_pool();
  if (rc != EXTREMZ_OK) {
    if (prev != ctx->c.device) cudaSetDevice(prev);
    return (extremz_status)rc;
  }
  if (dtype == EXTREMZ_F32)
    rc = run_one(ctx->c.e32, st, nullptr, nullptr, nullptr, (const float*)d_orig, (float*)d_decp,
                 width, height, depth, *params, report, trace, trace_cap);
  else
    rc = run_one(ctx->c.e64, st, nullptr, nullptr, nullptr, (const double*)d_orig,
                 (double*)d_decp, width, height, depth, *params, report, trace, trace_cap);
  if (report) report->status = rc;
  if (prev != ctx->c.device) cudaSetDevice(prev);
  return (extremz_status)rc;
}

extremz_status extremz_mismatch_census(extremz_ctx* ctx, const void* d_orig, const void* d_field,
                                      int dtype, int width, int height, int depth, double thr,
                                      int32_t* counters, void* stream) {
  if (!ctx || !d_orig || !d_field || !counters) return EXTREMZ_BAD_ARG;
  extremz_params p;
  extremz_default_params(&p);
  p.thr = thr;
  int rc = check_args(dtype, width, height, depth, &p);
  if (rc != EXTREMZ_OK) return (extremz_status)rc;
  int prev = 0;
  cudaGetDevice(&prev);
  if (prev != ctx->c.device) cudaSetDevice(ctx->c.device);
  cudaStream_t st = (cudaStream_t)stream;
  extremz_report rep;
  std::memset(&rep, 0, sizeof(rep));
  rc = ctx->c.ensure_pool();
  // The census job reads the field and writes only its own workspace.
  if (rc == EXTREMZ_OK) {
    if (dtype == EXTREMZ_F32)
      rc = run_one<float>(ctx->c.e32, st, nullptr, nullptr, nullptr, (const float*)d_orig,
                   const_cast<float*>((const float*)d_field), width, height, depth, p, &rep,
                   nullptr, 0, nullptr, nullptr, true);
    else
      rc = run_one<double>(ctx->c.e64, st, nullptr, nullptr, nullptr, (const double*)d_orig,
                   const_cast<double*>((const double*)d_field), width, height, depth, p, &rep,
                   nullptr, 0, nullptr, nullptr, true);
  }
  std::memcpy(counters, rep.counters, sizeof(rep.counters));
  if (prev != ctx->c.device) cudaSetDevice(prev);
  return (extremz_status)rc;
}

extremz_status extremz_correct_host(extremz_ctx* ctx, const void* h_orig, void* h_decp, int dtype,
                                    int width, int height, int depth, const extremz_params* params,
                                    extremz_report* report, void* stream) {
  if (!ctx || !h_orig || !h_decp) return EXTREMZ_BAD_ARG;
  int rc = check_args(dtype, width, height, depth, params);
  if (rc != EXTREMZ_OK) return (extremz_status)rc;
  if (report) std::memset(report, 0, sizeof(*report));
  int prev = 0;
  cudaGetDevice(&prev);
  if (prev != ctx->c.device) cudaSetDevice(ctx->c.device);
  const long long N = (long long)width * height * depth;
  const size_t bytes = (size_t)N * (dtype == EXTREMZ_F32 ? 4 : 8);
  cudaStream_t st = (cudaStream_t)stream;
  rc = ctx->c.stage.reserve(2 * bytes + 512);
  if (rc == EXTREMZ_OK) rc = ctx->c.ensure_pool();
  if (rc == EXTREMZ_OK) rc = ctx->c.ensure_aux();
  if (rc != EXTREMZ_OK) {
    if (prev != ctx->c.device) cudaSetDevice(prev);
    return (extremz_status)rc;
  }
  ctx->c.stage.used = 0;
  char* df = ctx->c.stage.take<char>(bytes);
  char* dg = ctx->c.stage.take<char>(bytes);
  // The original field first, on the caller's stream; then the decompressed
  // field on the second stream, behind it on the bus, while the setup (which
  // reads only the original) runs.
  cudaStream_t aux = ctx->c.aux;
  if (cudaMemcpyAsync(df, h_orig, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaEventRecord(ctx->c.orig_in, st) != cudaSuccess ||
      cudaStreamWaitEvent(aux, ctx->c.orig_in, 0) != cudaSuccess ||
      cudaMemcpyAsync(dg, h_decp, bytes, cudaMemcpyHostToDevice, aux) != cudaSuccess ||
      cudaEventRecord(ctx->c.decp_in, aux) != cudaSuccess)
    rc = EXTREMZ_CUDA_ERR;
  long long moved = 0;
  if (rc == EXTREMZ_OK) {
    // The corrected voxels come back into h_decp inside run_one.
    if (dtype == EXTREMZ_F32) {
      HostWriteBack<float> wb{&ctx->c, static_cast<float*>(h_decp), ctx->c.decp_in};
      rc = run_one(ctx->c.e32, st, nullptr, nullptr, nullptr, (const float*)df, (float*)dg, width,
                   height, depth, *params, report, nullptr, 0, nullptr, &wb);
      moved = wb.moved;
    } else {
      HostWriteBack<double> wb{&ctx->c, static_cast<double*>(h_decp), ctx->c.decp_in};
      rc = run_one(ctx->c.e64, st, nullptr, nullptr, nullptr, (const double*)df, (double*)dg, width,
                   height, depth, *params, report, nullptr, 0, nullptr, &wb);
      moved = wb.moved;
    }
  }
  // Whatever happened, the copy in has ended before h_decp is written or
  // handed back.
  if (cudaEventSynchronize(ctx->c.decp_in) != cudaSuccess && rc == EXTREMZ_OK) rc = EXTREMZ_CUDA_ERR;
  if (report) {
    report->status = rc;
    report->host_bytes_back = moved;
  }
  if (prev != ctx->c.device) cudaSetDevice(prev);
  return (extremz_status)rc;
}

extremz_status extremz_edit_stream_caps(int dtype, int width, int height, int depth, int edit_type,
                                        long long* index_cap, long long* edits_cap) {
  if ((dtype != EXTREMZ_F32 && dtype != EXTREMZ_F64) || width <= 0 || height <= 0 || depth <= 0 ||
      (edit_type != 0 && edit_type != 1) || !index_cap || !edits_cap)
    return EXTREMZ_BAD_ARG;
  const long long n = (long long)width * height * depth;
  *index_cap = edit_type == 0 ? (3 * n + 7) / 8 : 4 * n;
  *edits_cap = n * (dtype == EXTREMZ_F32 ? 4 : 8);
  return EXTREMZ_OK;
}

extremz_status extremz_correct_encode(extremz_ctx* ctx, const void* d_orig, void* d_decp, int dtype,
                                      int width, int height, int depth,
                                      const extremz_params* params, extremz_report* report,
                                      void* stream, extremz_edit_stream* es) {
  if (!ctx || !d_orig || !d_decp || !es) return EXTREMZ_BAD_ARG;
  int rc = check_args(dtype, width, height, depth, params);
  if (rc != EXTREMZ_OK) return (extremz_status)rc;
  if (report) std::memset(report, 0, sizeof(*report));
  int prev = 0;
  cudaGetDevice(&prev);
  if (prev != ctx->c.device) cudaSetDevice(ctx->c.device);
  cudaStream_t st = (cudaStream_t)stream;
  rc = ctx->c.ensure_pool();
  if (rc == EXTREMZ_OK) {
    if (dtype == EXTREMZ_F32)
      rc = run_one(ctx->c.e32, st, nullptr, nullptr, nullptr, (const float*)d_orig,
                   (float*)d_decp, width, height, depth, *params, report, nullptr, 0, es);
    else
      rc = run_one(ctx->c.e64, st, nullptr, nullptr, nullptr, (const double*)d_orig,
                   (double*)d_decp, width, height, depth, *params, report, nullptr, 0, es);
  }
  if (report) report->status = rc;
  if (prev != ctx->c.device) cudaSetDevice(prev);
  return (extremz_status)rc;
}

long long extremz_zstd_size(const void* host, long long bytes, int level) {
  typedef size_t (*bound_fn)(size_t);
  typedef size_t (*compress_fn)(void*, size_t, const void*, size_t, int);
  typedef unsigned (*is_error_fn)(size_t);
  static void* h = dlopen("libzstd.so.1", RTLD_NOW | RTLD_LOCAL);
  if (!h || !host || bytes < 0) return -1;
  static bound_fn zbound = (bound_fn)dlsym(h, "ZSTD_compressBound");
  static compress_fn zcompress = (compress_fn)dlsym(h, "ZSTD_compress");
  static is_error_fn ziserr = (is_error_fn)dlsym(h, "ZSTD_isError");
  if (!zbound || !zcompress || !ziserr) return -1;
  std::vector<char> out(zbound((size_t)bytes));
  const size_t n = zcompress(out.data(), out.size(), host, (size_t)bytes, level);
  return ziserr(n) ? -1 : (long long)n;
}

extremz_status extremz_persistence_tree(extremz_ctx* ctx, const void* d_field, int dtype, int width,
                                       int height, int depth, int32_t* d_max_pairs,
                                       long long max_pairs_cap, int32_t* d_min_pairs,
                                       long long min_pairs_cap, int32_t* d_max_parent,
                                       int32_t* d_min_parent, long long* n_max, long long* n_min,
                                       void* stream) {
  if (!ctx || !d_field) return EXTREMZ_BAD_ARG;
  extremz_params p;
  extremz_default_params(&p);
  int rc = check_args(dtype, width, height, depth, &p);
  if (rc != EXTREMZ_OK) return (extremz_status)rc;
  int prev = 0;
  cudaGetDevice(&prev);
  if (prev != ctx->c.device) cudaSetDevice(ctx->c.device);
  cudaStream_t st = (cudaStream_t)stream;
  long long counts[2] = {0, 0};
  rc = ctx->c.ensure_pool();
  if (rc == EXTREMZ_OK) {
    if (dtype == EXTREMZ_F32)
      rc = analyze_one(ctx->c.e32, st, (const float*)d_field, width, height, depth, d_max_pairs,
                       max_pairs_cap, d_min_pairs, min_pairs_cap, counts, d_max_parent,
                       d_min_parent);
    else
      rc = analyze_one(ctx->c.e64, st, (const double*)d_field, width, height, depth, d_max_pairs,
                       max_pairs_cap, d_min_pairs, min_pairs_cap, counts, d_max_parent,
                       d_min_parent);
  }
  if (n_max) *n_max = counts[0];
  if (n_min) *n_min = counts[1];
  if (prev != ctx->c.device) cudaSetDevice(prev);
  return (extremz_status)rc;
}

extremz_status extremz_classify(extremz_ctx* ctx, const void* d_field, int dtype, int width,
                                int height, int depth, int8_t* d_type, int32_t* d_ds,
                                int32_t* d_as, void* stream) {
  if (!ctx || !d_field) return EXTREMZ_BAD_ARG;
  extremz_params p;
  extremz_default_params(&p);
  int rc = check_args(dtype, width, height, depth, &p);
  if (rc != EXTREMZ_OK) return (extremz_status)rc;
  int prev = 0;
  cudaGetDevice(&prev);
  if (prev != ctx->c.device) cudaSetDevice(ctx->c.device);
  cudaStream_t st = (cudaStream_t)stream;
  rc = ctx->c.ensure_pool();
  if (rc == EXTREMZ_OK) {
    if (dtype == EXTREMZ_F32)
      rc = classify_one(ctx->c.e32, st, (const float*)d_field, width, height, depth, d_type, d_ds,
                        d_as);
    else
      rc = classify_one(ctx->c.e64, st, (const double*)d_field, width, height, depth, d_type,
                        d_ds, d_as);
  }
  if (prev != ctx->c.device) cudaSetDevice(prev);
  return (extremz_status)rc;
}

extremz_status extremz_persistence_pairs(extremz_ctx* ctx, const void* d_field, int dtype,
                                        int width, int height, int depth, int32_t* d_max_pairs,
                                        long long max_pairs_cap, int32_t* d_min_pairs,
                                        long long min_pairs_cap, long long* n_max,
                                        long long* n_min, void* stream) {
  return extremz_persistence_tree(ctx, d_field, dtype, width, height, depth, d_max_pairs,
                                  max_pairs_cap, d_min_pairs, min_pairs_cap, nullptr, nullptr,
                                  n_max, n_min, stream);
}

extremz_status extremz_correct_batch(extremz_ctx* ctx, const extremz_field* fields, int n,
                                     extremz_report* reports, void* stream) {
  if (!ctx || (n > 0 && !fields) || n < 0) return EXTREMZ_BAD_ARG;
  if (reports) std::memset(reports, 0, sizeof(extremz_report) * (size_t)n);
  int prev = 0;
  cudaGetDevice(&prev);
  if (prev != ctx->c.device) cudaSetDevice(ctx->c.device);
  int rc = correct_batch(ctx->c, fields, n, reports, (cudaStream_t)stream);
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


extremz_status extremz_server_create(int device, const extremz_server_config* cfg,
                                     extremz_server** out) {
  if (!out) return EXTREMZ_BAD_ARG;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return EXTREMZ_NO_DEVICE;
  }
  if (device < 0 || device >= n) return EXTREMZ_BAD_ARG;
  const long long budget =
      cfg && cfg->hbm_budget_bytes > 0 ? cfg->hbm_budget_bytes : 120ll * 1000 * 1000 * 1000;
  const int max_jobs = cfg && cfg->max_jobs > 0 ? cfg->max_jobs : extremz::kMaxSel;
  if (max_jobs > extremz::kMaxSel) return EXTREMZ_BAD_ARG;
  if (cfg && (cfg->reserve_bytes < 0 || cfg->reserve_bytes > budget)) return EXTREMZ_BAD_ARG;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  extremz_server* s = new (std::nothrow) extremz_server;
  if (!s) return EXTREMZ_OOM;
  s->device = device;
  s->budget = budget;
  s->max_jobs = max_jobs;
  s->split = cfg && cfg->split_voxels != 0 ? cfg->split_voxels : 4ll << 20;
  s->nlanes = s->split < 0 ? 1 : kServerLanes;
  int rc = EXTREMZ_OK;
  int lo = 0, hi = 0;  // numerically lower = higher priority
  cudaDeviceGetStreamPriorityRange(&lo, &hi);
  for (int l = 0; l < s->nlanes && rc == EXTREMZ_OK; ++l) {
    const int prio = l == 0 ? hi : lo;
    if (cudaStreamCreateWithPriority(&s->lane[l].st32, cudaStreamNonBlocking, prio) != cudaSuccess ||
        cudaStreamCreateWithPriority(&s->lane[l].st64, cudaStreamNonBlocking, prio) != cudaSuccess)
      rc = EXTREMZ_CUDA_ERR;
  }
  if (rc == EXTREMZ_OK && !(s->pool = make_pool(device))) rc = EXTREMZ_OOM;
  for (int l = 0; l < s->nlanes && rc == EXTREMZ_OK; ++l) {
    ServerLane& L = s->lane[l];
    L.e32.set_stream(L.st32);
    L.e64.set_stream(L.st64);
    L.e32.set_pool(s->pool);
    L.e64.set_pool(s->pool);
    rc = L.e32.init(nullptr, nullptr);
    if (rc == EXTREMZ_OK) rc = L.e64.init(nullptr, nullptr);
  }
  // Grow the pool to the reservation now, so that admissions do not pay for
  // mapping new memory.
  if (rc == EXTREMZ_OK && cfg && cfg->reserve_bytes > 0) {
    void* p = nullptr;
    if (cudaMallocFromPoolAsync(&p, (size_t)cfg->reserve_bytes, s->pool, s->lane[0].st32) !=
            cudaSuccess ||
        cudaFreeAsync(p, s->lane[0].st32) != cudaSuccess ||
        cudaStreamSynchronize(s->lane[0].st32) != cudaSuccess)
      rc = EXTREMZ_OOM;
  }
  if (rc != EXTREMZ_OK) {
    cudaGetLastError();
    for (int l = 0; l < s->nlanes; ++l) {
      s->lane[l].e32.release_all();
      s->lane[l].e64.release_all();
      if (s->lane[l].st32) cudaStreamDestroy(s->lane[l].st32);
      if (s->lane[l].st64) cudaStreamDestroy(s->lane[l].st64);
    }
    if (s->pool) cudaMemPoolDestroy(s->pool);
    delete s;
    cudaSetDevice(prev);
    return (extremz_status)rc;
  }
  for (int l = 0; l < s->nlanes; ++l) s->lane[l].th = std::thread(server_loop, s, l);
  cudaSetDevice(prev);
  *out = s;
  return EXTREMZ_OK;
}

void extremz_server_destroy(extremz_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    for (int l = 0; l < s->nlanes; ++l) {
      for (ServerReq& q : s->lane[l].queue) cudaEventDestroy(q.ready);
      s->lane[l].queue.clear();
    }
  }
  s->cv_work.notify_all();
  for (int l = 0; l < s->nlanes; ++l)
    if (s->lane[l].th.joinable()) s->lane[l].th.join();
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(s->device);
  for (int l = 0; l < s->nlanes; ++l) {
    ServerLane& L = s->lane[l];
    L.e32.release_all();
    L.e64.release_all();
    cudaStreamSynchronize(L.st32);
    cudaStreamSynchronize(L.st64);
  }
  if (s->pool) cudaMemPoolDestroy(s->pool);
  for (int l = 0; l < s->nlanes; ++l) {
    cudaStreamDestroy(s->lane[l].st32);
    cudaStreamDestroy(s->lane[l].st64);
  }
  cudaSetDevice(prev);
  delete s;
}

extremz_status extremz_server_submit(extremz_server* s, const extremz_field* f, void* stream,
                                     long long* ticket) {
  if (!s || !f || !ticket || !f->orig || !f->decp) return EXTREMZ_BAD_ARG;
  int rc = check_args(f->dtype, f->width, f->height, f->depth, &f->params);
  if (rc != EXTREMZ_OK) return (extremz_status)rc;
  const long long fp = field_footprint(*f);
  if (fp > s->budget) return EXTREMZ_TOO_LARGE;
  ServerReq r;
  r.field = *f;
  r.field.params.flags &= ~EXTREMZ_FLAG_PROFILE;
  r.footprint = fp;
  const long long voxels = (long long)f->width * f->height * f->depth;
  const int li = (s->nlanes > 1 && voxels > s->split) ? 1 : 0;
  int prev = 0;
  cudaGetDevice(&prev);
  if (prev != s->device) cudaSetDevice(s->device);
  if (cudaEventCreateWithFlags(&r.ready, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventRecord(r.ready, (cudaStream_t)stream) != cudaSuccess) {
    last_cuda_error() = cudaGetLastError();
    if (r.ready) cudaEventDestroy(r.ready);
    if (prev != s->device) cudaSetDevice(prev);
    return EXTREMZ_CUDA_ERR;
  }
  if (prev != s->device) cudaSetDevice(prev);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->broken != EXTREMZ_OK || s->stop) {
      cudaEventDestroy(r.ready);
      return (extremz_status)(s->broken != EXTREMZ_OK ? s->broken : EXTREMZ_BAD_ARG);
    }
    r.ticket = s->next_ticket++;
    r.t0 = Clock::now();
    s->results[r.ticket] = ServerResult();
    s->lane[li].queue.push_back(r);
    s->stats.submitted += 1;
    s->stats.queued += 1;
    *ticket = r.ticket;
  }
  s->cv_work.notify_all();
  return EXTREMZ_OK;
}

static extremz_status server_take(extremz_server* s, long long ticket, extremz_report* report,
                                  double* latency_ms) {
  auto it = s->results.find(ticket);
  if (it == s->results.end()) return EXTREMZ_BAD_ARG;
  if (!it->second.done) return EXTREMZ_PENDING;
  if (report) *report = it->second.rep;
  if (latency_ms) *latency_ms = it->second.latency_ms;
  const int st = it->second.status;
  s->results.erase(it);
  return (extremz_status)st;
}

extremz_status extremz_server_poll(extremz_server* s, long long ticket, extremz_report* report,
                                   double* latency_ms) {
  if (!s) return EXTREMZ_BAD_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  return server_take(s, ticket, report, latency_ms);
}

extremz_status extremz_server_wait(extremz_server* s, long long ticket, int timeout_ms,
                                   extremz_report* report, double* latency_ms) {
  if (!s) return EXTREMZ_BAD_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto ready = [&] {
    auto it = s->results.find(ticket);
    return it == s->results.end() || it->second.done;
  };
  if (timeout_ms < 0) s->cv_done.wait(lk, ready);
  else s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready);
  return server_take(s, ticket, report, latency_ms);
}

long long extremz_job_footprint(int dtype, int width, int height, int depth) {
  if ((dtype != EXTREMZ_F32 && dtype != EXTREMZ_F64) || width <= 0 || height <= 0 || depth <= 0)
    return -1;
  extremz_field f;
  std::memset(&f, 0, sizeof(f));
  f.dtype = dtype;
  f.width = width;
  f.height = height;
  f.depth = depth;
  return field_footprint(f);
}

void extremz_server_get_stats(extremz_server* s, extremz_server_stats* out) {
  if (!s || !out) return;
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  out->kernel_launches = 0;
  for (int l = 0; l < s->nlanes; ++l)
    out->kernel_launches += s->lane[l].e32.launches() + s->lane[l].e64.launches();
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
      return "field larger than the static workspace of the allocation-free entry point, "
             "or than the server's HBM budget";
    case EXTREMZ_PENDING: return "request still queued or running";
    default: return "unknown status";
  }
}

const char* extremz_last_cuda_error(void) { return cudaGetErrorString(last_cuda_error()); }

}  // extern "C"

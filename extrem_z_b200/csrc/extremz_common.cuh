// Shared device helpers for the ExtreM correction kernels (sm_100a).
//
// Grid convention (src/ExtreM_cuda.cu:649-651): vertex id v = x + y*W + z*W*H,
// x fastest.  Neighbourhood: the 14 Freudenthal directions in the reference's
// order (src/ExtreM_cuda.cu:155-162); star lists and LUT bit positions follow
// this order.  Total order: a above b  <=>  f[a] > f[b] || (f[a] == f[b] && a > b)
// (islarger/isless, src/ExtreM_cuda.cu:1779-1793).
#pragma once

#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace extremz {

constexpr int kNumDirs = 14;
constexpr int kLutSize = 24800;
constexpr int kNumKeys = 27;
constexpr int kRowStride = 16;  // 14 labels, [14] = count, [15] unused
constexpr int kCatMax = 1, kCatMin = 2, kCatSaddle = 4;
constexpr int kCatShift = 29;   // list entry = v | (cat << 29); needs N < 2^29
constexpr int kInf = 0x7fffffff;

__host__ __device__ constexpr int dir_x(int d) {
  return d == 0 ? 1 : d == 1 ? -1 : d == 6 ? -1 : d == 7 ? 1 : d == 10 ? -1 : d == 11 ? 1
       : d == 12 ? -1 : d == 13 ? 1 : 0;
}
__host__ __device__ constexpr int dir_y(int d) {
  return d == 2 ? 1 : d == 3 ? -1 : d == 6 ? 1 : d == 7 ? -1 : d == 8 ? 1 : d == 9 ? -1
       : d == 12 ? 1 : d == 13 ? -1 : 0;
}
__host__ __device__ constexpr int dir_z(int d) {
  return d == 4 ? 1 : d == 5 ? -1 : d == 8 ? 1 : d == 9 ? -1 : d == 10 ? 1 : d == 11 ? -1
       : d == 12 ? 1 : d == 13 ? -1 : 0;
}
// For every valid neighbour r = v + off(d), off(d) > 0 exactly for even d, so
// an index tie-break "r < v" is "d is odd".
__host__ __device__ constexpr bool dir_neighbour_is_before(int d) { return (d & 1) != 0; }

// Neighbour ids in ascending order, by rank j = 0..13: the centre falls
// between ranks 6 and 7.  Among the valid neighbours of any vertex the offsets
// dx + dy*W + dz*W*H are distinct and ordered as (dz, dy, dx) lexicographically
// (the ones that would tie are never valid together), so comparing ids of
// neighbours is comparing these static ranks.
__host__ __device__ constexpr int rank_dir(int j) {
  return j == 0 ? 9 : j == 1 ? 13 : j == 2 ? 5 : j == 3 ? 11 : j == 4 ? 3 : j == 5 ? 7
       : j == 6 ? 1 : j == 7 ? 0 : j == 8 ? 6 : j == 9 ? 2 : j == 10 ? 10 : j == 11 ? 4
       : j == 12 ? 12 : 8;
}
constexpr int kRankCentre = 7;  // the centre comes before rank_dir(7)

// Bit mask of the valid directions for boundary code bc (0x3fff inside).
__host__ __device__ __forceinline__ int valid_mask(int bc);

// Device tables: LUT entries (int8), key index / LUT offset per boundary code.
struct DeviceTables {
  const int8_t* lut;      // 24 800 entries, the reference's LUT.bin layout
  const int* key_offset;  // 64 entries: boundary code -> LUT offset, -1 unknown key
};

// Boundary code of (x, y, z): bit 0 = x-1 invalid, 1 = x+1 invalid, 2 = y-1,
// 3 = y+1, 4 = z-1, 5 = z+1.
__device__ __forceinline__ int boundary_code(int x, int y, int z, int W, int H, int D) {
  return (x == 0) | ((x == W - 1) << 1) | ((y == 0) << 2) | ((y == H - 1) << 3) |
         ((z == 0) << 4) | ((z == D - 1) << 5);
}

// Direction d valid at boundary code bc.
__host__ __device__ __forceinline__ bool dir_valid(int d, int bc) {
  const int dx = dir_x(d), dy = dir_y(d), dz = dir_z(d);
  if (dx < 0 && (bc & 1)) return false;
  if (dx > 0 && (bc & 2)) return false;
  if (dy < 0 && (bc & 4)) return false;
  if (dy > 0 && (bc & 8)) return false;
  if (dz < 0 && (bc & 16)) return false;
  if (dz > 0 && (bc & 32)) return false;
  return true;
}

__host__ __device__ __forceinline__ int valid_mask(int bc) {
  if (bc == 0) return (1 << kNumDirs) - 1;
  int m = 0;
#pragma unroll
  for (int d = 0; d < kNumDirs; ++d) m |= dir_valid(d, bc) << d;
  return m;
}

// ---------------------------------------------------------------------------
// TMA (bulk tensor copy) with an mbarrier, for halo tiles.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes)
               : "memory");
}
// Bounded wait for phase `parity`; returns false when the limit is reached.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, long long limit) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
  for (long long it = 0; it < limit; ++it) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
// 3-D tiled bulk copy global -> shared.  x must be a multiple of 16 bytes
// (callers start boxes 4 elements left of a 32-aligned tile origin).
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            uint64_t* bar) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const unsigned b = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(d),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(b)
      : "memory");
}

// ---------------------------------------------------------------------------
// Order-preserving integer keys for the delta atomic max.  The reference merges
// proposals with a CAS loop on doubles (swap/swap1, :2643-2691); an integer
// atomicMax on monotone keys gives the same maximum in one instruction.
// ---------------------------------------------------------------------------
template <class T> struct KeyOf;
template <> struct KeyOf<double> {
  using K = unsigned long long;
  __host__ __device__ static K enc(double v) {
#ifdef __CUDA_ARCH__
    K u = (K)__double_as_longlong(v);
#else
    K u; __builtin_memcpy(&u, &v, 8);
#endif
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
  }
  __host__ __device__ static double dec(K k) {
    K u = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)u);
#else
    double v; __builtin_memcpy(&v, &u, 8); return v;
#endif
  }
};
template <> struct KeyOf<float> {
  using K = unsigned int;
  __host__ __device__ static K enc(float v) {
#ifdef __CUDA_ARCH__
    K u = (K)__float_as_uint(v);
#else
    K u; __builtin_memcpy(&u, &v, 4);
#endif
    return (u >> 31) ? ~u : (u | 0x80000000u);
  }
  __host__ __device__ static float dec(K k) {
    K u = (k >> 31) ? (k & 0x7fffffffu) : ~k;
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float v; __builtin_memcpy(&v, &u, 4); return v;
#endif
  }
};

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

// Warp-aggregated append: one atomic per warp.  All lanes named in `mask`
// must call it.  Returns the slot for lanes with pred, else -1.
__device__ __forceinline__ int warp_append(int* count, bool pred, unsigned mask) {
  unsigned b = __ballot_sync(mask, pred);
  if (b == 0) return -1;
  int leader = __ffs(b) - 1;
  int base = 0;
  if ((int)lane_id() == leader) base = atomicAdd(count, __popc(b));
  base = __shfl_sync(mask, base, leader);
  unsigned lt = (1u << lane_id()) - 1u;
  return pred ? base + __popc(b & lt) : -1;
}

// Total-order comparisons (value, then id).
template <class T>
__device__ __forceinline__ bool above(T au, int u, T av, int v) {
  return au > av || (au == av && u > v);
}
template <class T>
__device__ __forceinline__ bool below(T au, int u, T av, int v) {
  return au < av || (au == av && u < v);
}

struct Dims {
  int W, H, D, N;
};

// Coordinates of v.
__device__ __forceinline__ void coords(int v, const Dims& g, int& x, int& y, int& z) {
  x = v % g.W;
  int t = v / g.W;
  y = t % g.H;
  z = t / g.H;
}

// Valid neighbours of v in direction order: writes ids and direction indices,
// returns the count.
__device__ __forceinline__ int neighbours(int v, const Dims& g, int* ids, int* dirs) {
  int x, y, z;
  coords(v, g, x, y, z);
  int bc = boundary_code(x, y, z, g.W, g.H, g.D);
  int k = 0;
#pragma unroll
  for (int d = 0; d < kNumDirs; ++d) {
    if (dir_valid(d, bc)) {
      ids[k] = v + dir_x(d) + dir_y(d) * g.W + dir_z(d) * g.W * g.H;
      if (dirs) dirs[k] = d;
      ++k;
    }
  }
  return k;
}

}  // namespace extremz

// Edit stream of a corrected field on the device: the reference's cost()
// (src/ExtreM_cuda.cu:4557-4675, edit_type 0) and floating_point_cost()
// (:4677-4797, edit_type 1) without their files and zstd step.
//
// A voxel is edited when its corrected value differs from the decompressed
// value it came in with (decp_data_copy[i] != decp_data[i]).
//  * edit_type 0: the index stream packs every voxel's edit counter (0 when
//    not edited) three bits per voxel, LSB first, as encodeTo3BitBitmap
//    (:4282-4312) does; the edit stream holds the snapped voxels'
//    (counter == q) lossless edits -(decp - (input - bound)) in id order.
//  * edit_type 1: the index stream holds the edited voxels' ids delta-coded
//    (get_diff_index :4315-4323) as int32; the edit stream every edited
//    voxel's -(decp - (input - bound)) in id order.
// Both lists are ordered compactions (block counts, one scan, writes); the
// 3-bit stream is written a byte per thread.  PSNR before and after follows
// calculatePSNR (:4263-4280), with the original's value range.
#pragma once

#include "extremz_kernels.cuh"

namespace extremz {

template <class T>
__device__ __forceinline__ int enc_bits(const T* __restrict__ d0, const T* __restrict__ d1,
                                        const int* __restrict__ counter, int v, int q, int et) {
  if (!(d0[v] != d1[v])) return 0;
  return 1 | ((et == 1 || counter[v] == q) ? 2 : 0);
}

// Per 1024-voxel block: edited voxels (list 0) and edit entries (list 1).
template <class T>
__global__ void __launch_bounds__(kCpBlock) k_enc_count(const T* __restrict__ d0,
                                                        const T* __restrict__ d1,
                                                        const int* __restrict__ counter, int N,
                                                        int q, int et, int* __restrict__ bcount) {
  __shared__ int cnt[2];
  if (threadIdx.x < 2) cnt[threadIdx.x] = 0;
  __syncthreads();
  const int v = blockIdx.x * kCpBlock + threadIdx.x;
  const int b = v < N ? enc_bits(d0, d1, counter, v, q, et) : 0;
  for (int l = 0; l < 2; ++l) {
    const unsigned m = __ballot_sync(0xffffffffu, (b >> l) & 1);
    if (lane_id() == 0 && m) atomicAdd(&cnt[l], __popc(m));
  }
  __syncthreads();
  if (threadIdx.x < 2) bcount[threadIdx.x * gridDim.x + blockIdx.x] = cnt[threadIdx.x];
}

// Ordered writes: edited ids (edit_type 1) and edit values, in id order.
template <class T>
__global__ void __launch_bounds__(kCpBlock) k_enc_write(const T* __restrict__ f,
                                                        const T* __restrict__ d0,
                                                        const T* __restrict__ d1,
                                                        const int* __restrict__ counter, int N,
                                                        T bound, int q, int et,
                                                        const int* __restrict__ boff,
                                                        int* __restrict__ ids,
                                                        T* __restrict__ edits) {
  __shared__ int wcnt[2][32];
  const int v = blockIdx.x * kCpBlock + threadIdx.x;
  const int b = v < N ? enc_bits(d0, d1, counter, v, q, et) : 0;
  const unsigned lt = (1u << lane_id()) - 1u;
  unsigned m[2];
  for (int l = 0; l < 2; ++l) {
    m[l] = __ballot_sync(0xffffffffu, (b >> l) & 1);
    if (lane_id() == 0) wcnt[l][threadIdx.x / 32] = __popc(m[l]);
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    for (int l = 0; l < 2; ++l) {
      const int w = wcnt[l][threadIdx.x];
      int wi = w;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, wi, o);
        if (lane_id() >= (unsigned)o) wi += y;
      }
      wcnt[l][threadIdx.x] = wi - w;
    }
  }
  __syncthreads();
  if ((b & 1) && et == 1) {
    const int pos = boff[blockIdx.x] + wcnt[0][threadIdx.x / 32] + __popc(m[0] & lt);
    ids[pos] = v;
  }
  if (b & 2) {
    const int pos = boff[gridDim.x + blockIdx.x] + wcnt[1][threadIdx.x / 32] + __popc(m[1] & lt);
    edits[pos] = -(d0[v] - (f[v] - bound));
  }
}

// Delta coding of the ascending edited ids: out[0] = ids[0], out[k] = ids[k] - ids[k-1].
__global__ void k_enc_diff(const int* __restrict__ ids, int n, int* __restrict__ out) {
  const int stride = gridDim.x * blockDim.x;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride)
    out[k] = k ? ids[k] - ids[k - 1] : ids[0];
}

// The 3-bit counter stream, one output byte per thread: byte j holds bits
// [8j, 8j + 8) of the LSB-first stream, value i at bits [3i, 3i + 3).
template <class T>
__global__ void k_enc_pack3(const T* __restrict__ d0, const T* __restrict__ d1,
                            const int* __restrict__ counter, long long N, uint8_t* __restrict__ out,
                            long long nbytes, unsigned long long* err) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < nbytes; j += stride) {
    unsigned byte = 0;
    long long cur = -1;
    int val = 0;
    for (int b = 0; b < 8; ++b) {
      const long long t = 8 * j + b, i = t / 3;
      if (i >= N) break;
      if (i != cur) {
        cur = i;
        val = d0[i] != d1[i] ? counter[i] : 0;
        if (val < 0 || val > 7) atomicOr(err, 1ull);
      }
      byte |= (unsigned)((val >> (int)(t % 3)) & 1) << b;
    }
    out[j] = (uint8_t)byte;
  }
}

// Sums of squared errors before / after (doubles, atomicAdd per block) and
// the original's min / max (order-preserving keys).
template <class T>
__global__ void __launch_bounds__(256) k_enc_stats(const T* __restrict__ f, const T* __restrict__ d0,
                                                   const T* __restrict__ d1, int N,
                                                   unsigned long long* acc) {
  double s0 = 0.0, s1 = 0.0;
  double lo = INFINITY, hi = -INFINITY;
  const int stride = gridDim.x * blockDim.x;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < N; v += stride) {
    const double fv = (double)f[v];
    const double e0 = fv - (double)d0[v], e1 = fv - (double)d1[v];
    s0 += e0 * e0;
    s1 += e1 * e1;
    lo = fmin(lo, fv);
    hi = fmax(hi, fv);
  }
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if (lane_id() == 0) {
    atomicAdd(reinterpret_cast<double*>(acc + 0), s0);
    atomicAdd(reinterpret_cast<double*>(acc + 1), s1);
    atomicMin(acc + 2, KeyOf<double>::enc(lo));
    atomicMax(acc + 3, KeyOf<double>::enc(hi));
  }
}

// List of the voxels whose value changed during a correction, for the
// host-buffer entry point: the caller's buffer already holds the decompressed
// field, so only these voxels travel back.  `bits` is the bitset k_apply
// keeps (Job::edited); one warp per 32 words (1024 voxels), one count per
// block, then (after k_scan_lists) ids and corrected values in id order.
__global__ void __launch_bounds__(32) k_edit_count(const unsigned* __restrict__ bits, int N,
                                                   int* __restrict__ bcount) {
  const int w = blockIdx.x * 32 + threadIdx.x;
  int c = w < (N + 31) / 32 ? __popc(bits[w]) : 0;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if (threadIdx.x == 0) bcount[blockIdx.x] = c;
}

template <class T>
__global__ void __launch_bounds__(32) k_edit_write(const unsigned* __restrict__ bits,
                                                   const T* __restrict__ g, int N,
                                                   const int* __restrict__ boff,
                                                   int* __restrict__ ids, T* __restrict__ vals) {
  const int w = blockIdx.x * 32 + threadIdx.x;
  unsigned m = w < (N + 31) / 32 ? bits[w] : 0u;
  const int c = __popc(m);
  int incl = c;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane_id() >= (unsigned)o) incl += y;
  }
  int pos = boff[blockIdx.x] + incl - c;
  while (m) {
    const int v = w * 32 + __ffs(m) - 1;
    m &= m - 1;
    ids[pos] = v;
    vals[pos] = g[v];
    ++pos;
  }
}

}  // namespace extremz

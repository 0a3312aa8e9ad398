// Merge-tree persistence pairs of a field on the device: the extremum-graph
// pairing of the reference's constructPersistencePairs (src/ExtreM.cpp
// :1863-1918, called by compute_MergeT :2930-2952), for the split tree
// (maxima with merge saddles of superlevel sets) and the join tree (minima
// with merge saddles of sublevel sets), from the field's own extrema,
// manifold labels and merge vertices (vertices whose upper, respectively
// lower, link has two or more components).
//
// Order.  The split tree ranks vertices by (value, id); the join tree by the
// reverse order.  Extrema are ranked ascending in the tree's order (the
// global extremum last), saddles descending (the "largest" saddle first).
// Row i of saddle i holds the distinct ranks of the extrema reached by the
// steepest paths of its neighbours on the tree's side (its descending- or
// ascending-manifold labels), ascending; a row with one entry is emptied.
//
// Rounds (:1878-1906): every extremum takes the first (largest) saddle whose
// row holds it; an extremum that is its saddle's smallest entry pairs with it
// and points to the saddle's largest entry; pointers are compressed
// (:1908-1921) and every row is rewritten through them, deduplicated, and
// emptied when one entry is left (:1923-1932).  Rounds repeat until none
// pairs.  The global extremum pairs with the opposite global extremum (:1937).
#pragma once

#include <cub/cub.cuh>

#include "extremz_kernels.cuh"

namespace extremz {

constexpr int kPpRow = 16;  // entries per row (<= 14 neighbours)

// Link adjacency of the 14-neighbourhood: two neighbours are joined by a link
// edge when their offset is itself one of the 14 directions.
__host__ __device__ constexpr int link_adj(int a) {
  int m = 0;
  for (int b = 0; b < kNumDirs; ++b) {
    if (a == b) continue;
    const int dx = dir_x(b) - dir_x(a), dy = dir_y(b) - dir_y(a), dz = dir_z(b) - dir_z(a);
    for (int c = 0; c < kNumDirs; ++c)
      if (dir_x(c) == dx && dir_y(c) == dy && dir_z(c) == dz) m |= 1 << b;
  }
  return m;
}

// Connected components of a set of link vertices (bit d = direction d).
__device__ __forceinline__ int link_comps(int nodes) {
  int comps = 0, left = nodes;
  while (left) {
    int comp = left & -left;
    for (;;) {
      int grow = comp;
#pragma unroll
      for (int d = 0; d < kNumDirs; ++d)
        if (comp >> d & 1) grow |= link_adj(d) & nodes;
      if (grow == comp) break;
      comp = grow;
    }
    left &= ~comp;
    ++comps;
  }
  return comps;
}

// Merge vertices of the two trees, from the link itself rather than the
// lookup table (which has no entries for grids thinner than 3 voxels): bit 0
// when the upper link (split tree) has two or more components, bit 1 when the
// lower link (join tree) has.
template <class T>
__device__ __forceinline__ int merge_bits(const T* __restrict__ a, const Dims& g, int v) {
  int x, y, z;
  coords(v, g, x, y, z);
  const int valid = valid_mask(boundary_code(x, y, z, g.W, g.H, g.D));
  const T c = a[v];
  int up = 0;
#pragma unroll
  for (int d = 0; d < kNumDirs; ++d) {
    if (!(valid >> d & 1)) continue;
    const int u = v + dir_x(d) + dir_y(d) * g.W + dir_z(d) * g.W * g.H;
    if (above(a[u], u, c, v)) up |= 1 << d;
  }
  return (link_comps(up) >= 2 ? 1 : 0) | (link_comps(valid & ~up) >= 2 ? 2 : 0);
}

// Ordered compaction of the merge vertices (split list 0, join list 1): block
// counts, then (after k_scan_lists) the writes in ascending id.
template <class T>
__global__ void __launch_bounds__(kCpBlock) k_pp_cand_count(const T* __restrict__ a, Dims g,
                                                            int* __restrict__ bcount) {
  __shared__ int cnt[2];
  if (threadIdx.x < 2) cnt[threadIdx.x] = 0;
  __syncthreads();
  const int v = blockIdx.x * kCpBlock + threadIdx.x;
  const int b = v < g.N ? merge_bits(a, g, v) : 0;
  for (int l = 0; l < 2; ++l) {
    const unsigned m = __ballot_sync(0xffffffffu, (b >> l) & 1);
    if (lane_id() == 0 && m) atomicAdd(&cnt[l], __popc(m));
  }
  __syncthreads();
  if (threadIdx.x < 2) bcount[threadIdx.x * gridDim.x + blockIdx.x] = cnt[threadIdx.x];
}

template <class T>
__global__ void __launch_bounds__(kCpBlock) k_pp_cand_write(const T* __restrict__ a, Dims g,
                                                            const int* __restrict__ boff,
                                                            int* __restrict__ split,
                                                            int* __restrict__ join) {
  __shared__ int wcnt[2][32];
  const int v = blockIdx.x * kCpBlock + threadIdx.x;
  const int b = v < g.N ? merge_bits(a, g, v) : 0;
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
  int* outs[2] = {split, join};
  for (int l = 0; l < 2; ++l)
    if ((b >> l) & 1)
      outs[l][boff[l * gridDim.x + blockIdx.x] + wcnt[l][threadIdx.x / 32] + __popc(m[l] & lt)] = v;
}

// Sort keys: 64-bit order-preserving value key, complemented for a
// descending sort.  -0 is keyed as +0: the total order compares values, and
// the two zeros are equal values (ties go by id).
template <class T>
__global__ void k_pp_keys(const T* __restrict__ a, const int* __restrict__ list, int n, bool reverse,
                          bool complement, unsigned long long* __restrict__ keys,
                          int* __restrict__ vals) {
  const int stride = gridDim.x * blockDim.x;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
    const int li = reverse ? n - 1 - k : k;  // ties keep the input's id order
    T v = a[list[li]];
    if (v == T(0)) v = T(0);
    const unsigned long long key = (unsigned long long)KeyOf<T>::enc(v);
    keys[k] = complement ? ~key : key;
    vals[k] = li;
  }
}

// rank[list index] = position in the sorted order.
__global__ void k_pp_rank(const int* __restrict__ sorted_li, int n, int* __restrict__ rank) {
  const int stride = gridDim.x * blockDim.x;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) rank[sorted_li[p]] = p;
}

// Row of each saddle (by sorted position): distinct extremum ranks of the
// labels of its neighbours on the tree's side, ascending.
template <class T, bool kMax>
__global__ void k_pp_rows(const T* __restrict__ a, Dims g, const int* __restrict__ sad,
                          const int* __restrict__ sorted_li, int ns, const int* __restrict__ lab,
                          const int* __restrict__ ext, const int* __restrict__ erank,
                          int* __restrict__ rows, int* __restrict__ cnt) {
  const int stride = gridDim.x * blockDim.x;
  const int WH = g.W * g.H;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += stride) {
    const int s = sad[sorted_li[i]];
    int x, y, z;
    coords(s, g, x, y, z);
    const int valid = valid_mask(boundary_code(x, y, z, g.W, g.H, g.D));
    const T sv = a[s];
    int r[kPpRow];
    int n = 0;
    for (int d = 0; d < kNumDirs; ++d) {
      if (!(valid >> d & 1)) continue;
      const int v = s + dir_x(d) + dir_y(d) * g.W + dir_z(d) * WH;
      const T vv = a[v];
      if (!(kMax ? above(vv, v, sv, s) : below(vv, v, sv, s))) continue;
      const int e = erank[ext[lab[v]]];
      int j = n;  // insertion, dropping duplicates
      bool dup = false;
      for (int q = 0; q < n; ++q) dup |= r[q] == e;
      if (dup) continue;
      while (j > 0 && r[j - 1] > e) {
        r[j] = r[j - 1];
        --j;
      }
      r[j] = e;
      ++n;
    }
    if (n == 1) n = 0;
    for (int q = 0; q < n; ++q) rows[(long long)i * kPpRow + q] = r[q];
    cnt[i] = n;
  }
}

// Largest saddle of every extremum but the global one.
__global__ void k_pp_largest(const int* __restrict__ rows, const int* __restrict__ cnt, int ns,
                             int glob, int* __restrict__ largest) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += stride)
    for (int q = 0; q < cnt[i]; ++q) {
      const int e = rows[(long long)i * kPpRow + q];
      if (e != glob) atomicMin(largest + e, i);
    }
}

// Pairing of the round; resets largest for the next round.  lmax keeps the
// extremum each paired one merges into (its saddle row's largest entry, the
// second element of the reference's maximaTriplets, :2187), which ptr then
// loses to compression.
__global__ void k_pp_pair(const int* __restrict__ rows, const int* __restrict__ cnt, int ne, int ns,
                          int* __restrict__ largest, int* __restrict__ ptr, int* __restrict__ pair,
                          int* __restrict__ lmax, int* changed) {
  const int stride = gridDim.x * blockDim.x;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += stride) {
    const int i = largest[e];
    largest[e] = kInf;
    if (i >= ns || pair[e] >= 0) continue;
    if (rows[(long long)i * kPpRow] == e) {
      pair[e] = i;
      const int l = rows[(long long)i * kPpRow + cnt[i] - 1];
      ptr[e] = l;
      lmax[e] = l;
      *changed = 1;
    }
  }
}

// Pointer compression to the surviving extremum.
__global__ void k_pp_jump(int* __restrict__ ptr, int ne, int cap, int* err) {
  const int stride = gridDim.x * blockDim.x;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += stride) {
    int u = ptr[e], it = 0;
    while (ptr[u] != u && it < cap) {
      u = ptr[u];
      ++it;
    }
    if (it == cap) atomicOr(err, kErrJump);
    ptr[e] = u;
  }
}

// Rows rewritten through the pointers, deduplicated, emptied at one entry.
__global__ void k_pp_remap(int* __restrict__ rows, int* __restrict__ cnt, int ns,
                           const int* __restrict__ ptr) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += stride) {
    const int c = cnt[i];
    if (c == 0) continue;
    int r[kPpRow];
    int n = 0;
    for (int q = 0; q < c; ++q) {
      const int e = ptr[rows[(long long)i * kPpRow + q]];
      int j = n;
      bool dup = false;
      for (int k = 0; k < n; ++k) dup |= r[k] == e;
      if (dup) continue;
      while (j > 0 && r[j - 1] > e) {
        r[j] = r[j - 1];
        --j;
      }
      r[j] = e;
      ++n;
    }
    if (n == 1) n = 0;
    for (int q = 0; q < n; ++q) rows[(long long)i * kPpRow + q] = r[q];
    cnt[i] = n;
  }
}

__global__ void k_iota(int* __restrict__ p, int n) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) p[i] = i;
}

// Output pairs (partner vertex, extremum vertex) by extremum rank; the global
// extremum's partner is the opposite global extremum, an unpaired one -1.
// parent (optional): the vertex of the extremum each one merges into (lmax),
// the global extremum its own, an unpaired one -1.
__global__ void k_pp_out(const int* __restrict__ pair, int ne, const int* __restrict__ ext_li,
                         const int* __restrict__ elist, const int* __restrict__ sad_li,
                         const int* __restrict__ slist, int opposite, int* __restrict__ out,
                         const int* __restrict__ lmax, int* __restrict__ parent) {
  const int stride = gridDim.x * blockDim.x;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += stride) {
    const int i = pair[e];
    out[2 * e] = e == ne - 1 ? opposite : (i >= 0 ? slist[sad_li[i]] : -1);
    out[2 * e + 1] = elist[ext_li[e]];
    if (parent)
      parent[e] = e == ne - 1 ? elist[ext_li[e]] : (i >= 0 ? elist[ext_li[lmax[e]]] : -1);
  }
}

}  // namespace extremz

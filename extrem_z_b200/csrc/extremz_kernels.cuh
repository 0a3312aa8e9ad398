// ExtreM correction kernels for sm_100a.
//
// Each kernel replaces one or more kernels of the reference GPU path
// (src/ExtreM_cuda.cu); the comment on each names them.  Integer, label and
// comparison work is exact; floating-point updates repeat the reference's
// operations in the field type T (build with -fmad=false).
#pragma once

#include "extremz_common.cuh"

namespace extremz {

// ---------------------------------------------------------------------------
// Per-job device state passed by value to every kernel.
// ---------------------------------------------------------------------------
template <class T>
struct Job {
  using K = typename KeyOf<T>::K;
  Dims dim;
  const T* f;  // original field
  T* g;        // decompressed field, corrected in place
  T* g0;       // copy of the decompressed field as it came in (edit streams only)
  T bound, thr, sentinel;
  K sentinel_key;
  int q, edit_type;

  int8_t* otype;      // original vertex type (-1, 0..5)
  uint16_t* olm;      // original lower-star direction mask
  uint8_t* ocnt2; uint8_t* ocnt1;  // original row counts (compact copy of row[14])
  int* ds; int* as;   // original steepest ascent / descent roots
  int* dds; int* das; // decompressed roots
  int* ext;           // vertex -> index in the maxima / minima list

  K* delta;           // proposal buffer (order-preserving keys), sentinel between phases
  int* counter;       // delta_counter of the reference (starts at -1)
  int* touched;       // vertices whose delta left the sentinel in this phase
  int* mm;            // mismatch list: v | cat << 29
  int* mm_next;       // the list being rebuilt by the incremental detection
  uint8_t* mstat;     // current mismatch categories of every vertex
  int* dirty;         // vertices whose value changed since the last detection
  int* dstamp;        // dirty-list membership stamps (== dirty epoch)
  int* rstamp;        // re-evaluation stamps (== detection epoch)
  unsigned long long* claim;  // wrong-neighbour arbitration, (round << 32) | ~saddle
  int* taken;         // wrong-neighbour flag stamps (== call id when flagged)
  int* taken1;
  int* cand; int* cand_next;  // wrong-neighbour candidate saddles (side being resolved)
  int* cand_j;        // join-side candidates, produced with the split side's
  int* flagged; int* flagged1;  // flagged neighbours (split / join)
  uint8_t* mis;       // per vertex: 1 if dds != ds, 2 if das != as
  unsigned* vchg;     // bitset: vertices whose value changed since the last computed round
  unsigned* edited;   // bitset: vertices whose value changed in this correction (or null)
  uint8_t* dirtyv;    // per vertex: the round stamp's low byte when an input of its saddle
                      // rows changed in that round
  int* bdirty;        // per 1024-id block: the round stamp when some dirtyv byte in it was
                      // set (when N % 4 == 0)
  uint8_t* has2; uint8_t* has1;  // per saddle row: its wrong-neighbour seed bit
  int* hcnt;          // per saddle-pass chunk: seed bits set in it
  int* cpoff;         // per list (2-saddles, 1-saddles, maxima, minima) and
                      // 1024-id block: offset of the block's first entry
  int* pdd; int* pda; // decompressed steepest pointers, tile-compressed (k_direction)
  uint8_t* tdirty;    // per tile: a value in the tile or its halo changed since
                      // the tile's pointers were computed
  unsigned* rtouch2; unsigned* rtouch1;  // bitsets: labels (of dds / das) of the vertices of
                                         // the tiles whose pointers this round recomputes

  int* sad2; int* sad1; int* maxima; int* minima;
  int* orow2; int* orow1;  // original rows of kRowStride ints: entries 4 .. count-1 as
                           // extremum indices, -1 for a repeated label (the first four
                           // are in orm2 / orm1)
  int4* orm2; int4* orm1;  // per row: its first four entries as extremum indices (-1 past the
                           // count and for a repeated label; rows are in direction order)
  int4* oend2; int4* oend1;  // per row: first and last entry, then both as extremum indices
  int* drow2; int* drow1;  // decompressed rows: 2 persistent slots per row, see k_saddle_pass
  int* largest; int* smallest;  // per maximum / minimum
  int* first1; int* flag2;      // per maximum: wrong_index_max arbitration
  int* first_min1; int* flag_min2;
  int* first_s; int* first_sj;  // per extremum: its first wrong saddle-row entry (kept across scans)
  int* moff2; int* ment2;       // per maximum: the row entries (i * kRowStride + p) that name it
  int* moff1; int* ment1;       // per minimum: the same over the 1-saddles' rows
  int* wstamp2; int* wstamp1;   // per extremum: the wrong-saddle epoch that last queued it
  int* aff;                     // extrema queued for the wrong-saddle update
  int* wlong;                   // of those, the ones with long entry lists
  unsigned* wchg2; unsigned* wchg1;  // bitsets: values changed since the last wrong-saddle scan
  K* ext_key; int* ext_id;      // largest / smallest saddle selection scratch; ext_id then
                                // the lowest-row arbitration of get_wrong_index_min (kInf)

  int* ctr;  // device counters, see Ctr
  DeviceTables tb;
  const CUtensorMap* map_f;  // tile maps of f and g in device memory (when tma_f / tma_g)
  const CUtensorMap* map_g;
  int tma_f, tma_g;
  int iter_cap;  // device-side limit of pointer jumping and path walks
  int pass_chunk; // 1024-id blocks per saddle-pass work item (a tuning knob)
  int wn_lockstep; // wrong neighbours by the lockstep resolution (k_wn_step, the
                   // default), else in ascending saddle order (k_wn_vote / commit / resolve)
};

// Jobs served by one launch.  Every per-round kernel takes the device array of
// job descriptors and a selection: indices into that array and, for tile
// kernels, the exclusive prefix of the selected jobs' tile counts (a block's
// flat index picks its job by binary search).  A plain correction is a
// selection of one job.
constexpr int kMaxSel = 64;
struct Sel {
  int n;
  int idx[kMaxSel];
  int off[kMaxSel + 1];
};

// Indices into the device counter block.
enum Ctr : int {
  C_MM = 0, C_CMAX, C_CMIN, C_CSAD, C_TOUCHED, C_NFC, C_NFC1, C_CAND, C_CAND_NEXT,
  C_WMC, C_WMC2, C_WSC, C_WMIN, C_WMIN2, C_WSCJ, C_NS2, C_NS1, C_NMAX, C_NMIN,
  C_E2, C_E1,  // row entries of the 2-saddles' / 1-saddles' original rows (upper bound)
  C_ERROR,
  C_CHANGED,   // some value changed since the last manifold round began
  C_DIRTY, C_MM_NEXT, C_CANDJ,
  C_MFSKIP,    // this manifold round repeats the last one's inputs: kernels skip it
  C_MFDONE,    // a manifold round has run
  C_MFREUSED,  // manifold rounds skipped so far
  // Per-job epochs and stamps, advanced by k_ctl so that one launch can serve
  // jobs at different points of their correction.
  C_DEPOCH,    // dirty-list epoch (k_apply)
  C_REPOCH,    // re-evaluation epoch (k_redetect / k_keep)
  C_WNSTAMP,   // wrong-neighbour flag stamp, one per manifold round
  C_WNROUND,   // wrong-neighbour arbitration round (vote high word)
  C_WNSMALL,   // this side's candidate list is small: the block completion does it all
  C_MFFIRST,   // the manifold round being computed is the job's first: every input is new
  C_TLIST,     // tiles listed for this manifold round's steepest pointers (k_tile_list)
  C_WEP2, C_WEP1,  // wrong-saddle scan epochs (maxima, minima); epoch 1 computes every extremum
  C_AFF,       // extrema queued for the current wrong-saddle update
  C_WLONG,     // of those, the ones with long entry lists (wlong)
  C_COUNT
};
// Error bits in ctr[C_ERROR].
constexpr int kErrJump = 1, kErrPath = 2, kErrTile = 4, kErrResolve = 8;
// Ids per changed-input flag of the jump (the CP-list block size, kCpBlock).
constexpr int kCpBlockJ = 1024;

template <class T>
__device__ __forceinline__ T tabs(T v) { return v < T(0) ? -v : v; }

// ---------------------------------------------------------------------------
// Classification over a shared-memory halo tile.
//
// Replaces classifyVertex_CUDA (:3720-3911).  kDetect = false writes the
// original type and lower-star mask (type=0 call, :5289); kDetect = true is the
// fused mismatch detection of the type=1 call (:3856-3910), appending each
// mismatching vertex once with its categories (max, min, saddle) through
// warp ballots.
// ---------------------------------------------------------------------------
constexpr int TX = 32, TY = 8, TZ = 4;
// Tile kernels run 256 threads, one per (x, y) column of the tile.
static_assert(TX * TY == 256, "tile kernels map one thread to each (x, y) column of a tile");
// Shared tile rows start 4 elements left of the tile origin so that the TMA
// box origin x = bx - 4 is 16-byte aligned; the tile's x = 0 sits at kXOff.
constexpr int SX = TX + 8, SY = TY + 2, SZ = TZ + 2, kXOff = 4;

template <class T>
struct alignas(128) Tile {
  T v[SZ][SY][SX];
};

// Job and tile origin of a tile kernel's block.
template <class T>
__device__ __forceinline__ const Job<T>& tile_job(const Job<T>* __restrict__ jobs, const Sel& sel,
                                                  int& bx, int& by, int& bz, int* tile = nullptr) {
  const int t = blockIdx.x;
  int lo = 0, hi = sel.n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (sel.off[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  const Job<T>& J = jobs[sel.idx[lo]];
  const int lt = t - sel.off[lo];
  const int ntx = (J.dim.W + TX - 1) / TX, nty = (J.dim.H + TY - 1) / TY;
  bx = (lt % ntx) * TX;
  by = ((lt / ntx) % nty) * TY;
  bz = (lt / (ntx * nty)) * TZ;
  if (tile) *tile = lt;
  return J;
}

// Marks the tiles whose halo tile contains vertex (x, y, z): those holding
// one of its 26 neighbours or itself.
__device__ __forceinline__ void mark_tiles(uint8_t* tdirty, const Dims& g, int x, int y, int z) {
  const int ntx = (g.W + TX - 1) / TX, nty = (g.H + TY - 1) / TY;
  const int x0 = max(x - 1, 0) / TX, x1 = min(x + 1, g.W - 1) / TX;
  const int y0 = max(y - 1, 0) / TY, y1 = min(y + 1, g.H - 1) / TY;
  const int z0 = max(z - 1, 0) / TZ, z1 = min(z + 1, g.D - 1) / TZ;
  for (int c = z0; c <= z1; ++c)
    for (int b = y0; b <= y1; ++b)
      for (int a = x0; a <= x1; ++a) tdirty[(c * nty + b) * ntx + a] = 1;
}

// Halo tile: TMA box (one bulk tensor copy, zero fill outside the grid) when
// the field's row stride allows it, else plain loads with every thread's loads
// issued before its first shared store.  Outside-grid entries are never read.
// A block that loads several tiles initialises the barrier once (init) and
// waits on alternating phases (parity = loads issued before this one, mod 2).
template <class T>
__device__ __forceinline__ bool load_tile(Tile<T>& s, uint64_t* bar, const CUtensorMap* map,
                                          bool tma, const T* __restrict__ a, const Dims& g, int bx,
                                          int by, int bz, unsigned parity = 0, bool init = true) {
  if (tma) {
    if (threadIdx.x == 0) {
      if (init) mbar_init(bar, 1);
      mbar_expect_tx(bar, (unsigned)sizeof(Tile<T>));
      tma_load_3d(&s.v[0][0][0], map, bx - kXOff, by - 1, bz - 1, bar);
    }
    __syncthreads();
    return mbar_wait(bar, parity, 1ll << 26);
  }
  constexpr int HX = TX + 2;
  constexpr int kTotal = HX * SY * SZ;
  constexpr int kPer = (kTotal + 255) / 256;
  T v[kPer];
  int off[kPer];
#pragma unroll
  for (int k = 0; k < kPer; ++k) {
    const int i = threadIdx.x + k * 256;
    const int lx = i % HX, t = i / HX, ly = t % SY, lz = t / SY;
    const int gx = bx + lx - 1, gy = by + ly - 1, gz = bz + lz - 1;
    const bool ok = i < kTotal && gx >= 0 && gx < g.W && gy >= 0 && gy < g.H && gz >= 0 && gz < g.D;
    off[k] = ok ? (lz * SY + ly) * SX + lx + kXOff - 1 : -1;
    v[k] = ok ? __ldg(a + gx + (long long)gy * g.W + (long long)gz * g.W * g.H) : T(0);
  }
#pragma unroll
  for (int k = 0; k < kPer; ++k)
    if (off[k] >= 0) (&s.v[0][0][0])[off[k]] = v[k];
  __syncthreads();
  return true;
}

// Lower-star direction mask and upper mask of the tile voxel at tile
// coordinates (tx, ty, tz).  A tie goes to the lower side exactly when the
// neighbour's id is smaller, i.e. for odd directions.
template <class T>
__device__ __forceinline__ void tile_masks(const Tile<T>& s, int tx, int ty, int tz, int valid,
                                           int& lm, int& um) {
  const T c = s.v[tz + 1][ty + 1][tx + kXOff];
  lm = 0;
#pragma unroll
  for (int d = 0; d < kNumDirs; ++d) {
    const T nv = s.v[tz + 1 + dir_z(d)][ty + 1 + dir_y(d)][tx + kXOff + dir_x(d)];
    const bool lower = dir_neighbour_is_before(d) ? (nv <= c) : (nv < c);
    lm |= (int)lower << d;
  }
  // Values and ids order the vertices totally: a valid neighbour is upper
  // exactly when it is not lower.
  lm &= valid;
  um = valid & ~lm;
}

// Vertex type from the masks (classifyVertex_CUDA :3835-3853): maximum when no
// upper neighbour, minimum when no lower one, else the LUT entry of the
// boundary configuration, or -1 for a configuration the LUT has no key for.
__device__ __forceinline__ int type_from_masks(int lm, int um, int valid, int bc,
                                               const DeviceTables& tb) {
  if (um == 0) return 4;
  if (lm == 0) return 0;
  const int off = tb.key_offset[bc];
  if (off < 0) return -1;
  int idx = um;
  if (bc != 0) {  // index bits follow the valid neighbours' order
    idx = 0;
    int k = 0;
#pragma unroll
    for (int d = 0; d < kNumDirs; ++d) {
      if (valid >> d & 1) {
        idx |= (um >> d & 1) << k;
        ++k;
      }
    }
  }
  return __ldg(tb.lut + off + idx);
}

__device__ __forceinline__ int mismatch_cats(int t, int o, int lm, int olm) {
  int cat = 0;
  if (t != o) {
    if ((t == 4) != (o == 4)) cat |= kCatMax;
    if ((t == 0) != (o == 0)) cat |= kCatMin;
    if ((t == 2) != (o == 2) || (t == 1) != (o == 1) || (t == 3) != (o == 3)) cat |= kCatSaddle;
  } else if ((t == 1 || t == 2 || t == 3) && lm != olm) {
    cat |= kCatSaddle;  // areVectorsDifferent_local (:909-921) on direction masks
  }
  return cat;
}

// Per-category counts of mismatching vertices, one atomic per warp and category.
__device__ __forceinline__ void count_cats(int* ctr, int cat) {
  const unsigned bm = __ballot_sync(0xffffffffu, cat & kCatMax);
  const unsigned bn = __ballot_sync(0xffffffffu, cat & kCatMin);
  const unsigned bs = __ballot_sync(0xffffffffu, cat & kCatSaddle);
  if (lane_id() == 0) {
    if (bm) atomicAdd(ctr + C_CMAX, __popc(bm));
    if (bn) atomicAdd(ctr + C_CMIN, __popc(bn));
    if (bs) atomicAdd(ctr + C_CSAD, __popc(bs));
  }
}

// kDetect = false classifies f (setup), true classifies g (detection).
template <class T, bool kDetect>
__global__ void __launch_bounds__(256) k_classify(const Job<T>* __restrict__ jobs,
                                                  const __grid_constant__ Sel sel) {
  __shared__ Tile<T> s;
  __shared__ uint64_t bar;
  int bx, by, bz;
  const Job<T>& J = tile_job(jobs, sel, bx, by, bz);
  const Dims g = J.dim;
  const T* a = kDetect ? J.g : J.f;
  // The block decides together: its threads meet at barriers further on.
  if (!__syncthreads_and(load_tile<T>(s, &bar, kDetect ? J.map_g : J.map_f,
                                      kDetect ? J.tma_g : J.tma_f, a, g, bx, by, bz))) {
    if (threadIdx.x == 0) atomicOr(J.ctr + C_ERROR, kErrTile);
    return;
  }
  // Detection: the tile's mismatching vertices are gathered in shared memory
  // and appended with one global atomic per block (per warp, the appends of a
  // dense pass all queue on the same counter).
  __shared__ int s_list[kDetect ? TZ * TY * TX : 1];
  __shared__ int s_n, s_base, s_cat[3];
  if (kDetect && threadIdx.x == 0) {
    s_n = 0;
    s_cat[0] = s_cat[1] = s_cat[2] = 0;
  }
  if (kDetect) __syncthreads();
  const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
  // A tile off the field's faces has every direction valid at every voxel.
  const bool interior = bx > 0 && by > 0 && bz > 0 && bx + TX < g.W && by + TY < g.H &&
                        bz + TZ < g.D;
  for (int tz = 0; tz < TZ; ++tz) {
    const int x = bx + tx, y = by + ty, z = bz + tz;
    const bool in = x < g.W && y < g.H && z < g.D;
    if (in) {
      const int v = x + y * g.W + z * g.W * g.H;
      const int bc = interior ? 0 : boundary_code(x, y, z, g.W, g.H, g.D);
      const int valid = interior ? (1 << kNumDirs) - 1 : valid_mask(bc);
      int lm, um;
      tile_masks(s, tx, ty, tz, valid, lm, um);
      const int t = type_from_masks(lm, um, valid, bc, J.tb);
      if (!kDetect) {
        J.otype[v] = (int8_t)t;
        J.olm[v] = (uint16_t)lm;
      } else {
        const int cat = mismatch_cats(t, J.otype[v], lm, J.olm[v]);
        J.mstat[v] = (uint8_t)cat;
        if (cat) {
          s_list[atomicAdd(&s_n, 1)] = v | (cat << kCatShift);
          if (cat & kCatMax) atomicAdd(&s_cat[0], 1);
          if (cat & kCatMin) atomicAdd(&s_cat[1], 1);
          if (cat & kCatSaddle) atomicAdd(&s_cat[2], 1);
        }
      }
    }
  }
  if (kDetect) {
    __syncthreads();
    if (threadIdx.x == 0 && s_n) {
      s_base = atomicAdd(J.ctr + C_MM, s_n);
      if (s_cat[0]) atomicAdd(J.ctr + C_CMAX, s_cat[0]);
      if (s_cat[1]) atomicAdd(J.ctr + C_CMIN, s_cat[1]);
      if (s_cat[2]) atomicAdd(J.ctr + C_CSAD, s_cat[2]);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < s_n; k += blockDim.x) J.mm[s_base + k] = s_list[k];
  }
}

// ---------------------------------------------------------------------------
// Incremental mismatch detection.
//
// The type of v depends only on the values of v and its 14 neighbours, so after
// the first dense detection only the closed neighbourhoods of vertices whose
// value changed can change status.  k_redetect re-evaluates them (once each,
// by stamp) and appends the mismatching ones to the next list; k_keep carries
// over the entries of the previous list that were not re-evaluated.  The
// resulting set equals a dense re-detection (the lists are unordered; every
// consumer merges by atomic max).
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ int global_type(const Job<T>& J, int v, int& lmask) {
  const Dims g = J.dim;
  int x, y, z;
  coords(v, g, x, y, z);
  const int bc = boundary_code(x, y, z, g.W, g.H, g.D);
  const T c = J.g[v];
  int lm = 0, up = 0, k = 0, nl = 0, nu = 0;
#pragma unroll
  for (int d = 0; d < kNumDirs; ++d) {
    if (!dir_valid(d, bc)) continue;
    const T nv = J.g[v + dir_x(d) + dir_y(d) * g.W + dir_z(d) * g.W * g.H];
    const bool before = dir_neighbour_is_before(d);
    if (nv < c || (nv == c && before)) {
      lm |= 1 << d;
      ++nl;
    } else if (nv > c || (nv == c && !before)) {
      up |= 1 << k;
      ++nu;
    }
    ++k;
  }
  lmask = lm;
  if (nu == 0) return 4;
  if (nl == 0) return 0;
  const int off = J.tb.key_offset[bc];
  if (off < 0) return -1;
  return __ldg(J.tb.lut + off + up);
}

template <class T>
__global__ void __launch_bounds__(256) k_redetect(const Job<T>* __restrict__ jobs,
                                                  const __grid_constant__ Sel sel) {
  for (int jk = 0; jk < sel.n; ++jk) {
  const Job<T>& J = jobs[sel.idx[jk]];
  const int n = J.ctr[C_DIRTY];
  const int epoch = J.ctr[C_REPOCH];
  const long long total = (long long)n * (kNumDirs + 1);
  const long long stride = (long long)gridDim.x * blockDim.x;
  const Dims g = J.dim;
  for (long long base = blockIdx.x * (long long)blockDim.x; base < total; base += stride) {
    const long long e = base + threadIdx.x;
    int cat = 0, v = -1;
    if (e < total) {
      const int c = J.dirty[e / (kNumDirs + 1)];
      const int d = (int)(e % (kNumDirs + 1)) - 1;  // -1: the vertex itself
      v = c;
      if (d >= 0) {
        int x, y, z;
        coords(c, g, x, y, z);
        v = dir_valid(d, boundary_code(x, y, z, g.W, g.H, g.D))
                ? c + dir_x(d) + dir_y(d) * g.W + dir_z(d) * g.W * g.H
                : -1;
      }
      if (v >= 0 && atomicExch(J.rstamp + v, epoch) != epoch) {
        int lm;
        const int t = global_type(J, v, lm);
        cat = mismatch_cats(t, J.otype[v], lm, J.olm[v]);
        J.mstat[v] = (uint8_t)cat;
      }
    }
    const int slot = warp_append(J.ctr + C_MM_NEXT, cat != 0, 0xffffffffu);
    if (slot >= 0) J.mm_next[slot] = v | (cat << kCatShift);
    count_cats(J.ctr, cat);
  }
  }
}

template <class T>
__global__ void __launch_bounds__(256) k_keep(const Job<T>* __restrict__ jobs,
                                              const __grid_constant__ Sel sel) {
  for (int jk = 0; jk < sel.n; ++jk) {
  const Job<T>& J = jobs[sel.idx[jk]];
  const int n = J.ctr[C_MM];
  const int epoch = J.ctr[C_REPOCH];
  const int stride = gridDim.x * blockDim.x;
  for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {
    const int e = base + threadIdx.x;
    int ent = 0, cat = 0;
    if (e < n) {
      ent = J.mm[e];
      const int v = ent & ((1 << kCatShift) - 1);
      if (J.rstamp[v] != epoch) cat = (unsigned)ent >> kCatShift;
    }
    const int slot = warp_append(J.ctr + C_MM_NEXT, cat != 0, 0xffffffffu);
    if (slot >= 0) J.mm_next[slot] = ent;
    count_cats(J.ctr, cat);
  }
  }
}

// ---------------------------------------------------------------------------
// Steepest directions with tile-local path compression.
//
// Replaces ComputeDirection (:1464-1512) and the first steps of the pointer
// jumping (:1514-1611): each voxel's steepest-ascent (descent) pointer is
// followed inside the tile in shared memory until it leaves the tile or stops
// at a root, so the global jump that follows moves a tile per hop.
// Output: ds/as (original field) or pdd/pda (decompressed field) = first
// vertex outside the tile on the path, or the root.  On the decompressed field
// only tiles marked dirty (a value in the tile or its halo changed) are
// recomputed; the others keep their pointers, which depend on nothing else.
// ---------------------------------------------------------------------------
// Direction components packed two bits per direction (component + 1), so a
// runtime direction index decodes with a shift and a mask.
__host__ __device__ constexpr unsigned pack_dir(int axis) {
  unsigned p = 0;
  for (int d = 0; d < kNumDirs; ++d)
    p |= (unsigned)((axis == 0 ? dir_x(d) : axis == 1 ? dir_y(d) : dir_z(d)) + 1) << (2 * d);
  return p;
}
__device__ __forceinline__ int ddx(int d) { return (int)((pack_dir(0) >> (2 * d)) & 3u) - 1; }
__device__ __forceinline__ int ddy(int d) { return (int)((pack_dir(1) >> (2 * d)) & 3u) - 1; }
__device__ __forceinline__ int ddz(int d) { return (int)((pack_dir(2) >> (2 * d)) & 3u) - 1; }

// Steepest-ascent and steepest-descent directions of one tile voxel: the
// maximum (minimum) of (value, id) over the voxel and its valid neighbours.
// Ids are scanned in ascending order so that ">=" keeps the larger id on a tie;
// the descent scans in descending order with "<=".  (Finite inputs: the scans
// start from -inf / +inf and always meet the centre.)  kAll: every direction
// valid, no per-direction test.
template <class T, bool kAll>
__device__ __forceinline__ void steepest_dirs(const Tile<T>& s, int tx, int ty, int tz, int valid,
                                              int& hd, int& ld) {
  const T c = s.v[tz + 1][ty + 1][tx + kXOff];
  T hv = -T(INFINITY), lv = T(INFINITY);
  hd = -1;
  ld = -1;
  T nv[kNumDirs];
#pragma unroll
  for (int d = 0; d < kNumDirs; ++d)
    nv[d] = s.v[tz + 1 + dir_z(d)][ty + 1 + dir_y(d)][tx + kXOff + dir_x(d)];
#pragma unroll
  for (int j = 0; j < kNumDirs; ++j) {
    const int d = rank_dir(j);
    if (j == kRankCentre && c >= hv) { hv = c; hd = -1; }
    if ((kAll || (valid >> d & 1)) && nv[d] >= hv) { hv = nv[d]; hd = d; }
  }
#pragma unroll
  for (int j = kNumDirs - 1; j >= 0; --j) {
    const int d = rank_dir(j);
    if ((kAll || (valid >> d & 1)) && nv[d] <= lv) { lv = nv[d]; ld = d; }
    if (j == kRankCentre && c <= lv) { lv = c; ld = -1; }
  }
}

// Next-step codes of the in-tile path following (besides local indices).
constexpr int kExit = -1, kRoot = -2;

// Follows next-pointers inside the tile from local voxel li to the path's
// exit (global id of the first outside vertex) or root.
__device__ __forceinline__ int follow(const int16_t* nxt, const int* exit_gid, int li, int bx,
                                      int by, int bz, int W, int WH, int* err) {
  int cur = li, t = nxt[li];
  for (int step = 0; t >= 0; ++step) {
    cur = t;
    t = nxt[cur];
    if (step > TX * TY * TZ) {  // a path never revisits a voxel; guard anyway
      atomicOr(err, kErrTile);
      break;
    }
  }
  if (t == kExit) return exit_gid[cur];
  const int cx = cur % TX, cy = (cur / TX) % TY, cz = cur / (TX * TY);
  return (bx + cx) + (by + cy) * W + (bz + cz) * WH;
}

// Steepest pointers of one tile, compressed to the tile's exits: every voxel's
// pointer is the first vertex outside the tile on its steepest path, or the
// path's root inside the tile.  kDec = false: f into ds / as (setup), with the
// original classification (otype, olm) from the same tile load; true: g into
// pdd / pda.  Returns false when the tile's load did not complete.
template <class T, bool kDec>
__device__ __noinline__ bool direction_tile(const Job<T>& J, Tile<T>& s, uint64_t* bar,
                                               int16_t* hnext, int16_t* lnext, int* hexit,
                                               int* lexit, int bx, int by, int bz,
                                               unsigned parity, bool init) {
  const Dims g = J.dim;
  const int WH = g.W * g.H;
  const T* a = kDec ? J.g : J.f;
  int* ds = kDec ? J.pdd : J.ds;
  int* as = kDec ? J.pda : J.as;
  // The block decides together: its threads meet at a barrier further on.
  if (!__syncthreads_and(load_tile<T>(s, bar, kDec ? J.map_g : J.map_f, kDec ? J.tma_g : J.tma_f,
                                      a, g, bx, by, bz, parity, init))) {
    if (threadIdx.x == 0) atomicOr(J.ctr + C_ERROR, kErrTile);
    return false;
  }
  const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
  // A tile off the field's faces has every direction valid at every voxel.
  const bool interior = bx > 0 && by > 0 && bz > 0 && bx + TX < g.W && by + TY < g.H &&
                        bz + TZ < g.D;
  for (int tz = 0; tz < TZ; ++tz) {
    const int li = (tz * TY + ty) * TX + tx;
    const int x = bx + tx, y = by + ty, z = bz + tz;
    int hd = -1, ld = -1;
    const bool in = x < g.W && y < g.H && z < g.D;
    if (interior) {
      steepest_dirs<T, true>(s, tx, ty, tz, (1 << kNumDirs) - 1, hd, ld);
    } else if (in) {
      const int bc = boundary_code(x, y, z, g.W, g.H, g.D);
      if (bc == 0) steepest_dirs<T, true>(s, tx, ty, tz, (1 << kNumDirs) - 1, hd, ld);
      else steepest_dirs<T, false>(s, tx, ty, tz, valid_mask(bc), hd, ld);
    }
    const int v = x + y * g.W + z * WH;
    if (!kDec && in) {
      // The original field's classification from the same tile
      // (classifyVertex_CUDA, the type = 0 call :5289): type and lower-star
      // direction mask.
      const int bc = interior ? 0 : boundary_code(x, y, z, g.W, g.H, g.D);
      const int valid = interior ? (1 << kNumDirs) - 1 : valid_mask(bc);
      int lm, um;
      tile_masks(s, tx, ty, tz, valid, lm, um);
      J.otype[v] = (int8_t)type_from_masks(lm, um, valid, bc, J.tb);
      J.olm[v] = (uint16_t)lm;
    }
    // Next step in tile terms: the local index when it stays in the tile,
    // kExit (the first outside vertex to the exit slot) when it leaves it,
    // kRoot at a root.
    auto step = [&](int d, int* exit_gid) {
      if (d < 0) return kRoot;
      const int dx = ddx(d), dy = ddy(d), dz = ddz(d);
      const int nx = tx + dx, ny = ty + dy, nz = tz + dz;
      if ((unsigned)nx < (unsigned)TX && (unsigned)ny < (unsigned)TY && (unsigned)nz < (unsigned)TZ)
        return (nz * TY + ny) * TX + nx;
      *exit_gid = v + dx + dy * g.W + dz * WH;
      return kExit;
    };
    hnext[li] = (int16_t)(in ? step(hd, &hexit[li]) : kRoot);
    lnext[li] = (int16_t)(in ? step(ld, &lexit[li]) : kRoot);
  }
  __syncthreads();
  for (int tz = 0; tz < TZ; ++tz) {
    const int x = bx + tx, y = by + ty, z = bz + tz;
    if (!(x < g.W && y < g.H && z < g.D)) continue;
    const int li = (tz * TY + ty) * TX + tx;
    const int v = x + y * g.W + z * WH;
    ds[v] = follow(hnext, hexit, li, bx, by, bz, g.W, WH, J.ctr + C_ERROR);
    as[v] = follow(lnext, lexit, li, bx, by, bz, g.W, WH, J.ctr + C_ERROR);
  }
  return true;
}

// Setup: every tile of the original field, one block per tile.
template <class T, bool kDec>
__global__ void __launch_bounds__(256, sizeof(T) == 8 ? 4 : 6) k_direction(const Job<T>* __restrict__ jobs,
                                                   const __grid_constant__ Sel sel) {
  __shared__ Tile<T> s;
  __shared__ uint64_t bar;
  __shared__ int16_t hnext[TZ * TY * TX], lnext[TZ * TY * TX];
  __shared__ int hexit[TZ * TY * TX], lexit[TZ * TY * TX];
  int bx, by, bz, tile;
  const Job<T>& J = tile_job(jobs, sel, bx, by, bz, &tile);
  if (kDec && J.ctr[C_MFSKIP]) return;  // same inputs as the last manifold round
  if (kDec && !J.tdirty[tile]) return;  // tile and halo unchanged: pointers stand
  if (!direction_tile<T, kDec>(J, s, &bar, hnext, lnext, hexit, lexit, bx, by, bz, 0, true))
    return;
  if (kDec && threadIdx.x == 0) J.tdirty[tile] = 0;
}

// The tiles of each selected job whose tile or halo changed since their
// pointers were computed (every tile in a job's first round), into the
// job's tile list (cand_next, free at this point of a manifold round;
// count C_TLIST, zeroed when the round begins).
template <class T>
__global__ void __launch_bounds__(256) k_tile_list(const Job<T>* __restrict__ jobs,
                                                   const __grid_constant__ Sel sel) {
  for (int jk = 0; jk < sel.n; ++jk) {
    const Job<T>& J = jobs[sel.idx[jk]];
    if (J.ctr[C_MFSKIP]) continue;
    const int nt = ((J.dim.W + TX - 1) / TX) * ((J.dim.H + TY - 1) / TY) *
                   ((J.dim.D + TZ - 1) / TZ);
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x; base < nt; base += stride) {  // uniform per warp
      const int t = base + threadIdx.x;
      const bool dirty = t < nt && J.tdirty[t];
      const int slot = warp_append(J.ctr + C_TLIST, dirty, 0xffffffffu);
      if (slot >= 0) J.cand_next[slot] = t;
    }
  }
}

// A manifold round's steepest pointers of the decompressed field: a fixed
// grid whose blocks take the listed tiles of every selected job in turn, so
// that a round with few changed tiles launches few blocks' worth of work
// instead of one block per tile of the field.  It also marks, per side, the
// current labels of every vertex of a listed tile as touched roots (rtouch2,
// rtouch1): only vertices with a touched label can change label this round
// (k_jump2).
template <class T>
__global__ void __launch_bounds__(256, 4) k_direction_list(const Job<T>* __restrict__ jobs,
                                                        const __grid_constant__ Sel sel) {
  __shared__ Tile<T> s;
  __shared__ uint64_t bar;
  __shared__ int16_t hnext[TZ * TY * TX], lnext[TZ * TY * TX];
  __shared__ int hexit[TZ * TY * TX], lexit[TZ * TY * TX];
  unsigned loads = 0;  // TMA loads issued by this block: the barrier's phase
  for (int jk = 0; jk < sel.n; ++jk) {
    const Job<T>& J = jobs[sel.idx[jk]];
    if (J.ctr[C_MFSKIP]) continue;
    const int n = J.ctr[C_TLIST];
    const int ntx = (J.dim.W + TX - 1) / TX, nty = (J.dim.H + TY - 1) / TY;
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
      const int t = J.cand_next[k];
      const int bx = (t % ntx) * TX, by = ((t / ntx) % nty) * TY, bz = (t / (ntx * nty)) * TZ;
      __syncthreads();  // every thread is done with the shared tile of the last one
      const bool tma = J.tma_g != 0;
      if (!direction_tile<T, true>(J, s, &bar, hnext, lnext, hexit, lexit, bx, by, bz,
                                   loads & 1u, loads == 0))
        return;
      loads += tma;
      if (threadIdx.x == 0) J.tdirty[t] = 0;
      const int x = bx + (int)threadIdx.x % TX, y = by + (int)threadIdx.x / TX;
      if (x < J.dim.W && y < J.dim.H) {
        for (int tz = 0; tz < TZ && bz + tz < J.dim.D; ++tz) {
          const int v = x + y * J.dim.W + (bz + tz) * J.dim.W * J.dim.H;
          const int r2 = J.dds[v], r1 = J.das[v];
          // Read first: most roots are marked by many vertices.
          if (!(J.rtouch2[r2 >> 5] >> (r2 & 31) & 1u)) atomicOr(J.rtouch2 + (r2 >> 5), 1u << (r2 & 31));
          if (!(J.rtouch1[r1 >> 5] >> (r1 & 31) & 1u)) atomicOr(J.rtouch1 + (r1 >> 5), 1u << (r1 & 31));
        }
      }
    }
  }
}

// Global pointer jumping of both label arrays (ComputeDescendingManifold /
// ComputeAscendingManifold, :1514-1611), the two chains interleaved for
// memory-level parallelism.  Labels always point further along the path, so
// concurrent readers of a label being finalised see either value correctly.
// Every vertex is resolved (the reference resolves descending labels only next
// to original 2-saddles, the only places they are read).  Iterations are
// capped; hitting the cap sets the error word instead of spinning.  On the
// decompressed field it also writes each vertex's label-mismatch bits
// and changed-input bytes for the saddle pass.  kLater (decompressed field,
// a job's rounds after its first): the label-mismatch bits of a group change
// only with its labels, so the original roots are loaded only for groups
// whose labels changed, after the chase.
template <class T, bool kDec, bool kLater = false>
__global__ void __launch_bounds__(256, 4) k_jump2(const Job<T>* __restrict__ jobs,
                                               const __grid_constant__ Sel sel) {
  for (int jk = 0; jk < sel.n; ++jk) {
  const Job<T>& J = jobs[sel.idx[jk]];
  if (kDec && J.ctr[C_MFSKIP]) continue;
  // Original field: in place on ds / as.  Decompressed field: from the
  // tile-compressed pointers pdd / pda (kept for the next round) into dds / das.
  const int* a = kDec ? J.pdd : J.ds;
  const int* b = kDec ? J.pda : J.as;
  int* ra = kDec ? J.dds : J.ds;
  int* rb = kDec ? J.das : J.as;
  // Descriptor fields in registers: stores below could alias the descriptor.
  const unsigned* __restrict__ vchg = J.vchg;
  const int* __restrict__ ods = J.ds;
  const int* __restrict__ oas = J.as;
  uint8_t* __restrict__ dirtyv = J.dirtyv;
  uint8_t* __restrict__ mis = J.mis;
  int* err = J.ctr + C_ERROR;
  const int N = J.dim.N;
  const int cap_j = J.iter_cap;
  auto jump_one = [&](int v) {
    int u1 = a[v], u2 = b[v];
    // Decompressed field: this vertex's old labels, original roots and
    // change stamp, loaded while the chains are followed.
    int o1 = 0, o2 = 0, r1 = 0, r2 = 0;
    unsigned c0 = 0;
    if constexpr (kDec) {
      o1 = ra[v];
      o2 = rb[v];
      r1 = ods[v];
      r2 = oas[v];
      c0 = vchg[v >> 5] >> (v & 31);
    }
    bool d1 = false, d2 = false;
    int it = 0;
    for (; it < cap_j && !(d1 && d2); ++it) {
      if (!d1) {
        const int w = a[u1];
        if (w == u1) d1 = true;
        else u1 = w;
      }
      if (!d2) {
        const int w = b[u2];
        if (w == u2) d2 = true;
        else u2 = w;
      }
    }
    if (it == cap_j) atomicOr(err, kErrJump);
    if constexpr (kDec) {
      // For the saddle pass: label-mismatch bits, and whether an input of the
      // rows this vertex feeds changed since the previous computed round (its
      // value, either label, or the value of either label's root).  The
      // change bitset starts full, so the first round marks every vertex.
      const unsigned c1 = vchg[u1 >> 5] >> (u1 & 31), c2 = vchg[u2 >> 5] >> (u2 & 31);
      dirtyv[v] = ((o1 != u1) | (o2 != u2) | ((c0 | c1 | c2) & 1u)) ? (uint8_t)J.ctr[C_WNSTAMP]
                                                                    : (uint8_t)0;
      mis[v] = (uint8_t)((u1 != r1) | (u2 != r2) << 1);
    }
    ra[v] = u1;
    rb[v] = u2;
  };
  if constexpr (kDec) {
    if ((N & 3) == 0) {
      // Four consecutive vertices per thread: one 16-byte load per array and
      // one 4-byte store per byte array, a quarter of the memory requests of
      // the vertex-per-thread loop, with eight chains interleaved.  A quad
      // with a changed-input byte stamps its 1024-id block (bdirty, read by
      // the saddle pass; its address is read where it is used: kept in a
      // register for the whole loop it costs spills).  Changed-input bytes
      // are round stamps (low byte): a quad that is not followed leaves its
      // bytes, which then read as unchanged.
      //
      // kLater: a vertex's label on a side can change only when its path
      // crosses a tile whose pointers this round recomputed, and every vertex
      // of a path carries the path's label.  So a quad none of whose old
      // labels is a root marked by k_direction_list (rtouch2 / rtouch1: the
      // old labels of the recomputed tiles' vertices) keeps its labels and
      // mismatch bits and has no changed input (a changed value, own or of a
      // root, lies in a recomputed tile too).
      const int stamp = J.ctr[C_WNSTAMP];
      const unsigned st8 = (unsigned)stamp & 0xffu;
      // Returns the quad's labels through u1 / u2 (the old ones when it is
      // not followed) and the old ones through o1 / o2 (-1 in a first round).
      auto quad = [&](int v0, int* u1, int* u2, int* o1, int* o2) {
        // A job's first round writes every label (its change bitset starts
        // full, and the stored labels may be another job's): no old labels.
        const int4 O1 = kLater ? *reinterpret_cast<const int4*>(ra + v0) : make_int4(-1, -1, -1, -1);
        const int4 O2 = kLater ? *reinterpret_cast<const int4*>(rb + v0) : make_int4(-1, -1, -1, -1);
        o1[0] = O1.x; o1[1] = O1.y; o1[2] = O1.z; o1[3] = O1.w;
        o2[0] = O2.x; o2[1] = O2.y; o2[2] = O2.z; o2[3] = O2.w;
        if constexpr (kLater) {
          unsigned hit = 0u;
#pragma unroll
          for (int k = 0; k < 4; ++k)
            hit |= (J.rtouch2[o1[k] >> 5] >> (o1[k] & 31)) | (J.rtouch1[o2[k] >> 5] >> (o2[k] & 31));
          if (!(hit & 1u)) {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              u1[k] = o1[k];
              u2[k] = o2[k];
            }
            return;
          }
        }
        const int4 A = *reinterpret_cast<const int4*>(a + v0);
        const int4 B = *reinterpret_cast<const int4*>(b + v0);
        int4 R1 = make_int4(0, 0, 0, 0), R2 = make_int4(0, 0, 0, 0);
        if constexpr (!kLater) {
          R1 = *reinterpret_cast<const int4*>(ods + v0);
          R2 = *reinterpret_cast<const int4*>(oas + v0);
        }
        const unsigned cw = vchg[v0 >> 5] >> (v0 & 31);
        u1[0] = A.x; u1[1] = A.y; u1[2] = A.z; u1[3] = A.w;
        u2[0] = B.x; u2[1] = B.y; u2[2] = B.z; u2[3] = B.w;
        // One hop of every unfinished chain per iteration: the eight loads
        // depend only on their own chain, so they are all in flight at once.
        bool more = true;
        int it = 0;
        for (; it < cap_j && more; ++it) {
          int w1[4], w2[4];
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            w1[k] = a[u1[k]];
            w2[k] = b[u2[k]];
          }
          more = false;
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            more |= (w1[k] != u1[k]) | (w2[k] != u2[k]);
            u1[k] = w1[k];
            u2[k] = w2[k];
          }
        }
        if (it == cap_j && more) atomicOr(err, kErrJump);
        unsigned dv = 0;
        bool n1 = false, n2 = false;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const unsigned c1 = vchg[u1[k] >> 5] >> (u1[k] & 31);
          const unsigned c2 = vchg[u2[k] >> 5] >> (u2[k] & 31);
          n1 |= o1[k] != u1[k];
          n2 |= o2[k] != u2[k];
          const unsigned d = (o1[k] != u1[k]) | (o2[k] != u2[k]) | ((cw >> k | c1 | c2) & 1u);
          dv |= (d ? st8 : 0u) << (8 * k);
        }
        *reinterpret_cast<unsigned*>(dirtyv + v0) = dv;
        // Stores that would rewrite the stored value are skipped.  The
        // mismatch bits follow the labels alone (the original roots are
        // fixed), so a group whose labels did not change keeps last round's
        // bits.
        if (kLater ? (n1 || n2) : true) {
          if constexpr (kLater) {
            R1 = *reinterpret_cast<const int4*>(ods + v0);
            R2 = *reinterpret_cast<const int4*>(oas + v0);
          }
          const int r1[4] = {R1.x, R1.y, R1.z, R1.w}, r2[4] = {R2.x, R2.y, R2.z, R2.w};
          unsigned mv = 0;
#pragma unroll
          for (int k = 0; k < 4; ++k)
            mv |= ((unsigned)(u1[k] != r1[k]) | (unsigned)(u2[k] != r2[k]) << 1) << (8 * k);
          *reinterpret_cast<unsigned*>(mis + v0) = mv;
        }
        if (n1) *reinterpret_cast<int4*>(ra + v0) = make_int4(u1[0], u1[1], u1[2], u1[3]);
        if (n2) *reinterpret_cast<int4*>(rb + v0) = make_int4(u2[0], u2[1], u2[2], u2[3]);
        if (dv) J.bdirty[v0 >> 10] = stamp;
      };
      const int nq = N >> 2;
      const int qstride = gridDim.x * blockDim.x;
      for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += qstride) {
        int u1[4], u2[4], o1[4], o2[4];
        quad(q << 2, u1, u2, o1, o2);
      }
      continue;
    }
  }
  const int stride = gridDim.x * blockDim.x;
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < N; v += stride) jump_one(v);
  }
}

// ---------------------------------------------------------------------------
// Ordered compaction of the critical-point lists (ExtractCP :1694-1741, here in
// ascending vertex id).  Pass 1 counts per 1024-vertex block, pass 2 scans the
// block counts, pass 3 writes.
// ---------------------------------------------------------------------------
constexpr int kCpBlock = 1024;
static_assert(kCpBlockJ == kCpBlock, "the jump's flags cover the CP-list blocks");

__device__ __forceinline__ int cp_bits(int t) {
  return ((t == 2 || t == 3) ? 1 : 0) | ((t == 1 || t == 3) ? 2 : 0) | (t == 4 ? 4 : 0) |
         (t == 0 ? 8 : 0);
}

// One warp per 1024-id block, each lane 32 consecutive ids: the types come in
// as two 16-byte loads per lane (one coalesced kilobyte per warp), where one
// 1024-thread block per 1024 ids spent its time scheduling blocks.
constexpr int kCpWarps = 8;  // warps (1024-id blocks) per CTA

// The CP-list membership bits of the lane's 32 ids, one word per list.
__device__ __forceinline__ void cp_lane_bits(const int8_t* __restrict__ otype, int N, int v0,
                                             unsigned bits[4]) {
  int8_t t[32];
  if (v0 + 32 <= N) {
    const int4 q0 = *reinterpret_cast<const int4*>(otype + v0);
    const int4 q1 = *reinterpret_cast<const int4*>(otype + v0 + 16);
    const int w[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
#pragma unroll
    for (int k = 0; k < 32; ++k) t[k] = (int8_t)(w[k >> 2] >> (8 * (k & 3)));
  } else {
#pragma unroll
    for (int k = 0; k < 32; ++k) t[k] = v0 + k < N ? otype[v0 + k] : (int8_t)-1;
  }
#pragma unroll
  for (int l = 0; l < 4; ++l) bits[l] = 0u;
#pragma unroll
  for (int k = 0; k < 32; ++k) {
    const int b = cp_bits(t[k]);
#pragma unroll
    for (int l = 0; l < 4; ++l) bits[l] |= (unsigned)((b >> l) & 1) << k;
  }
}

// Also counts the entries the original rows will hold (lists 4 and 5): a
// 2-saddle's row has one entry per upper neighbour, a 1-saddle's one per lower
// neighbour (rows keep repeated labels; the persistence filter thr can only
// drop entries, so with thr > 0 this is an upper bound).
__global__ void __launch_bounds__(32 * kCpWarps) k_cp_count(const int8_t* __restrict__ otype,
                                                           const uint16_t* __restrict__ olm,
                                                           Dims g, int nb,
                                                           int* __restrict__ bcount) {
  const int b = blockIdx.x * kCpWarps + (int)(threadIdx.x >> 5);
  if (b >= nb) return;  // whole warps leave together
  const int v0 = b * kCpBlock + (int)lane_id() * 32;
  unsigned bits[4];
  cp_lane_bits(otype, g.N, v0, bits);
  int e2 = 0, e1 = 0;
  if ((bits[0] | bits[1]) != 0u) {
    int x, y, z;
    coords(v0, g, x, y, z);
    for (int k = 0; k < 32; ++k) {
      if (((bits[0] | bits[1]) >> k) & 1u) {
        const int nvalid = __popc(valid_mask(boundary_code(x, y, z, g.W, g.H, g.D)));
        const int lower = __popc((unsigned)olm[v0 + k]);
        if ((bits[0] >> k) & 1u) e2 += nvalid - lower;
        if ((bits[1] >> k) & 1u) e1 += lower;
      }
      if (++x == g.W) {
        x = 0;
        if (++y == g.H) {
          y = 0;
          ++z;
        }
      }
    }
  }
  int c[6] = {__popc(bits[0]), __popc(bits[1]), __popc(bits[2]), __popc(bits[3]), e2, e1};
#pragma unroll
  for (int l = 0; l < 6; ++l) {
    for (int o = 16; o > 0; o >>= 1) c[l] += __shfl_xor_sync(0xffffffffu, c[l], o);
    if (lane_id() == 0) bcount[l * nb + b] = c[l];
  }
}

// Single block: exclusive scan of nlists x nb block counts in place, list
// totals to totals[0 .. nlists).  The CP lists use totals = ctr + C_NS2.  Each
// thread takes 32 consecutive counts per pass.
__global__ void __launch_bounds__(1024) k_scan_lists(int* __restrict__ bcount, int nb, int nlists,
                                                     int* totals) {
  constexpr int kPer = 32;
  __shared__ int carry;
  __shared__ int warp_sums[32];
  for (int l = 0; l < nlists; ++l) {
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    int* c = bcount + (long long)l * nb;
    for (int base = 0; base < nb; base += 1024 * kPer) {
      const int i0 = base + (int)threadIdx.x * kPer;
      int x[kPer];
      int sum = 0;
#pragma unroll
      for (int k = 0; k < kPer; ++k) {
        x[k] = i0 + k < nb ? c[i0 + k] : 0;
        sum += x[k];
      }
      int incl = sum;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane_id() >= (unsigned)o) incl += y;
      }
      if (lane_id() == 31) warp_sums[threadIdx.x / 32] = incl;
      __syncthreads();
      if (threadIdx.x < 32) {
        int w = warp_sums[threadIdx.x], wi = w;
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, wi, o);
          if (lane_id() >= (unsigned)o) wi += y;
        }
        warp_sums[threadIdx.x] = wi - w;
      }
      __syncthreads();
      int run = carry + warp_sums[threadIdx.x / 32] + incl - sum;
#pragma unroll
      for (int k = 0; k < kPer; ++k) {
        if (i0 + k < nb) c[i0 + k] = run;
        run += x[k];
      }
      __syncthreads();
      if (threadIdx.x == 1023) carry = run;
      __syncthreads();
    }
    if (threadIdx.x == 0) totals[l] = carry;
    __syncthreads();
  }
}

// Exclusive scan in place of lists of n counts (list l at c + l * n, one per
// blockIdx.y) for lists too long for one block: the sum of every 1024-count
// chunk (k_chunk_sums, into sums + l * gridDim.x), a scan of the sums with the
// list totals (k_scan_lists, one block), then each chunk scanned from its
// offset (k_chunk_scan).
__global__ void __launch_bounds__(1024) k_chunk_sums(const int* __restrict__ c, int n,
                                                     int* __restrict__ sums) {
  __shared__ int ws[32];
  c += (long long)blockIdx.y * n;
  sums += (long long)blockIdx.y * gridDim.x;
  const int i = blockIdx.x * 1024 + threadIdx.x;
  int x = i < n ? c[i] : 0;
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  if (lane_id() == 0) ws[threadIdx.x >> 5] = x;
  __syncthreads();
  if (threadIdx.x < 32) {
    int y = ws[threadIdx.x];
    for (int o = 16; o > 0; o >>= 1) y += __shfl_xor_sync(0xffffffffu, y, o);
    if (threadIdx.x == 0) sums[blockIdx.x] = y;
  }
}

__global__ void __launch_bounds__(1024) k_chunk_scan(int* __restrict__ c, int n,
                                                     const int* __restrict__ offs) {
  __shared__ int ws[32];
  c += (long long)blockIdx.y * n;
  offs += (long long)blockIdx.y * gridDim.x;
  const int i = blockIdx.x * 1024 + threadIdx.x;
  const int x = i < n ? c[i] : 0;
  int incl = x;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane_id() >= (unsigned)o) incl += y;
  }
  if (lane_id() == 31) ws[threadIdx.x >> 5] = incl;
  __syncthreads();
  if (threadIdx.x < 32) {
    const int w = ws[threadIdx.x];
    int wi = w;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane_id() >= (unsigned)o) wi += y;
    }
    ws[threadIdx.x] = wi - w;
  }
  __syncthreads();
  if (i < n) c[i] = offs[blockIdx.x] + ws[threadIdx.x >> 5] + incl - x;
}

__global__ void __launch_bounds__(32 * kCpWarps) k_cp_write(const int8_t* __restrict__ otype,
                                                           int N, int nb,
                                                           const int* __restrict__ boff,
                                                           int* sad2, int* sad1, int* maxima,
                                                           int* minima) {
  const int b = blockIdx.x * kCpWarps + (int)(threadIdx.x >> 5);
  if (b >= nb) return;
  const int v0 = b * kCpBlock + (int)lane_id() * 32;
  unsigned bits[4];
  cp_lane_bits(otype, N, v0, bits);
  int* outs[4] = {sad2, sad1, maxima, minima};
#pragma unroll
  for (int l = 0; l < 4; ++l) {
    const int c = __popc(bits[l]);
    int incl = c;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane_id() >= (unsigned)o) incl += y;
    }
    int pos = boff[l * nb + b] + incl - c;
    for (unsigned m = bits[l]; m; m &= m - 1) {
      const int v = v0 + __ffs(m) - 1;
      outs[l][pos] = v;
      ++pos;
    }
  }
}

// ext[maxima[i]] = i and ext[minima[i]] = i (computeMaxIndex / computeMinIndex
// :1928-1939 share one array).
template <class T>
__global__ void k_ext_index(Job<T> J) {
  const int nmax = J.ctr[C_NMAX], nmin = J.ctr[C_NMIN];
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nmax + nmin; i += stride) {
    if (i < nmax) J.ext[J.maxima[i]] = i;
    else J.ext[J.minima[i - nmax]] = i - nmax;
  }
}

// ---------------------------------------------------------------------------
// Saddle rows: findAscPaths (:1832-1926) and findDescPaths (:1956-2049).
// Row i belongs to the i-th ORIGINAL saddle for both fields.  Only [0, count)
// and the count are written, so entries past a shorter row keep their last
// value, as in the reference.
// ---------------------------------------------------------------------------
template <class T, bool kAsc>
__global__ void __launch_bounds__(256, 4) k_rows(Job<T> J, const T* __restrict__ a,
                                              const int* __restrict__ lab, const int* __restrict__ sad,
                                              int ns_slot, int* __restrict__ rows,
                                              uint8_t* __restrict__ ocnt, int4* __restrict__ orm,
                                              int4* __restrict__ oend) {
  const int ns = J.ctr[ns_slot];
  const int stride = gridDim.x * blockDim.x;
  const Dims g = J.dim;
  const int WH = g.W * g.H;
  for (int base = blockIdx.x * blockDim.x; base < ns; base += stride) {  // uniform per warp
    const int i = base + threadIdx.x;
    const bool act = i < ns;
    const int s = act ? sad[i] : 0;
    int x, y, z;
    coords(s, g, x, y, z);
    const int valid = act ? valid_mask(boundary_code(x, y, z, g.W, g.H, g.D)) : 0;
    const T sv = a[s];
    // Neighbour values, then the side's labels, then their values: three
    // batches of independent loads; the sort below compares cached values.
    T val[kNumDirs];
#pragma unroll
    for (int d = 0; d < kNumDirs; ++d)
      val[d] = (valid >> d & 1) ? a[s + dir_x(d) + dir_y(d) * g.W + dir_z(d) * WH] : T(0);
    int lb[kNumDirs];
#pragma unroll
    for (int d = 0; d < kNumDirs; ++d) {
      const int r = s + dir_x(d) + dir_y(d) * g.W + dir_z(d) * WH;
      const bool side = (valid >> d & 1) && (kAsc ? above(val[d], r, sv, s) : below(val[d], r, sv, s));
      lb[d] = side ? lab[r] : -1;
    }
#pragma unroll
    for (int d = 0; d < kNumDirs; ++d) val[d] = lb[d] >= 0 ? a[lb[d]] : T(0);
    unsigned keep = 0;
#pragma unroll
    for (int d = 0; d < kNumDirs; ++d)
      if (lb[d] >= 0 && (!kAsc || tabs(T(val[d] - sv)) >= J.thr)) keep |= 1u << d;
    const int cnt = __popc(keep);
    // The reference sorts each row (insertionSort :1795-1811, descending, for
    // ascending rows; reversed_insertionSort :1813-1829, ascending, for
    // descending rows) by (value, label).  What is read back from an original
    // row is its count, its first and last entry in that order
    // (get_wrong_index_max / _min) and the set of extrema it names
    // (findLargestSaddlePerMax / _Min, get_wrong_index_saddles(_join), where a
    // repeated label adds nothing: only the row decides).  So the row is not
    // sorted: the first and last entry come from one pass, and the entries
    // are kept in direction order as extremum indices, a repeated label's
    // entry as -1.
    int fl = -1, ll = -1;
    T fv = T(0), lv = T(0);
#pragma unroll
    for (int d = 0; d < kNumDirs; ++d) {
      if (!(keep >> d & 1u)) continue;
      // Strict comparisons: among equal entries (one label) the first kept
      // direction stays, so first and last are never a repeat.
      const bool first = fl < 0 || (kAsc ? above(val[d], lb[d], fv, fl) : below(val[d], lb[d], fv, fl));
      const bool last = ll < 0 || (kAsc ? below(val[d], lb[d], lv, ll) : above(val[d], lb[d], lv, ll));
      if (first) { fv = val[d]; fl = lb[d]; }
      if (last) { lv = val[d]; ll = lb[d]; }
    }
    unsigned dup = 0u;  // kept entries whose label an earlier kept entry has
#pragma unroll
    for (int d = 1; d < kNumDirs; ++d)
#pragma unroll
      for (int e = 0; e < d; ++e)
        if ((keep >> e & keep >> d & 1u) && lb[e] == lb[d]) dup |= 1u << d;
    int* out = rows + (long long)i * kRowStride;
    if (act) {
      ocnt[i] = (uint8_t)cnt;
      oend[i] = make_int4(fl, ll, fl >= 0 ? J.ext[fl] : -1, ll >= 0 ? J.ext[ll] : -1);
    }
    // Per kept entry, at its position among the kept ones: the first four in
    // the compact copy, the rest in the row.  And the first pass of
    // findLargestSaddlePerMax / findSmallestSaddlePerMin (:4890-4940) over
    // the row: each named extremum's largest (smallest) saddle key, and the
    // number of rows naming it, for the per-extremum entry lists of the
    // incremental wrong-saddle scan (filled by k_extreme_saddle).  Lanes
    // naming the same extremum share one atomic; a read first skips most key
    // atomics (the key only moves one way).
    using KK = typename KeyOf<T>::K;
    const KK key = KeyOf<T>::enc(sv + T(0));  // -0 and +0 compare equal
    int* mcount = kAsc ? J.moff2 : J.moff1;
    // The extremum indices of the fresh entries first, all gathers in flight
    // together (loads after an atomic would wait for it).
    int mp[kNumDirs];
#pragma unroll
    for (int d = 0; d < kNumDirs; ++d)
      mp[d] = (keep >> d & ~dup >> d & 1u) ? J.ext[lb[d]] : -1;
    int m0 = -1, m1 = -1, m2 = -1, m3 = -1;
    int pos = 0;
#pragma unroll
    for (int d = 0; d < kNumDirs; ++d) {
      const bool kd = keep >> d & 1u;
      const unsigned grp = __match_any_sync(0xffffffffu, mp[d]);
      if (mp[d] >= 0 && (grp & ((1u << lane_id()) - 1u)) == 0u) atomicAdd(mcount + mp[d], __popc(grp));
      if (kd) {
        m0 = pos == 0 ? mp[d] : m0;
        m1 = pos == 1 ? mp[d] : m1;
        m2 = pos == 2 ? mp[d] : m2;
        m3 = pos == 3 ? mp[d] : m3;
        if (pos >= 4) out[pos] = mp[d];
        ++pos;
      }
    }
    if (act) orm[i] = make_int4(m0, m1, m2, m3);
    // Then the key reads, seven at a time, and the atomics they call for.
#pragma unroll
    for (int h = 0; h < kNumDirs; h += 7) {
      KK cur[7];
#pragma unroll
      for (int d = 0; d < 7; ++d) cur[d] = mp[h + d] >= 0 ? J.ext_key[mp[h + d]] : KK(0);
#pragma unroll
      for (int d = 0; d < 7; ++d) {
        if (mp[h + d] < 0 || !(kAsc ? key > cur[d] : key < cur[d])) continue;
        if (kAsc) atomicMax(J.ext_key + mp[h + d], key);
        else atomicMin(J.ext_key + mp[h + d], key);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Largest saddle per maximum / smallest per minimum on the ORIGINAL field
// (findLargestSaddlePerMax / findSmallestSaddlePerMin :4890-4940): the CSR
// max->saddle table is never materialised; every (row, entry) pair votes.
// k_rows selects the extreme value key per extremum (and counts the entries
// naming it); this pass selects the extreme id at that key and files the
// entries into the per-extremum lists (cursors start at the scanned offsets).
// ---------------------------------------------------------------------------
template <class T, bool kMax>
__global__ void __launch_bounds__(256) k_extreme_saddle(Job<T> J) {
  using K = typename KeyOf<T>::K;
  const int ns = J.ctr[kMax ? C_NS2 : C_NS1];
  const int* sad = kMax ? J.sad2 : J.sad1;
  const int* rows = kMax ? J.orow2 : J.orow1;
  const uint8_t* ocnt = kMax ? J.ocnt2 : J.ocnt1;
  int* cur = kMax ? J.wstamp2 : J.wstamp1;
  int* ent = kMax ? J.ment2 : J.ment1;
  const int stride = gridDim.x * blockDim.x;
  // Uniform per warp: lanes naming the same extremum (neighbouring saddles
  // usually do) share one cursor atomic.
  for (int base = blockIdx.x * blockDim.x; base < ns; base += stride) {
    const int i = base + threadIdx.x;
    const int cnt = i < ns ? ocnt[i] : 0;
    const int s = i < ns ? sad[i] : 0;
    const K key = KeyOf<T>::enc(J.f[s] + T(0));  // -0 and +0 compare equal
    const int* row = rows + (long long)(i < ns ? i : 0) * kRowStride;
    // The first four entries as extremum indices from the compact copy
    // (k_rows), longer rows' tails from the row (stored as extremum indices).
    const int4 m4 = i < ns ? (kMax ? J.orm2 : J.orm1)[i] : make_int4(-1, -1, -1, -1);
    const int pmax = __reduce_max_sync(0xffffffffu, (unsigned)cnt);
    // Seven entries at a time, each step's loads and atomics issued together
    // (a load after an atomic would wait for it).  A row names an extremum in
    // one entry only (a repeat is -1), as counted by k_rows.
#pragma unroll
    for (int h = 0; h < kNumDirs; h += 7) {
      if (h >= pmax) break;
      int m[7];
#pragma unroll
      for (int q = 0; q < 7; ++q) {
        const int p = h + q;
        m[q] = p >= cnt ? -1 : p == 0 ? m4.x : p == 1 ? m4.y : p == 2 ? m4.z : p == 3 ? m4.w : row[p];
      }
      unsigned grp[7];
#pragma unroll
      for (int q = 0; q < 7; ++q) grp[q] = __match_any_sync(0xffffffffu, m[q]);
      int at[7];
#pragma unroll
      for (int q = 0; q < 7; ++q)
        at[q] = (m[q] >= 0 && (grp[q] & ((1u << lane_id()) - 1u)) == 0u)
                    ? atomicAdd(cur + m[q], __popc(grp[q])) : 0;
      K ek[7];
#pragma unroll
      for (int q = 0; q < 7; ++q) ek[q] = m[q] >= 0 ? J.ext_key[m[q]] : K(0);
#pragma unroll
      for (int q = 0; q < 7; ++q) {
        const unsigned below = grp[q] & ((1u << lane_id()) - 1u);
        const int pos = __shfl_sync(0xffffffffu, at[q], __ffs(grp[q]) - 1) + __popc(below);
        if (m[q] < 0) continue;
        if (ek[q] == key) {
          if (kMax) atomicMax(J.ext_id + m[q], s);
          else atomicMin(J.ext_id + m[q], s);
        }
        ent[pos] = i * kRowStride + h + q;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Proposals and their application.
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ T midpoint_delta(const Job<T>& J, int i) {
  const T gi = J.g[i];
  return ((J.f[i] - J.bound) + gi) / T(2) - gi;
}
template <class T>
__device__ __forceinline__ T step_delta(const Job<T>& J, int i) {
  return J.edit_type == 1 ? midpoint_delta(J, i) : -J.bound / T(J.q);
}

// Atomic max into the proposal buffer (swap / swap1 / atomicCASDouble
// :2643-2691).  The thread that lifts a vertex off the sentinel records it.
template <class T>
__device__ __forceinline__ void propose(const Job<T>& J, int i, T d) {
  using K = typename KeyOf<T>::K;
  const K k = KeyOf<T>::enc(d);
  const K old = atomicMax(J.delta + i, k);
  if (old == J.sentinel_key && k > old) {
    const int slot = atomicAdd(J.ctr + C_TOUCHED, 1);
    J.touched[slot] = i;
  }
}

// c_loop(0..2) (:2887-3055) over the mismatch list.
template <class T>
__global__ void __launch_bounds__(256) k_propose_cp(const Job<T>* __restrict__ jobs, const __grid_constant__ Sel sel) {
  for (int jk = 0; jk < sel.n; ++jk) {
  const Job<T>& J = jobs[sel.idx[jk]];
  const int n = J.ctr[C_MM];
  const int stride = gridDim.x * blockDim.x;
  const Dims g = J.dim;
  const int WH = g.W * g.H;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
    const int ent = J.mm[e];
    const int v = ent & ((1 << kCatShift) - 1);
    const int cat = (unsigned)ent >> kCatShift;
    int x, y, z;
    coords(v, g, x, y, z);
    // Neighbours in direction order (the reference's scan order), visited
    // through static indices so that the values stay in registers and their
    // loads go out together.
    const int valid = valid_mask(boundary_code(x, y, z, g.W, g.H, g.D));
    const int ot = J.otype[v];
    const T gv = J.g[v];
    const bool need_g = (cat & kCatSaddle) || ((cat & kCatMax) && ot == 4);
    T gn[kNumDirs];
#pragma unroll
    for (int d = 0; d < kNumDirs; ++d)
      gn[d] = (need_g && (valid >> d & 1)) ? J.g[v + dir_x(d) + dir_y(d) * g.W + dir_z(d) * WH] : T(0);
    if (cat & kCatMin) {  // c_loop(1) (:2965-3039)
      if (ot != 0) {
        T fn[kNumDirs];
#pragma unroll
        for (int d = 0; d < kNumDirs; ++d)
          fn[d] = (valid >> d & 1) ? J.f[v + dir_x(d) + dir_y(d) * g.W + dir_z(d) * WH] : T(0);
        int S = v;
        T sval = J.f[v];
#pragma unroll
        for (int d = 0; d < kNumDirs; ++d) {
          const int r = v + dir_x(d) + dir_y(d) * g.W + dir_z(d) * WH;
          if ((valid >> d & 1) && below(fn[d], r, sval, S)) { S = r; sval = fn[d]; }
        }
        const T gs = J.g[S];
        const T d = J.edit_type == 1 ? ((sval - J.bound) + gs) / T(2) - gs : -J.bound / T(J.q);
        if (!(gv > gs || (gv == gs && v > S))) propose(J, S, d);
      } else {
        propose(J, v, step_delta(J, v));
      }
    }
    if (cat & kCatSaddle) {  // c_loop(2) -> fix_saddle_local (:2804-2884)
      int dm = 0;
#pragma unroll
      for (int d = 0; d < kNumDirs; ++d) {
        const int r = v + dir_x(d) + dir_y(d) * g.W + dir_z(d) * WH;
        if ((valid >> d & 1) && (gn[d] < gv || (gn[d] == gv && r < v))) dm |= 1 << d;
      }
      const int om = J.olm[v];
#pragma unroll
      for (int d = 0; d < kNumDirs; ++d) {
        const int r = v + dir_x(d) + dir_y(d) * g.W + dir_z(d) * WH;
        if ((valid >> d & 1) && (om >> d & 1) && !(dm >> d & 1)) propose(J, r, step_delta(J, r));
      }
      if (dm & ~om) propose(J, v, step_delta(J, v));
    }
    if (cat & kCatMax) {  // c_loop(0) (:2890-2963)
      if (ot != 4) {
        propose(J, v, step_delta(J, v));
      } else {
        int L = v;
        T lval = gv;
#pragma unroll
        for (int d = 0; d < kNumDirs; ++d) {
          const int r = v + dir_x(d) + dir_y(d) * g.W + dir_z(d) * WH;
          if ((valid >> d & 1) && above(gn[d], r, lval, L)) { L = r; lval = gn[d]; }
        }
        if (L != v) propose(J, L, step_delta(J, L));
      }
    }
  }
  }
}

// applyDeltaBuffer (:3061-3111) over the vertices that received a proposal;
// the proposal buffer is reset to the sentinel on the way (init_delta).
template <class T>
__global__ void __launch_bounds__(256) k_apply(const Job<T>* __restrict__ jobs, const __grid_constant__ Sel sel) {
  for (int jk = 0; jk < sel.n; ++jk) {
  const Job<T>& J = jobs[sel.idx[jk]];
  const int dirty_epoch = J.ctr[C_DEPOCH];
  const int n = J.ctr[C_TOUCHED];
  const int stride = gridDim.x * blockDim.x;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
    const int v = J.touched[e];
    const T d = KeyOf<T>::dec(J.delta[v]);
    J.delta[v] = J.sentinel_key;
    if (d == J.sentinel) continue;
    const T fv = J.f[v];
    const T g0 = J.g[v];
    T gv = g0;
    if (J.edit_type == 0) {
      const int c = J.counter[v];
      if (c < J.q - 1 && tabs(T(fv - (gv + d))) <= J.bound) {
        gv += d;
        J.counter[v] = c + 1;
      } else {
        J.counter[v] = J.q;
        gv = fv - J.bound;
      }
    } else {
      if (tabs(T(fv - (gv + d))) <= J.bound) gv += d;
      else gv = fv - J.bound;
    }
    J.g[v] = gv;
    if (KeyOf<T>::enc(gv) != KeyOf<T>::enc(g0)) {
      J.ctr[C_CHANGED] = 1;
      atomicOr(J.vchg + (v >> 5), 1u << (v & 31));
      atomicOr(J.wchg2 + (v >> 5), 1u << (v & 31));
      atomicOr(J.wchg1 + (v >> 5), 1u << (v & 31));
      if (J.edited) atomicOr(J.edited + (v >> 5), 1u << (v & 31));
      int x, y, z;
      coords(v, J.dim, x, y, z);
      mark_tiles(J.tdirty, J.dim, x, y, z);
      if (atomicExch(J.dstamp + v, dirty_epoch) != dirty_epoch)
        J.dirty[atomicAdd(J.ctr + C_DIRTY, 1)] = v;
    }
  }
  }
}

// ---------------------------------------------------------------------------
// Wrong manifold neighbours (get_wrong_split_neighbors / get_wrong_join_neighbors
// :2400-2513) in the canonical order "saddles in ascending id": saddle s flags
// its first candidate neighbour not flagged by a smaller saddle.
//
// Candidates of s: valid neighbours r (direction order) with r above s in the
// decompressed field and dds[r] != ds[r] (split), or below and das[r] != as[r]
// (join).  Resolution runs in rounds: every unresolved saddle votes (atomic
// max of (round << 32) | ~s) on each of its remaining candidates; a saddle
// commits its first remaining candidate when its own vote won, i.e. no smaller
// unresolved saddle can still take it.  The smallest unresolved saddle always
// commits, and a larger one never takes what a smaller one could still take,
// so the result equals the sequential greedy.
// ---------------------------------------------------------------------------
// Candidate lists this short are resolved by one block (k_wn_resolve) alone.
constexpr int kWnBlockMax = 4096;

template <class T, bool kSplit>
__device__ __forceinline__ int wn_candidates(const Job<T>& J, int s, int* ids) {
  const int n = neighbours(s, J.dim, ids, nullptr);
  const T sv = J.g[s];
  int k = 0;
  for (int j = 0; j < n; ++j) {
    const int r = ids[j];
    const T rv = J.g[r];
    const bool side = kSplit ? above(rv, r, sv, s) : below(rv, r, sv, s);
    const bool wrong = kSplit ? (J.dds[r] != J.ds[r]) : (J.das[r] != J.as[r]);
    if (side && wrong) ids[k++] = r;
  }
  return k;
}

// Row order of the decompressed rows: "comes first in the row" is descending
// for ascending rows, ascending else.
template <class T, bool kSplit>
__device__ __forceinline__ bool row_first(T v, int m, T bv, int bm) {
  return kSplit ? above(v, m, bv, bm) : below(v, m, bv, bm);
}

template <class T, bool kSplit>
__device__ __noinline__ int row_entry_k(const Job<T>& J, int s, int k) {
  const int* lab = kSplit ? J.dds : J.das;
  int ids[kNumDirs];
  const int n = neighbours(s, J.dim, ids, nullptr);
  const T sv = J.g[s];
  int ml[kNumDirs];
  T mv[kNumDirs];
  int cnt = 0;
  for (int j = 0; j < n; ++j) {
    const int r = ids[j];
    const T rv = J.g[r];
    if (kSplit ? above(rv, r, sv, s) : below(rv, r, sv, s)) {
      const int m = lab[r];
      const T v = J.g[m];
      if (!kSplit || tabs(T(v - sv)) >= J.thr) {
        ml[cnt] = m;
        mv[cnt] = v;
        ++cnt;
      }
    }
  }
  for (int a = 0; a < cnt; ++a) {
    int before = 0, same = 0;
    for (int b = 0; b < cnt; ++b) {
      before += row_first<T, kSplit>(mv[b], ml[b], mv[a], ml[a]);
      same += ml[b] == ml[a];
    }
    if (before <= k && k < before + same) return ml[a];
  }
  return -1;
}

// One saddle of one side: its decompressed row summary (count, first and
// last entry in row order) into the row slots, and whether some neighbour on
// the side has a wrong label.  The loads go out in three batches of
// independent gathers (neighbour values; labels and mismatch bits of the
// neighbours on the side; the labels' values), not one dependent chain per
// neighbour.
template <class T, bool kSplit>
__device__ __forceinline__ bool saddle_row(const Job<T>& J, int i, int s) {
  const Dims g = J.dim;
  const int WH = g.W * g.H;
  int x, y, z;
  coords(s, g, x, y, z);
  const int valid = valid_mask(boundary_code(x, y, z, g.W, g.H, g.D));
  const T* __restrict__ gv = J.g;
  const int* __restrict__ lab = kSplit ? J.dds : J.das;
  const T sv = __ldg(gv + s);
  // Neighbour values, then the side's labels and mismatch bytes, then the
  // labels' values: batches of independent gathers, values seven at a time
  // (fourteen live values spill at 64 registers).
  unsigned side = 0;
#pragma unroll
  for (int h = 0; h < kNumDirs; h += 7) {
    T val[7];
#pragma unroll
    for (int q = 0; q < 7; ++q) {
      const int d = h + q;
      val[q] = (valid >> d & 1) ? __ldg(gv + s + dir_x(d) + dir_y(d) * g.W + dir_z(d) * WH) : T(0);
    }
#pragma unroll
    for (int q = 0; q < 7; ++q) {
      const int d = h + q;
      const int r = s + dir_x(d) + dir_y(d) * g.W + dir_z(d) * WH;
      if ((valid >> d & 1) && (kSplit ? above(val[q], r, sv, s) : below(val[q], r, sv, s)))
        side |= 1u << d;
    }
  }
  int ml[kNumDirs];
  int mb = 0;
#pragma unroll
  for (int d = 0; d < kNumDirs; ++d) {
    const int r = s + dir_x(d) + dir_y(d) * g.W + dir_z(d) * WH;
    ml[d] = (side >> d & 1) ? __ldg(lab + r) : -1;
    mb |= (side >> d & 1) ? __ldg(J.mis + r) : 0;
  }
  T fv = T(0), lv = T(0);
  int cnt = 0, fm = -1, lm = -1;
#pragma unroll
  for (int h = 0; h < kNumDirs; h += 7) {
    T val[7];
#pragma unroll
    for (int q = 0; q < 7; ++q) val[q] = ml[h + q] >= 0 ? __ldg(gv + ml[h + q]) : T(0);
#pragma unroll
    for (int q = 0; q < 7; ++q) {
      const int m = ml[h + q];
      const T v = val[q];
      if (m >= 0 && (!kSplit || tabs(T(v - sv)) >= J.thr)) {
        if (cnt == 0 || row_first<T, kSplit>(v, m, fv, fm)) { fv = v; fm = m; }
        if (cnt == 0 || row_first<T, kSplit>(lv, lm, v, m)) { lv = v; lm = m; }
        ++cnt;
      }
    }
  }
  const int oc = (kSplit ? J.ocnt2 : J.ocnt1)[i];
  if (oc > 0 && cnt > 0) {
    int* slots = kSplit ? J.drow2 : J.drow1;
    const int k = oc - 1;
    slots[2ll * i] = fm;
    if (cnt > k) {
      int kth;
      if (k == cnt - 1) kth = lm;
      else if (k == 0) kth = fm;
      else kth = row_entry_k<T, kSplit>(J, s, k);
      slots[2ll * i + 1] = kth;
    }
  }
  return (mb >> (kSplit ? 0 : 1)) & 1;
}

// Clears the value-change bitset after a computed round's jump has read it.
template <class T>
__global__ void k_clear_changed(const Job<T>* __restrict__ jobs, const __grid_constant__ Sel sel) {
  for (int jk = 0; jk < sel.n; ++jk) {
    const Job<T>& J = jobs[sel.idx[jk]];
    if (J.ctr[C_MFSKIP]) continue;
    const int nw = (J.dim.N + 31) >> 5;
    const int stride = gridDim.x * blockDim.x;
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += stride) {
      J.vchg[w] = 0u;
      J.rtouch2[w] = 0u;
      J.rtouch1[w] = 0u;
    }

  }
}

// Whether any input of saddle s's rows changed since the previous computed
// round: the changed-input byte of s or of a neighbour (see k_jump2).
template <class T>
__device__ __forceinline__ bool saddle_inputs_changed(const Job<T>& J, int s) {
  const Dims g = J.dim;
  int x, y, z;
  coords(s, g, x, y, z);
  const int valid = valid_mask(boundary_code(x, y, z, g.W, g.H, g.D));
  // Changed-input bytes hold the low byte of the round stamp that set them.
  const uint8_t st8 = (uint8_t)J.ctr[C_WNSTAMP];
  bool d = J.dirtyv[s] == st8;
#pragma unroll
  for (int k = 0; k < kNumDirs; ++k)
    if (valid >> k & 1) d |= J.dirtyv[s + dir_x(k) + dir_y(k) * g.W + dir_z(k) * g.W * g.H] == st8;
  return d;
}

// Fused pass over the original saddles after a manifold round, both sides in
// one grid.  A saddle whose inputs did not change since the previous computed
// round keeps its row slots and reuses its stored seed bit.  A block takes a chunk of the id space (pass_chunk blocks of 1024
// ids) and the entries of both saddle lists in it, so that the two sides read
// the same neighbourhoods together:
//  * decompressed row slots.  The reference rewrites row i (findAscPaths /
//    findDescPaths, :1832-2049) in place each round, and its only reader,
//    get_wrong_index_max / _min (:3113-3171), reads entry 0 and entry k =
//    (original count - 1), possibly stale when the new row is shorter.  So two
//    persistent slots per row reproduce it: slot 0 takes the new entry 0 when
//    the new row is non-empty, slot 1 takes the new entry k when the new row
//    has more than k entries.  Entry 0 is the row's extreme label in the sort
//    order and entry count-1 the opposite extreme, found in one pass; any other
//    entry k is found by ranking the candidates (rare: the rows of both fields
//    usually have the same length).
//  * wrong-neighbour seeds (get_wrong_split_neighbors / _join_ :2400-2513):
//    saddles with a neighbour on the side whose label differs from the
//    original's, 2-saddles to cand, 1-saddles to cand_j.
template <class T>
__global__ void __launch_bounds__(256, 4) k_saddle_pass(const Job<T>* __restrict__ jobs,
                                                        const __grid_constant__ Sel sel) {
  for (int jk = 0; jk < sel.n; ++jk) {
    const Job<T>& J = jobs[sel.idx[jk]];
    if (J.ctr[C_MFSKIP]) continue;
    const int ns2 = J.ctr[C_NS2], ns1 = J.ctr[C_NS1];
    const int nb = (J.dim.N + kCpBlock - 1) / kCpBlock;
    const int chunk = J.pass_chunk;
    const int nchunk = (nb + chunk - 1) / chunk;
    // In the first round every changed-input byte is set (the change bitset
    // starts full), so the check is skipped.
    const bool all_new = J.ctr[C_MFFIRST] != 0;
    // Later rounds first ask the jump's per-block flags (written when N is a
    // multiple of 4) whether any changed-input byte is set where the chunk's
    // saddles could see one: the 3 x 3 row windows of the planes and rows
    // next to the chunk, one id wider on each side.
    const bool by_block = !all_new && (J.dim.N & 3) == 0;
    const long long W = J.dim.W, WH = W * J.dim.H, N = J.dim.N;
    for (int c = blockIdx.x; c < nchunk; c += gridDim.x) {
      const int b0 = c * chunk, b1 = min(b0 + chunk, nb);
      const int a2 = J.cpoff[b0], e2 = b1 < nb ? J.cpoff[b1] : ns2;
      const int a1 = J.cpoff[nb + b0], e1 = b1 < nb ? J.cpoff[nb + b1] : ns1;
      const int n2 = e2 - a2, n = n2 + (e1 - a1);
      if (by_block) {
        int seen = 0;
        if (threadIdx.x < 9) {
          const int t = (int)threadIdx.x;  // signed: the offsets below go negative
          const long long off = (long long)(t / 3 - 1) * WH + (long long)(t % 3 - 1) * W;
          const long long lo = max(0ll, (long long)b0 * kCpBlock + off - 1);
          const long long hi = min(N - 1, (long long)b1 * kCpBlock - 1 + off + 1);
          const int stamp = J.ctr[C_WNSTAMP];
          for (long long b = lo >> 10; b <= (hi >> 10) && lo <= hi; ++b)
            seen |= J.bdirty[b] == stamp;
        }
        if (!__syncthreads_or(seen)) {  // no saddle here has a changed input
          // Seed bits as computed in an earlier round; none set: nothing to list.
          if (J.hcnt[c] == 0) continue;
          for (int base = 0; base < n; base += blockDim.x) {
            const int k = base + threadIdx.x;
            const bool split = k < n2;
            bool has = false;
            int s = 0;
            if (k < n) {
              const int i = split ? a2 + k : a1 + k - n2;
              s = split ? J.sad2[i] : J.sad1[i];
              has = (split ? J.has2 : J.has1)[i] != 0;
            }
            const int slot2 = warp_append(J.ctr + C_CAND, has && split, 0xffffffffu);
            if (slot2 >= 0) J.cand[slot2] = s;
            const int slot1 = warp_append(J.ctr + C_CANDJ, has && !split, 0xffffffffu);
            if (slot1 >= 0) J.cand_j[slot1] = s;
          }
          continue;
        }
      }
      int nhas = 0;  // seed bits set in the chunk
      for (int base = 0; base < n; base += blockDim.x) {  // uniform in the block
        const int k = base + threadIdx.x;
        const bool split = k < n2;
        bool has = false;
        int s = 0;
        if (k < n) {
          const int i = split ? a2 + k : a1 + k - n2;
          uint8_t* hb = split ? J.has2 : J.has1;
          s = split ? J.sad2[i] : J.sad1[i];
          const uint8_t kept = hb[i];  // loaded with the id: no round trip of its own
          if (all_new || saddle_inputs_changed(J, s)) {
            has = split ? saddle_row<T, true>(J, i, s) : saddle_row<T, false>(J, i, s);
            hb[i] = (uint8_t)has;
          } else {  // rows and seed bit as computed in an earlier round
            has = kept != 0;
          }
        }
        const int slot2 = warp_append(J.ctr + C_CAND, has && split, 0xffffffffu);
        if (slot2 >= 0) J.cand[slot2] = s;
        const int slot1 = warp_append(J.ctr + C_CANDJ, has && !split, 0xffffffffu);
        if (slot1 >= 0) J.cand_j[slot1] = s;
        nhas += __syncthreads_count(has);
      }
      if (threadIdx.x == 0) J.hcnt[c] = nhas;
    }
  }
}

template <class T, bool kSplit>
__global__ void __launch_bounds__(256) k_wn_vote(const Job<T>* __restrict__ jobs, const __grid_constant__ Sel sel,
                                                 int r) {
  for (int jk = 0; jk < sel.n; ++jk) {
  const Job<T>& J = jobs[sel.idx[jk]];
  if (J.ctr[C_MFSKIP] || J.wn_lockstep) continue;
  if (r == 0) {
    // A short list (every round after the first few of a correction) goes to
    // the block completion whole: the grid rounds would be launches with
    // nothing to do.
    const bool small = J.ctr[C_CAND] <= kWnBlockMax;
    if (blockIdx.x == 0 && threadIdx.x == 0) J.ctr[C_WNSMALL] = small;
    if (small) continue;
  } else if (J.ctr[C_WNSMALL]) {
    continue;
  }
  const unsigned long long round = (unsigned)(J.ctr[C_WNROUND] + r + 1);
  const int stamp = J.ctr[C_WNSTAMP];
  const int n = J.ctr[C_CAND + (r & 1)];
  const int* cur = (r & 1) ? J.cand_next : J.cand;
  // The list this round's commit fills (the one read two rounds ago).
  if (blockIdx.x == 0 && threadIdx.x == 0) J.ctr[C_CAND + ((r + 1) & 1)] = 0;
  const int* taken = kSplit ? J.taken : J.taken1;
  const int stride = gridDim.x * blockDim.x;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
    const int s = cur[e];
    int ids[kNumDirs];
    const int k = wn_candidates<T, kSplit>(J, s, ids);
    const unsigned long long vote = (round << 32) | (unsigned)(~s);
    for (int j = 0; j < k; ++j)
      if (taken[ids[j]] != stamp) atomicMax(J.claim + ids[j], vote);
  }
  }
}

template <class T, bool kSplit>
__global__ void __launch_bounds__(256) k_wn_commit(const Job<T>* __restrict__ jobs, const __grid_constant__ Sel sel,
                                                   int r) {
  for (int jk = 0; jk < sel.n; ++jk) {
  const Job<T>& J = jobs[sel.idx[jk]];
  if (J.ctr[C_MFSKIP] || J.ctr[C_WNSMALL] || J.wn_lockstep) continue;
  const unsigned long long round = (unsigned)(J.ctr[C_WNROUND] + r + 1);
  const int stamp = J.ctr[C_WNSTAMP];
  const int n = J.ctr[C_CAND + (r & 1)];
  const int* cur = (r & 1) ? J.cand_next : J.cand;
  int* nxt = (r & 1) ? J.cand : J.cand_next;
  int* nnext = J.ctr + C_CAND + ((r + 1) & 1);
  int* taken = kSplit ? J.taken : J.taken1;
  int* flagged = kSplit ? J.flagged : J.flagged1;
  int* nflag = J.ctr + (kSplit ? C_NFC : C_NFC1);
  const int stride = gridDim.x * blockDim.x;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
    const int s = cur[e];
    int ids[kNumDirs];
    const int k = wn_candidates<T, kSplit>(J, s, ids);
    int first = -1;
    for (int j = 0; j < k; ++j)
      if (taken[ids[j]] != stamp) { first = ids[j]; break; }
    if (first < 0) continue;  // every candidate already flagged: resolved
    const unsigned long long vote = (round << 32) | (unsigned)(~s);
    if (J.claim[first] == vote) {
      taken[first] = stamp;
      flagged[atomicAdd(nflag, 1)] = first;
    } else {
      nxt[atomicAdd(nnext, 1)] = s;
    }
  }
  }
}

// Grid-wide vote / commit rounds per side before the per-job completion.
// Round r reads the candidate list of parity r & 1 (cand / cand_next, counts
// C_CAND / C_CAND_NEXT) and refills the other; its vote number is the job's
// base round + r + 1.  Lists of at most kWnBlockMax saddles skip them.
constexpr int kWnGridRounds = 3;

// Completion of the arbitration for whatever the grid-wide rounds left
// unresolved: one block per job runs further vote / commit rounds until no
// saddle is left.  Each round commits at least the smallest unresolved saddle
// (its vote wins on every candidate it votes on), so at most n rounds run; the
// device iteration limit bounds them as well.  claim and taken are read
// through L2 (__ldcg): other threads of the block update them with atomics
// and stores between the barriers.
template <class T, bool kSplit>
__global__ void __launch_bounds__(1024) k_wn_resolve(Job<T>* __restrict__ jobs, const __grid_constant__ Sel sel) {
  if (blockIdx.x >= sel.n) return;
  Job<T>& J = jobs[sel.idx[blockIdx.x]];
  if (J.ctr[C_MFSKIP] || J.wn_lockstep) return;
  __shared__ int s_next;
  const int stamp = J.ctr[C_WNSTAMP];
  int* taken = kSplit ? J.taken : J.taken1;
  int* flagged = kSplit ? J.flagged : J.flagged1;
  int* nflag = J.ctr + (kSplit ? C_NFC : C_NFC1);
  // The grid-wide rounds left their list in parity kWnGridRounds & 1; a short
  // list skipped them and is still in parity 0.
  const int par = J.ctr[C_WNSMALL] ? 0 : (kWnGridRounds & 1);
  int* cur = par ? J.cand_next : J.cand;
  int* nxt = par ? J.cand : J.cand_next;
  int n = J.ctr[C_CAND + par];
  unsigned long long round = (unsigned)(J.ctr[C_WNROUND] + kWnGridRounds);
  const int cap = J.iter_cap;
  int it = 0;
  while (n > 0) {
    if (it++ >= cap) {
      if (threadIdx.x == 0) atomicOr(J.ctr + C_ERROR, kErrResolve);
      break;
    }
    ++round;
    const unsigned long long hi = round << 32;
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
      const int s = __ldcg(cur + e);
      int ids[kNumDirs];
      const int k = wn_candidates<T, kSplit>(J, s, ids);
      const unsigned long long vote = hi | (unsigned)(~s);
      for (int j = 0; j < k; ++j)
        if (__ldcg(taken + ids[j]) != stamp) atomicMax(J.claim + ids[j], vote);
    }
    if (threadIdx.x == 0) s_next = 0;
    __syncthreads();
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
      const int s = __ldcg(cur + e);
      int ids[kNumDirs];
      const int k = wn_candidates<T, kSplit>(J, s, ids);
      int first = -1;
      for (int j = 0; j < k; ++j)
        if (__ldcg(taken + ids[j]) != stamp) {
          first = ids[j];
          break;
        }
      if (first < 0) continue;  // every candidate already flagged: resolved
      const unsigned long long vote = hi | (unsigned)(~s);
      if (__ldcg(J.claim + first) == vote) {
        taken[first] = stamp;
        flagged[atomicAdd(nflag, 1)] = first;
      } else {
        nxt[atomicAdd(&s_next, 1)] = s;
      }
    }
    __syncthreads();
    n = s_next;
    int* t = cur;
    cur = nxt;
    nxt = t;
    __syncthreads();  // every thread has read s_next before it is reset
  }
  if (threadIdx.x == 0) {
    J.ctr[C_WNROUND] = (int)round;
    if (kSplit) {  // the join side's candidates become the list to resolve next
      int* t = J.cand;
      J.cand = J.cand_j;
      J.cand_j = t;
      J.ctr[C_CAND] = J.ctr[C_CANDJ];
    } else {
      J.ctr[C_CAND] = 0;
    }
    J.ctr[C_CAND_NEXT] = 0;
  }
}

// Lockstep resolution of the wrong-neighbour flags (jobs with wn_lockstep).
// Step d flags, for every saddle of a side's candidate list that no earlier
// step resolved, its direction-d neighbour when that neighbour is a candidate
// (on the side, label differs from the original's) and no earlier step flagged
// it.  Two saddles never share their direction-d neighbour, so a step has no
// conflict, and the steps in direction order make each see every earlier one.
// This is how the reference's concurrent launch resolves its check-then-set
// when its threads advance through their neighbour loops in step
// (get_wrong_split_neighbors / _join_, src/ExtreM_cuda.cu:2400-2513): a shared
// candidate goes to the saddle that meets it at the earlier neighbour index.
// The two sides flag into separate arrays, as the reference's two kernels do,
// so one step serves both.  A saddle's resolution is marked in claim[]
// (unused by this mode) with the round's stamp: the low 32-bit half for the
// split side, the high half for the join side, so that a saddle on both lists
// (type 3) keeps one mark per side.
template <class T>
__device__ __forceinline__ void wn_step_entry(const Job<T>& J, int e, int n2, int d, int stamp) {
  const bool split = e < n2;
  const int s = split ? J.cand[e] : J.cand_j[e - n2];
  const Dims g = J.dim;
  int x, y, z;
  coords(s, g, x, y, z);
  if (!dir_valid(d, boundary_code(x, y, z, g.W, g.H, g.D))) return;
  unsigned* mark = reinterpret_cast<unsigned*>(J.claim + s) + (split ? 0 : 1);
  const unsigned done = (unsigned)stamp | 0x80000000u;  // never the zeroed initial value
  if (*mark == done) return;
  const int r = s + ddx(d) + ddy(d) * g.W + ddz(d) * g.W * g.H;
  const T sv = J.g[s], rv = J.g[r];
  if (!(split ? above(rv, r, sv, s) : below(rv, r, sv, s))) return;
  int* taken = split ? J.taken : J.taken1;
  if ((split ? J.dds[r] == J.ds[r] : J.das[r] == J.as[r]) || taken[r] == stamp) return;
  taken[r] = stamp;
  (split ? J.flagged : J.flagged1)[atomicAdd(J.ctr + (split ? C_NFC : C_NFC1), 1)] = r;
  *mark = done;
}

// One step over every selected job's two candidate lists (a large list: one
// launch per direction).
template <class T>
__global__ void __launch_bounds__(256) k_wn_step(const Job<T>* __restrict__ jobs,
                                                 const __grid_constant__ Sel sel, int d) {
  for (int jk = 0; jk < sel.n; ++jk) {
    const Job<T>& J = jobs[sel.idx[jk]];
    if (J.ctr[C_MFSKIP] || !J.wn_lockstep) continue;
    const int stamp = J.ctr[C_WNSTAMP];
    const int n2 = J.ctr[C_CAND], n = n2 + J.ctr[C_CANDJ];
    const int stride = gridDim.x * blockDim.x;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride)
      wn_step_entry(J, e, n2, d, stamp);
  }
}

// All fourteen steps in one block per job, with a barrier between steps (a
// short list: fourteen grid launches would cost more than the work).  The
// barrier makes one step's flags and marks visible to the next.
template <class T>
__global__ void __launch_bounds__(1024) k_wn_steps_block(const Job<T>* __restrict__ jobs,
                                                         const __grid_constant__ Sel sel) {
  if (blockIdx.x >= sel.n) return;
  const Job<T>& J = jobs[sel.idx[blockIdx.x]];
  if (J.ctr[C_MFSKIP] || !J.wn_lockstep) return;
  const int stamp = J.ctr[C_WNSTAMP];
  const int n2 = J.ctr[C_CAND], n = n2 + J.ctr[C_CANDJ];
  for (int d = 0; d < kNumDirs; ++d) {
    for (int e = threadIdx.x; e < n; e += blockDim.x) wn_step_entry(J, e, n2, d, stamp);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// fixpath (:4046-4206): walk the steepest ascent (descent) of both fields from a
// flagged vertex until they diverge; lower the decompressed choice (split) or
// the original choice (join).
// ---------------------------------------------------------------------------
template <class T, bool kSplit>
__global__ void __launch_bounds__(256) k_fixpath(const Job<T>* __restrict__ jobs, const __grid_constant__ Sel sel) {
  for (int jk = 0; jk < sel.n; ++jk) {
  const Job<T>& J = jobs[sel.idx[jk]];
  const int cap = J.iter_cap;
  const int n = J.ctr[kSplit ? C_NFC : C_NFC1];
  const int* list = kSplit ? J.flagged : J.flagged1;
  const int stride = gridDim.x * blockDim.x;
  const Dims g = J.dim;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
    int cur = list[e];
    int t = -1, fl = -1;
    int steps = 0;
    for (; steps < cap; ++steps) {
      int ids[kNumDirs];
      const int nn = neighbours(cur, g, ids, nullptr);
      int ni = cur, nd = cur;
      T fi = J.f[cur], gd = J.g[cur];
      for (int j = 0; j < nn; ++j) {
        const int r = ids[j];
        const T fr = J.f[r], gr = J.g[r];
        if (kSplit) {
          if (fi < fr || (fi == fr && ni < r)) { ni = r; fi = fr; }
          if (gd < gr || (gd == gr && nd < r)) { nd = r; gd = gr; }
        } else {
          if (fi > fr || (fi == fr && ni > r)) { ni = r; fi = fr; }
          if (gd > gr || (gd == gr && nd > r)) { nd = r; gd = gr; }
        }
      }
      if (ni != nd) { t = ni; fl = nd; break; }
      if (ni == cur) break;
      cur = ni;
    }
    if (steps == cap) {
      atomicOr(J.ctr + C_ERROR, kErrPath);
      continue;
    }
    if (fl == t) continue;
    const int target = kSplit ? fl : t;
    propose(J, target, step_delta(J, target));
  }
  }
}

// ---------------------------------------------------------------------------
// s_loops (:3465-3487) / s_loops_join (:3489-3512): get_wrong_index_max
// (:3113-3141) and get_wrong_index_min (:3143-3171) with the lowest saddle row
// winning per extremum, followed by the fixes (:3320-3413).
// ---------------------------------------------------------------------------
template <class T, bool kMax>
__global__ void __launch_bounds__(256) k_wim_scan(const Job<T>* __restrict__ jobs, const __grid_constant__ Sel sel) {
  for (int jk = 0; jk < sel.n; ++jk) {
  const Job<T>& J = jobs[sel.idx[jk]];
  const int ns = J.ctr[kMax ? C_NS2 : C_NS1];
  const int4* oend = kMax ? J.oend2 : J.oend1;
  const int* drow = kMax ? J.drow2 : J.drow1;
  int* first = kMax ? J.first1 : J.first_min1;
  int* flag = kMax ? J.flag2 : J.flag_min2;
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += stride) {
    const int cnt = (kMax ? J.ocnt2 : J.ocnt1)[i];
    if (cnt == 0) continue;
    // Original entries 0 and count - 1 (labels, extremum indices) against the
    // decompressed row slots: entry 0, entry (count - 1).
    const int4 o = oend[i];
    const int2 d = *reinterpret_cast<const int2*>(drow + 2ll * i);
    if (o.x != d.x) atomicMin(first + o.z, i);
    if (o.y != d.y) flag[o.w] = 1;
  }
  }
}

// Collect per extremum, count, propose the fix and reset the arbitration slots.
// fix = false: detection only (the third block of the outer loop, :5932-5951).
template <class T, bool kMax>
__global__ void __launch_bounds__(256) k_wim_collect(const Job<T>* __restrict__ jobs, const __grid_constant__ Sel sel, int fix) {
  for (int jk = 0; jk < sel.n; ++jk) {
  const Job<T>& J = jobs[sel.idx[jk]];
  const int next = J.ctr[kMax ? C_NMAX : C_NMIN];
  const int* ext_list = kMax ? J.maxima : J.minima;
  const int* drow = kMax ? J.drow2 : J.drow1;
  int* first = kMax ? J.first1 : J.first_min1;
  int* flag = kMax ? J.flag2 : J.flag_min2;
  int* c1 = J.ctr + (kMax ? C_WMC : C_WMIN);
  int* c2 = J.ctr + (kMax ? C_WMC2 : C_WMIN2);
  const int stride = gridDim.x * blockDim.x;
  for (int base = blockIdx.x * blockDim.x; base < next; base += stride) {
    const int m = base + threadIdx.x;
    bool h1 = false, h2 = false;
    if (m < next) {
      const int row = first[m];
      if (row != kInf) {
        h1 = true;
        first[m] = kInf;
        if (fix) {
          // split: lower the false maximum, entry 0 of the winning
          // decompressed row (:3326-3344); join: lower the true minimum
          // itself (:3375-3391).
          const int target = kMax ? drow[2ll * row] : ext_list[m];
          propose(J, target, step_delta(J, target));
        }
      }
      if (flag[m]) {
        h2 = true;
        flag[m] = 0;
        if (fix) {
          if (kMax) {
            // lower the true maximum (:3346-3364)
            propose(J, ext_list[m], step_delta(J, ext_list[m]));
          }
        }
      }
    }
    const unsigned mask = 0xffffffffu;
    const unsigned b1 = __ballot_sync(mask, h1), b2 = __ballot_sync(mask, h2);
    if (lane_id() == 0) {
      if (b1) atomicAdd(c1, __popc(b1));
      if (b2) atomicAdd(c2, __popc(b2));
    }
  }
  }
}

// get_wrong_index_min direction 1 (:3157-3168, fix :3393-3410) keeps the pair of
// the lowest row per minimum and lowers the row's FALSE last entry, so it needs
// the winning row: one more scan, arbitrating through ext_id (the setup's
// scratch, left at kInf; first_sj keeps the wrong-saddle results between
// scans).
template <class T>
__global__ void __launch_bounds__(256) k_wim_min2_scan(const Job<T>* __restrict__ jobs, const __grid_constant__ Sel sel) {
  for (int jk = 0; jk < sel.n; ++jk) {
  const Job<T>& J = jobs[sel.idx[jk]];
  const int ns = J.ctr[C_NS1];
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += stride) {
    const int cnt = J.ocnt1[i];
    if (cnt == 0) continue;
    const int4 o = J.oend1[i];
    if (o.y != J.drow1[2ll * i + 1]) atomicMin(J.ext_id + o.w, i);
  }
  }
}
template <class T>
__global__ void __launch_bounds__(256) k_wim_min2_collect(const Job<T>* __restrict__ jobs, const __grid_constant__ Sel sel) {
  for (int jk = 0; jk < sel.n; ++jk) {
  const Job<T>& J = jobs[sel.idx[jk]];
  const int next = J.ctr[C_NMIN];
  const int stride = gridDim.x * blockDim.x;
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < next; m += stride) {
    const int row = J.ext_id[m];
    if (row == kInf) continue;
    J.ext_id[m] = kInf;
    const int target = J.drow1[2ll * row + 1];
    propose(J, target, step_delta(J, target));
  }
  }
}

// ---------------------------------------------------------------------------
// saddle_loops (:4229-4243) / saddle_loops_join (:4245-4261):
// get_wrong_index_saddles(_join) (:3173-3270) -- the first saddle in an
// extremum's CSR list (row order, then entry order) that outranks the true
// largest (smallest) saddle in the decompressed field -- and
// fix_wrong_index_saddle (:3415-3463).
// ---------------------------------------------------------------------------
// The scan is incremental.  An extremum's result -- its first row entry
// (i * kRowStride + p, row order then entry order) whose saddle outranks the
// extremum's true largest (smallest) saddle in the decompressed field, or kInf
// -- depends only on the values of the saddles whose rows name it, and the true
// largest saddle is one of them.  So after the first scan of a correction
// (epoch 1: every extremum) only the extrema named in the rows of saddles whose
// value changed since the previous scan are recomputed, each from its list of
// row entries (moff / ment, built at setup); the others keep their result.
// k_apply marks changed values in wchg2 / wchg1, one bitset per side.

// Row index of vertex v on the side (its index in sad2 / sad1), or -1: a
// binary search among the list entries of v's 1024-id block (cpoff).
template <class T, bool kMax>
__device__ __forceinline__ int side_row(const Job<T>& J, int v) {
  const int t = J.otype[v];
  if (!(kMax ? (t == 2 || t == 3) : (t == 1 || t == 3))) return -1;
  const int nb = (J.dim.N + kCpBlock - 1) / kCpBlock, b = v / kCpBlock;
  const int* off = J.cpoff + (kMax ? 0 : nb);
  const int* sad = kMax ? J.sad2 : J.sad1;
  int lo = off[b], hi = (b + 1 < nb ? off[b + 1] : J.ctr[kMax ? C_NS2 : C_NS1]) - 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (sad[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Queues the extrema named in the rows of the saddles whose value changed
// (and clears the bitset).  In epoch 1 every extremum is recomputed, so the
// bitset is only cleared.
template <class T, bool kMax>
__global__ void __launch_bounds__(256) k_wis_mark(const Job<T>* __restrict__ jobs,
                                                  const __grid_constant__ Sel sel) {
  for (int jk = 0; jk < sel.n; ++jk) {
    const Job<T>& J = jobs[sel.idx[jk]];
    const int epoch = J.ctr[kMax ? C_WEP2 : C_WEP1];
    unsigned* chg = kMax ? J.wchg2 : J.wchg1;
    const uint8_t* ocnt = kMax ? J.ocnt2 : J.ocnt1;
    const int4* orm = kMax ? J.orm2 : J.orm1;
    const int* rows = kMax ? J.orow2 : J.orow1;
    int* stamp = kMax ? J.wstamp2 : J.wstamp1;
    const int nw = (J.dim.N + 31) >> 5;
    const int stride = gridDim.x * blockDim.x;
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += stride) {
      unsigned bits = chg[w];
      if (!bits) continue;
      chg[w] = 0u;
      if (epoch == 1) continue;
      for (; bits; bits &= bits - 1) {
        const int i = side_row<T, kMax>(J, (w << 5) + __ffs(bits) - 1);
        if (i < 0) continue;
        const int cnt = ocnt[i];
        const int4 m4 = orm[i];
        for (int p = 0; p < cnt; ++p) {
          const int m = p == 0 ? m4.x : p == 1 ? m4.y : p == 2 ? m4.z : p == 3 ? m4.w
                                                               : rows[(long long)i * kRowStride + p];
          if (m < 0) continue;  // a repeated label
          if (atomicExch(stamp + m, epoch) != epoch) J.aff[atomicAdd(J.ctr + C_AFF, 1)] = m;
        }
      }
    }
  }
}

// The first entry among ent[k0 + i * step], i >= 0, below k1 whose saddle
// outranks extremum saddle tb (value gt), or kInf.  Four entries at a time:
// their three dependent loads (entry, saddle, value) go out together.
template <class T, bool kMax>
__device__ __forceinline__ int wis_first(const Job<T>& J, const int* sad, const int* ent, int k0,
                                         int k1, int step, int tb, T gt) {
  int hit = kInf;
  for (int k = k0; k < k1; k += 4 * step) {
    int key[4], s[4];
    T gs[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) key[j] = k + j * step < k1 ? ent[k + j * step] : -1;
#pragma unroll
    for (int j = 0; j < 4; ++j) s[j] = key[j] >= 0 ? sad[key[j] / kRowStride] : 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) gs[j] = key[j] >= 0 ? J.g[s[j]] : T(0);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const bool wrong = kMax ? (gs[j] > gt || (gs[j] == gt && s[j] > tb))
                              : (gs[j] < gt || (gs[j] == gt && s[j] < tb));
      if (key[j] >= 0 && wrong && key[j] < hit) hit = key[j];
    }
  }
  return hit;
}

// Recomputes the queued extrema (every extremum in epoch 1) from their row
// entries, a thread per extremum; an extremum with more than kWisShort
// entries goes to the long queue (wlong) for a block of its own
// (k_wis_long), so that one long list does not hold up the launch.
constexpr int kWisShort = 48;
template <class T, bool kMax>
__global__ void __launch_bounds__(256) k_wis_update(const Job<T>* __restrict__ jobs,
                                                    const __grid_constant__ Sel sel) {
  for (int jk = 0; jk < sel.n; ++jk) {
    const Job<T>& J = jobs[sel.idx[jk]];
    const bool all = J.ctr[kMax ? C_WEP2 : C_WEP1] == 1;
    const int n = all ? J.ctr[kMax ? C_NMAX : C_NMIN] : J.ctr[C_AFF];
    const int* sad = kMax ? J.sad2 : J.sad1;
    const int* best = kMax ? J.largest : J.smallest;
    const int* off = kMax ? J.moff2 : J.moff1;
    const int* ent = kMax ? J.ment2 : J.ment1;
    int* first = kMax ? J.first_s : J.first_sj;
    const int N = J.dim.N;
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x; base < n; base += stride) {  // uniform per warp
      const int e = base + threadIdx.x;
      bool lng = false;
      int m = 0;
      if (e < n) {
        m = all ? e : J.aff[e];
        const int tb = best[m];
        const int k0 = off[m], k1 = off[m + 1];
        lng = k1 - k0 > kWisShort;
        // An extremum named by no row has no saddle.
        if (!lng)
          first[m] = (tb >= 0 && tb < N) ? wis_first<T, kMax>(J, sad, ent, k0, k1, 1, tb, J.g[tb])
                                         : kInf;
      }
      const int slot = warp_append(J.ctr + C_WLONG, lng, 0xffffffffu);
      if (slot >= 0) J.wlong[slot] = m;
    }
  }
}

// The long lists of k_wis_update, a block per extremum.
template <class T, bool kMax>
__global__ void __launch_bounds__(256) k_wis_long(const Job<T>* __restrict__ jobs,
                                                  const __grid_constant__ Sel sel) {
  __shared__ int part[8];
  for (int jk = 0; jk < sel.n; ++jk) {
    const Job<T>& J = jobs[sel.idx[jk]];
    const int n = J.ctr[C_WLONG];
    const int* sad = kMax ? J.sad2 : J.sad1;
    const int* ent = kMax ? J.ment2 : J.ment1;
    const int* off = kMax ? J.moff2 : J.moff1;
    for (int e = blockIdx.x; e < n; e += gridDim.x) {  // uniform per block
      const int m = J.wlong[e];
      const int tb = (kMax ? J.largest : J.smallest)[m];  // valid: the lists are non-empty
      int hit = wis_first<T, kMax>(J, sad, ent, off[m] + (int)threadIdx.x, off[m + 1], 256, tb,
                                   J.g[tb]);
      for (int o = 16; o > 0; o >>= 1) hit = min(hit, __shfl_xor_sync(0xffffffffu, hit, o));
      if (lane_id() == 0) part[threadIdx.x >> 5] = hit;
      __syncthreads();
      if (threadIdx.x == 0) {
        for (int w = 1; w < 8; ++w) hit = min(hit, part[w]);
        (kMax ? J.first_s : J.first_sj)[m] = hit;
      }
      __syncthreads();
    }
  }
}

template <class T, bool kMax>
__global__ void __launch_bounds__(256) k_wis_collect(const Job<T>* __restrict__ jobs, const __grid_constant__ Sel sel, int fix) {
  for (int jk = 0; jk < sel.n; ++jk) {
  const Job<T>& J = jobs[sel.idx[jk]];
  const int next = J.ctr[kMax ? C_NMAX : C_NMIN];
  const int* sad = kMax ? J.sad2 : J.sad1;
  const int* best = kMax ? J.largest : J.smallest;
  int* first = kMax ? J.first_s : J.first_sj;
  int* cnt = J.ctr + (kMax ? C_WSC : C_WSCJ);
  const int stride = gridDim.x * blockDim.x;
  for (int base = blockIdx.x * blockDim.x; base < next; base += stride) {
    const int m = base + threadIdx.x;
    bool hit = false;
    if (m < next && first[m] != kInf) {  // kept: the scan is incremental
      hit = true;
      const int s = sad[first[m] / kRowStride];
      const int t = best[m];
      if (fix) {
        const T gt = J.g[t], gs = J.g[s];
        if (kMax) {
          if (!(gt > gs || (gt == gs && t > s))) propose(J, s, step_delta(J, s));
        } else if (!(gt < gs || (gt == gs && t < s))) {
          // store -bound/q, then (edit_type 1) atomic max with the midpoint:
          // max(-bound/q, midpoint) whatever the interleaving (:3447-3458).
          propose(J, t, -J.bound / T(J.q));
          if (J.edit_type == 1) propose(J, t, midpoint_delta(J, t));
        }
      }
    }
    const unsigned b = __ballot_sync(0xffffffffu, hit);
    if (lane_id() == 0 && b) atomicAdd(cnt, __popc(b));
  }
  }
}

// ---------------------------------------------------------------------------
// Small helpers.
// ---------------------------------------------------------------------------
// Per-job control operations between kernels, one thread per selected job
// (counter resets, epoch advances and list swaps; the job descriptors live in
// device memory, so list swaps happen here too).
enum CtlOp : int {
  OP_DETECT_DENSE_BEGIN = 0,  // mismatch list and category counts to zero
  OP_DETECT_BEGIN,            // next re-evaluation epoch, next list and counts to zero
  OP_DETECT_END_DENSE,        // dirty list to zero, next dirty epoch
  OP_DETECT_END,              // swap mismatch lists, then as OP_DETECT_END_DENSE
  OP_MF_BEGIN,                // start of a manifold round: skip it if nothing changed,
                              // else next flag stamp, flagged / candidate counts to zero
  OP_ZERO_TOUCHED,
  OP_SLOOPS_BEGIN,            // wrong_max counters and touched to zero
  OP_SADDLE_BEGIN,            // wrong_saddle counter and touched to zero
  OP_SLOOPS_JOIN_BEGIN,
  OP_SADDLE_JOIN_BEGIN,
  OP_DETECT3_BEGIN,           // wrong_max / wrong_saddle counters to zero
  OP_DETECT3_JOIN_BEGIN
};

template <class T>
__global__ void k_ctl(Job<T>* jobs, const __grid_constant__ Sel sel, int op) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= sel.n) return;
  Job<T>& J = jobs[sel.idx[k]];
  int* c = J.ctr;
  switch (op) {
    case OP_DETECT_DENSE_BEGIN:
      c[C_MM] = c[C_CMAX] = c[C_CMIN] = c[C_CSAD] = 0;
      break;
    case OP_DETECT_BEGIN:
      c[C_REPOCH] += 1;
      c[C_MM_NEXT] = c[C_CMAX] = c[C_CMIN] = c[C_CSAD] = 0;
      break;
    case OP_DETECT_END: {
      int* t = J.mm;
      J.mm = J.mm_next;
      J.mm_next = t;
      c[C_MM] = c[C_MM_NEXT];
    }  // fall through
    case OP_DETECT_END_DENSE:
      c[C_DIRTY] = 0;
      c[C_DEPOCH] += 1;
      break;
    case OP_MF_BEGIN:
      // The round's outputs (labels, row slots, flagged neighbours and their
      // counts) are functions of the decompressed field alone, so when no
      // value changed since the last round began they are still in place.
      c[C_MFSKIP] = c[C_MFDONE] && !c[C_CHANGED];
      c[C_MFREUSED] += c[C_MFSKIP];
      c[C_MFFIRST] = !c[C_MFDONE];
      c[C_CHANGED] = 0;
      c[C_MFDONE] = 1;
      if (c[C_MFSKIP]) break;
      c[C_WNSTAMP] += 1;  // next flag stamp; flagged and candidate counts to zero
      c[C_NFC] = c[C_NFC1] = 0;
      c[C_CAND] = c[C_CANDJ] = c[C_CAND_NEXT] = c[C_TLIST] = 0;
      break;
    case OP_ZERO_TOUCHED:
      c[C_TOUCHED] = 0;
      break;
    case OP_SLOOPS_BEGIN:
      c[C_WMC] = c[C_WMC2] = c[C_TOUCHED] = 0;
      break;
    case OP_SADDLE_BEGIN:
      c[C_WSC] = c[C_TOUCHED] = 0;
      c[C_WEP2] += 1;  // next wrong-saddle epoch, empty queue
      c[C_AFF] = c[C_WLONG] = 0;
      break;
    case OP_SLOOPS_JOIN_BEGIN:
      c[C_WMIN] = c[C_WMIN2] = c[C_TOUCHED] = 0;
      break;
    case OP_SADDLE_JOIN_BEGIN:
      c[C_WSCJ] = c[C_TOUCHED] = 0;
      c[C_WEP1] += 1;
      c[C_AFF] = c[C_WLONG] = 0;
      break;
    case OP_DETECT3_BEGIN:
      c[C_WMC] = c[C_WMC2] = c[C_WSC] = 0;
      c[C_WEP2] += 1;
      c[C_AFF] = c[C_WLONG] = 0;
      break;
    case OP_DETECT3_JOIN_BEGIN:
      c[C_WMIN] = c[C_WMIN2] = c[C_WSCJ] = 0;
      c[C_WEP1] += 1;
      c[C_AFF] = c[C_WLONG] = 0;
      break;
    default:
      break;
  }
}

// ---------------------------------------------------------------------------
// Small helpers.
// ---------------------------------------------------------------------------
template <class K>
__global__ void k_fill(K* p, K v, long long n) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride) p[i] = v;
}

}  // namespace extremz

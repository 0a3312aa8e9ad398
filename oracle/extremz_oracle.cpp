// ExtreM correction oracle -- TEST INFRASTRUCTURE ONLY.
//
// A single-threaded CPU restatement of the reference GPU correction
// (src/ExtreM_cuda.cu, main() at :4954-6078 and the kernels it launches).  It
// is the checker for this repository's CUDA path: only tests, the smoke check
// and the CPU-baseline leg of bench.py load it.  The product never links it.
//
// Canonical order.  Three sites of the reference GPU path are racy; this
// restatement resolves them sequentially, which the CUDA path reproduces:
//   * ExtractCP (:1694-1741) appends with atomicAdd; here every CP list is in
//     ascending vertex id, which fixes the triplet row order and the
//     max->saddle CSR order (:4806-4888).
//   * get_wrong_split_neighbors / get_wrong_join_neighbors (:2400-2513) flag a
//     neighbour with check-then-set from concurrent threads; here by default
//     in lockstep order (every saddle examines its j-th neighbour at step j,
//     so a shared neighbour goes to the saddle meeting it at the earlier
//     step: the reference's own outcome on the fields its runs were pinned
//     on), or with saddles visited sequentially in ascending id.
//   * get_wrong_index_max / _min (:3113-3171) keep one (true, false) pair per
//     extremum with check-then-set; here the lowest saddle row wins.
// The stale read in get_wrong_index_max (:3128-3130: the decompressed row is
// read at the ORIGINAL row's last position even when the decompressed row is
// shorter) is reproduced by keeping decompressed rows persistent across
// rounds, zero-initialised, and rewriting only [0, count) each time, exactly as
// the reference's findAscPaths/findDescPaths do (:1892-1918, :2026-2047).
//
// Manifold labels are full roots for every vertex.  The reference jumps
// descending labels only next to original 2-saddles (:1514-1557) but every
// consumer reads labels only there, so consumed values are identical.
//
// Arithmetic follows the reference operation by operation in the field type T
// (double as in the reference; float keeps data, bound and deltas in float as
// the reference's float variant does, src/ExtreM_cuda_f.cu:124).  Build with
// -ffp-contract=off so that no multiply-add is fused.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <type_traits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// The 14 Freudenthal directions in the reference's order
// (src/ExtreM_cuda.cu:155-162, src/ExtreM.cpp:16-21).  Star lists and LUT bit
// positions follow this order.
const int kDir[14][3] = {
    {1, 0, 0},  {-1, 0, 0}, {0, 1, 0},  {0, -1, 0}, {0, 0, 1},
    {0, 0, -1}, {-1, 1, 0}, {1, -1, 0}, {0, 1, 1},  {0, -1, -1},
    {-1, 0, 1}, {1, 0, -1}, {-1, 1, 1}, {1, -1, -1}};

constexpr int kLutSize = 24800;
constexpr int kNumKeys = 27;

// ---------------------------------------------------------------------------
// Lookup table (src/ExtreM_cuda.cu:263-467 calculateLUT, :3280-3318
// generateLookupTable, :84-113 keys/lutOffsets, :5233-5266 representatives).
// ---------------------------------------------------------------------------
struct Lut {
  int8_t table[kLutSize];
  int key_mask[kNumKeys];
  int offset[kNumKeys];
  int16_t key_of_valid[1 << 14];  // valid-direction mask -> key index or -1
};

bool is_direction(int dx, int dy, int dz) {
  for (int d = 0; d < 14; ++d)
    if (kDir[d][0] == dx && kDir[d][1] == dy && kDir[d][2] == dz) return true;
  return false;
}

int count_components(const std::vector<int>& nodes, const int adj[14][14]) {
  int n = (int)nodes.size();
  std::vector<int> seen(n, 0);
  int comps = 0;
  for (int s = 0; s < n; ++s) {
    if (seen[s]) continue;
    ++comps;
    std::vector<int> stack{s};
    seen[s] = 1;
    while (!stack.empty()) {
      int u = stack.back();
      stack.pop_back();
      for (int t = 0; t < n; ++t)
        if (!seen[t] && adj[nodes[u]][nodes[t]]) {
          seen[t] = 1;
          stack.push_back(t);
        }
    }
  }
  return comps;
}

void build_lut(Lut& L) {
  // Boundary classes: each axis is low (0), interior (1) or high (3) in a
  // 4x4x4 grid.  Keys are grouped by neighbour count, then ordered by the
  // representative vertex id -- the layout of the reference's LUT.bin.
  struct Rep { int id, mask, count; };
  std::vector<Rep> reps;
  const int cls[3] = {0, 1, 3};
  for (int cz : cls)
    for (int cy : cls)
      for (int cx : cls) {
        int mask = 0;
        for (int d = 0; d < 14; ++d) {
          int nx = cx + kDir[d][0], ny = cy + kDir[d][1], nz = cz + kDir[d][2];
          if (nx >= 0 && nx < 4 && ny >= 0 && ny < 4 && nz >= 0 && nz < 4) mask |= 1 << d;
        }
        reps.push_back({cx + 4 * cy + 16 * cz, mask, __builtin_popcount(mask)});
      }
  std::sort(reps.begin(), reps.end(), [](const Rep& a, const Rep& b) {
    return a.count != b.count ? a.count < b.count : a.id < b.id;
  });
  int adj[14][14];
  for (int a = 0; a < 14; ++a)
    for (int b = 0; b < 14; ++b)
      adj[a][b] = a != b && is_direction(kDir[b][0] - kDir[a][0], kDir[b][1] - kDir[a][1],
                                         kDir[b][2] - kDir[a][2]);
  for (int i = 0; i < (1 << 14); ++i) L.key_of_valid[i] = -1;
  std::memset(L.table, 0, sizeof(L.table));
  int off = 0;
  for (int k = 0; k < kNumKeys; ++k) {
    const Rep& r = reps[k];
    L.key_mask[k] = r.mask;
    L.offset[k] = off;
    L.key_of_valid[r.mask] = (int16_t)k;
    std::vector<int> valid;
    for (int d = 0; d < 14; ++d)
      if (r.mask >> d & 1) valid.push_back(d);
    int n = (int)valid.size();
    for (int cfg = 0; cfg < (1 << n); ++cfg) {
      std::vector<int> lower, upper;
      for (int j = 0; j < n; ++j) ((cfg >> j & 1) ? upper : lower).push_back(valid[j]);
      int lc = count_components(lower, adj), uc = count_components(upper, adj);
      int t = 0;  // lc == uc == 0 cannot occur (>= 4 valid neighbours)
      if (lc == 0 && uc == 1) t = 0;
      else if (lc == 1 && uc == 0) t = 4;
      else if (lc == 1 && uc == 1) t = 5;
      else if (lc > 1 && uc > 1) t = 3;
      else if (lc > 1) t = 1;
      else if (uc > 1) t = 2;
      L.table[off + cfg] = (int8_t)t;
    }
    off += 1 << n;
  }
}

const Lut& lut() {
  static Lut* L = [] {
    Lut* p = new Lut;
    build_lut(*p);
    return p;
  }();
  return *L;
}

// ---------------------------------------------------------------------------
// Grid and total order.
// ---------------------------------------------------------------------------
struct Grid {
  int W, H, D, N;
  // Valid neighbours of v in direction order; returns the count.  dirs (if
  // given) receives the direction index of each.
  int nbrs(int v, int* out, int* dirs = nullptr) const {
    int x = v % W, y = (v / W) % H, z = (v / (W * H)) % D;
    int k = 0;
    for (int d = 0; d < 14; ++d) {
      int nx = x + kDir[d][0], ny = y + kDir[d][1], nz = z + kDir[d][2];
      if (nx < 0 || nx >= W || ny < 0 || ny >= H || nz < 0 || nz >= D) continue;
      if (dirs) dirs[k] = d;
      out[k++] = nx + (ny + nz * H) * W;
    }
    return k;
  }
};

// u above v in the total order (value, then id): islarger (:1779-1781).
template <class T>
inline bool above(const T* a, int u, int v) {
  return a[u] > a[v] || (a[u] == a[v] && u > v);
}
// u below v: isless (:1787-1789).
template <class T>
inline bool below(const T* a, int u, int v) {
  return a[u] < a[v] || (a[u] == a[v] && u < v);
}

// classifyVertex_CUDA (:3720-3911): type of v and its lower-star mask (bit d
// set when the neighbour in direction d exists and is below v).
template <class T>
int classify(const T* a, const Grid& g, int v, uint16_t* lmask_out) {
  const Lut& L = lut();
  int x = v % g.W, y = (v / g.W) % g.H, z = (v / (g.W * g.H)) % g.D;
  int valid = 0, lmask = 0, upbits = 0, k = 0, lower = 0, upper = 0;
  T c = a[v];
  for (int d = 0; d < 14; ++d) {
    int nx = x + kDir[d][0], ny = y + kDir[d][1], nz = z + kDir[d][2];
    if (nx < 0 || nx >= g.W || ny < 0 || ny >= g.H || nz < 0 || nz >= g.D) continue;
    int r = nx + (ny + nz * g.H) * g.W;
    T nv = a[r];
    if (nv < c || (nv == c && r < v)) {
      lmask |= 1 << d;
      ++lower;
    } else if (nv > c || (nv == c && r > v)) {
      upbits |= 1 << k;
      ++upper;
    }
    valid |= 1 << d;
    ++k;
  }
  if (lmask_out) *lmask_out = (uint16_t)lmask;
  if (upper == 0) return 4;
  if (lower == 0) return 0;
  int key = L.key_of_valid[valid];
  if (key < 0) return -1;
  return L.table[L.offset[key] + upbits];
}

// ComputeDirection + pointer jumping (:1464-1611): full roots of the steepest
// ascent (ds) and descent (as) graphs.
template <class T>
void roots(const T* a, const Grid& g, int* ds, int* as) {
#pragma omp parallel for schedule(static)
  for (int v = 0; v < g.N; ++v) {
    int nb[14];
    int hi = v, lo = v;
    int n = g.nbrs(v, nb);
    for (int j = 0; j < n; ++j) {
      int r = nb[j];
      if (a[hi] < a[r] || (a[hi] == a[r] && hi < r)) hi = r;
      if (a[lo] > a[r] || (a[lo] == a[r] && lo > r)) lo = r;
    }
    ds[v] = hi;
    as[v] = lo;
  }
  // Synchronous pointer doubling until every label is a root.
  std::vector<int> tmp(g.N);
  for (int* m : {ds, as}) {
    for (;;) {
      int changed = 0;
#pragma omp parallel for schedule(static) reduction(| : changed)
      for (int v = 0; v < g.N; ++v) {
        int w = m[m[v]];
        tmp[v] = w;
        changed |= (w != m[v]);
      }
      std::memcpy(m, tmp.data(), sizeof(int) * (size_t)g.N);
      if (!changed) break;
    }
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Parameters, report and trace (mirrored by tests/oracle_ffi.py).
// ---------------------------------------------------------------------------
extern "C" {
struct oracle_params {
  double bound;          // absolute error bound (cast to T)
  double thr;            // persistence filter thr = sim * range (:231)
  int q;                 // step divisor / counter threshold (:4962, :5015)
  int edit_type;         // 0: fixed step with counter; 1: midpoint (:4963)
  int max_outer;         // cap on outer iterations (the reference has none)
  int max_cloop_rounds;  // cap on rounds of one c_loops call
  int final_join;        // run the final saddle_loops_join (:5997)
  int preserve_join;     // preserve_join_tree (:4969, false in the reference)
  int wn_lag;            // wrong-neighbour flagging: k >= 0 the lockstep model of
                         // the reference's concurrent launch (0: the default, see
                         // wrong_neighbors_lockstep); < 0 ascending saddle id,
                         // sequentially
};
struct oracle_report {
  int status;        // 0 ok, 1 round cap hit
  int outer_iters;
  int cloop_rounds;  // total c_loops correction rounds
  int manifold_rounds;
  long long edited;  // voxels whose value differs from the input decp
  int counters[11];  // final host counters (order of the loop test :5603)
};
struct oracle_edit_report {
  long long index_bytes;  // bytes of the index stream
  long long edit_bytes;   // bytes of the edit stream
  long long edited;       // voxels whose value changed
  long long n_edits;      // entries of the edit stream
  double psnr_before;     // PSNR of the decompressed field against the original
  double psnr_after;      // PSNR of the corrected field
};
}

namespace {

enum Phase : int {
  PH_CLOOP_DETECT = 1,  // counts: max, min, saddle
  PH_WRONG_NBR = 2,     // nfc, nfc1
  PH_SLOOPS = 3,        // wmc, wmc2
  PH_SADDLE = 4,        // wsc
  PH_DETECT3 = 5,       // wsc, wmc, wmc2
  PH_SLOOPS_JOIN = 6,   // wmin, wmin2
  PH_SADDLE_JOIN = 7,   // wscj
  PH_OUTER = 8,         // 11 counters
  PH_CHECKSUM = 9,      // running value checksum after a phase (lo, hi)
};

template <class T>
struct Corrector {
  Grid g;
  const T* f;
  T* a;  // decompressed field, corrected in place
  T bound, thr;
  int q, edit_type;
  int wn_lag = 0;
  T sentinel;

  std::vector<int8_t> otype;
  std::vector<uint16_t> olmask;
  std::vector<int> DS, AS, dDS, dAS;
  std::vector<int> sad2, sad1, maxima, minima, ext_index;
  // Rows of 14 labels + count.
  std::vector<int> orow2, orow1, drow2, drow1;
  std::vector<int> max_off, max_sad, min_off, min_sad;
  std::vector<int> largest, smallest;

  std::vector<T> delta;
  std::vector<int> touched;
  std::vector<int> counter;

  std::vector<int> lmax, lmin, lsad;
  std::vector<uint8_t> wn_ds, wn_as, wr_max, wr_max2, wr_min, wr_min2;
  std::vector<int> wn_ds_list, wn_as_list;
  std::vector<int> pmax1, pmax2, pmin1, pmin2, psad, psadj;

  // Device-side counters of the reference (:133, :150-152).
  int d_nfc = 0, d_nfc1 = 0, d_cfmax = 0, d_cfmin = 0, d_cfsad = 0;
  int d_wmc = 0, d_wmc2 = 0, d_wsc = 0, d_wmin = 0, d_wmin2 = 0, d_wscj = 0;
  // File-scope host copies (:62): s_loops, saddle_loops and their join
  // variants refresh them as a side effect (:3473-3476, :4236, :3498-3501,
  // :4252); c_loops and r_loops take counters by value and refresh nothing.
  int h_wmc = 0, h_wmc2 = 0, h_wsc = 0, h_wmin = 0, h_wmin2 = 0, h_wscj = 0;

  int cloop_rounds = 0, manifold_rounds = 0, max_cloop_rounds = 0;
  bool capped = false;
  int* trace;
  int trace_cap, trace_len = 0;

  static constexpr int kRow = 15;  // 14 labels + count

  void emit(int phase, int c0 = 0, int c1 = 0, int c2 = 0) {
    if (!trace || trace_len + 4 > trace_cap) return;
    trace[trace_len++] = phase;
    trace[trace_len++] = c0;
    trace[trace_len++] = c1;
    trace[trace_len++] = c2;
  }

  void amax(int i, T d) {
    if (delta[i] == sentinel) touched.push_back(i);
    if (d > delta[i]) delta[i] = d;
  }

  T midpoint_delta(int i) const {  // e.g. :2906, :3334-3337, :3433
    return ((f[i] - bound) + a[i]) / T(2) - a[i];
  }
  T step_delta(int i) const { return edit_type == 1 ? midpoint_delta(i) : -bound / T(q); }

  void init_delta() {  // init_delta (:2569-2577), sparse form
    for (int i : touched) delta[i] = sentinel;
    touched.clear();
  }

  // applyDeltaBuffer (:3061-3111).
  void apply() {
    std::sort(touched.begin(), touched.end());
    for (int i : touched) {
      T d = delta[i];
      if (d == sentinel) continue;
      if (edit_type == 0) {
        if (counter[i] < q - 1 && std::fabs(f[i] - (a[i] + d)) <= bound) {
          a[i] += d;
          counter[i] += 1;
        } else {
          counter[i] = q;
          a[i] = f[i] - bound;
        }
      } else {
        if (std::fabs(f[i] - (a[i] + d)) <= bound) a[i] += d;
        else a[i] = f[i] - bound;
      }
    }
  }

  // classifyVertex_CUDA(type=1) fused detection (:3856-3910).  Threads take
  // contiguous ranges and their lists are joined in order, so the lists are in
  // ascending id whatever the thread count.
  void detect() {
    lmax.clear();
    lmin.clear();
    lsad.clear();
    int nt = 1;
#ifdef _OPENMP
    nt = omp_get_max_threads();
#endif
    std::vector<std::vector<int>> pmax(nt), pmin(nt), psad_(nt);
#pragma omp parallel num_threads(nt)
    {
      int t = 0;
#ifdef _OPENMP
      t = omp_get_thread_num();
#endif
      long long lo = (long long)g.N * t / nt, hi = (long long)g.N * (t + 1) / nt;
      for (int v = (int)lo; v < (int)hi; ++v) {
        uint16_t lm;
        int ty = classify(a, g, v, &lm);
        int o = otype[v];
        if (ty != o) {
          if ((ty == 4) != (o == 4)) pmax[t].push_back(v);
          if ((ty == 0) != (o == 0)) pmin[t].push_back(v);
          if ((ty == 2) != (o == 2) || (ty == 1) != (o == 1) || (ty == 3) != (o == 3))
            psad_[t].push_back(v);
        } else if (ty == 1 || ty == 2 || ty == 3) {
          if (lm != olmask[v]) psad_[t].push_back(v);  // areVectorsDifferent_local (:909-921)
        }
      }
    }
    for (int t = 0; t < nt; ++t) {
      lmax.insert(lmax.end(), pmax[t].begin(), pmax[t].end());
      lmin.insert(lmin.end(), pmin[t].begin(), pmin[t].end());
      lsad.insert(lsad.end(), psad_[t].begin(), psad_[t].end());
    }
    d_cfmax = (int)lmax.size();
    d_cfmin = (int)lmin.size();
    d_cfsad = (int)lsad.size();
    emit(PH_CLOOP_DETECT, d_cfmax, d_cfmin, d_cfsad);
  }

  // c_loop(0) (:2890-2963).
  void propose_max(int v) {
    if (otype[v] != 4) {
      amax(v, step_delta(v));
      return;
    }
    int nb[14];
    int n = g.nbrs(v, nb);
    int L = v;
    for (int j = 0; j < n; ++j)
      if (above(a, nb[j], L)) L = nb[j];
    if (L == v) return;
    amax(L, step_delta(L));
  }

  // c_loop(1) (:2965-3039).
  void propose_min(int v) {
    if (otype[v] != 0) {
      int nb[14];
      int n = g.nbrs(v, nb);
      int S = v;
      for (int j = 0; j < n; ++j)
        if (below(f, nb[j], S)) S = nb[j];
      T d = edit_type == 1 ? ((f[S] - bound) + a[S]) / T(2) - a[S] : -bound / T(q);
      if (a[v] > a[S] || (a[v] == a[S] && v > S)) return;
      amax(S, d);
      return;
    }
    amax(v, step_delta(v));
  }

  // c_loop(2) -> fix_saddle_local (:2804-2884).
  void propose_saddle(int v) {
    int nb[14], dirs[14];
    int n = g.nbrs(v, nb, dirs);
    int dmask = 0;
    for (int j = 0; j < n; ++j)
      if (a[nb[j]] < a[v] || (a[nb[j]] == a[v] && nb[j] < v)) dmask |= 1 << dirs[j];
    int om = olmask[v];
    for (int j = 0; j < n; ++j)
      if ((om >> dirs[j] & 1) && !(dmask >> dirs[j] & 1)) amax(nb[j], step_delta(nb[j]));
    if (dmask & ~om) amax(v, step_delta(v));
  }

  // c_loops host driver (:3913-4044).
  void c_loops() {
    init_delta();
    detect();
    int rounds = 0;
    while (!lmax.empty() || !lmin.empty() || !lsad.empty()) {
      if (rounds >= max_cloop_rounds) {
        capped = true;
        return;
      }
      ++rounds;
      ++cloop_rounds;
      init_delta();
      for (int v : lmin) propose_min(v);
      for (int v : lsad) propose_saddle(v);
      for (int v : lmax) propose_max(v);
      apply();
      detect();
    }
  }

  // Row of a 2-saddle (findAscPaths :1832-1926) or 1-saddle (findDescPaths
  // :1956-2049) into row[0..14].
  void asc_row(const T* val, const int* dsm, int s, int* row) const {
    int nb[14], cnt = 0;
    int n = g.nbrs(s, nb);
    T sv = val[s];
    for (int j = 0; j < n; ++j) {
      int r = nb[j];
      int m = dsm[r];
      if (above(val, r, s) && std::fabs(val[m] - sv) >= thr) row[cnt++] = m;
    }
    // insertionSort (:1795-1811): descending in the total order.
    for (int i = 1; i < cnt; ++i) {
      int key = row[i], j = i - 1;
      while (j >= 0 && below(val, row[j], key)) {
        row[j + 1] = row[j];
        --j;
      }
      row[j + 1] = key;
    }
    row[14] = cnt;
  }
  void desc_row(const T* val, const int* asm_, int s, int* row) const {
    int nb[14], cnt = 0;
    int n = g.nbrs(s, nb);
    for (int j = 0; j < n; ++j) {
      int r = nb[j];
      if (below(val, r, s)) row[cnt++] = asm_[r];
    }
    // reversed_insertionSort (:1813-1829): ascending.
    for (int i = 1; i < cnt; ++i) {
      int key = row[i], j = i - 1;
      while (j >= 0 && above(val, row[j], key)) {
        row[j + 1] = row[j];
        --j;
      }
      row[j + 1] = key;
    }
    row[14] = cnt;
  }

  // Decompressed rows: only [0, count) and the count are rewritten.
  void dec_rows() {
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)sad2.size(); ++i) {
      int tmp[kRow];
      asc_row(a, dDS.data(), sad2[i], tmp);
      int* r = &drow2[i * kRow];
      for (int k = 0; k < tmp[14]; ++k) r[k] = tmp[k];
      r[14] = tmp[14];
    }
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)sad1.size(); ++i) {
      int tmp[kRow];
      desc_row(a, dAS.data(), sad1[i], tmp);
      int* r = &drow1[i * kRow];
      for (int k = 0; k < tmp[14]; ++k) r[k] = tmp[k];
      r[14] = tmp[14];
    }
  }

  void manifolds() {
    ++manifold_rounds;
    roots(a, g, dDS.data(), dAS.data());
    dec_rows();
  }

  // The same flagging under a lockstep model of the reference's launch, in
  // which every saddle thread examines its j-th neighbour at step j and a
  // flag set at step i is seen by reads from step i + lag + 1 on.  A saddle
  // whose candidate was flagged within the last `lag` steps flags it again
  // (a duplicate list entry) and stops, where the sequential rule would go on
  // to its next candidate: the check-then-set race of :2426-2431 / :2483-2488.
  void wrong_neighbors_lockstep(const std::vector<int>& sads, bool split,
                                std::vector<uint8_t>& flag, std::vector<int>& list, int lag) {
    std::vector<int> set_at(g.N, -1);  // step at which this launch flagged a vertex
    std::vector<uint8_t> done(sads.size(), 0);
    for (int j = 0; j < 14; ++j) {
      for (size_t i = 0; i < sads.size(); ++i) {
        if (done[i]) continue;
        const int s = sads[i];
        int x = s % g.W, y = (s / g.W) % g.H, z = s / (g.W * g.H);
        int nx = x + kDir[j][0], ny = y + kDir[j][1], nz = z + kDir[j][2];
        if (nx < 0 || nx >= g.W || ny < 0 || ny >= g.H || nz < 0 || nz >= g.D) continue;
        const int r = nx + (ny + nz * g.H) * g.W;
        const bool cand = split ? (above(a, r, s) && dDS[r] != DS[r])
                                : (below(a, r, s) && dAS[r] != AS[r]);
        if (!cand) continue;
        const bool seen = flag[r] && set_at[r] + lag + 1 <= j;
        if (seen) continue;
        if (!flag[r]) set_at[r] = j;
        flag[r] = 1;
        list.push_back(r);
        done[i] = 1;
      }
    }
  }

  // get_wrong_split_neighbors / get_wrong_join_neighbors (:2400-2513): the
  // lockstep resolution above, or saddles visited sequentially in ascending id.
  void wrong_neighbors() {
    for (int v : wn_ds_list) wn_ds[v] = 0;
    for (int v : wn_as_list) wn_as[v] = 0;
    wn_ds_list.clear();
    wn_as_list.clear();
    if (wn_lag >= 0) {
      wrong_neighbors_lockstep(sad2, true, wn_ds, wn_ds_list, wn_lag);
      wrong_neighbors_lockstep(sad1, false, wn_as, wn_as_list, wn_lag);
      d_nfc = (int)wn_ds_list.size();
      d_nfc1 = (int)wn_as_list.size();
      emit(PH_WRONG_NBR, d_nfc, d_nfc1);
      return;
    }
    int nb[14];
    for (int s : sad2) {
      int n = g.nbrs(s, nb);
      for (int j = 0; j < n; ++j) {
        int r = nb[j];
        if (above(a, r, s) && dDS[r] != DS[r] && !wn_ds[r]) {
          wn_ds[r] = 1;
          wn_ds_list.push_back(r);
          break;
        }
      }
    }
    for (int s : sad1) {
      int n = g.nbrs(s, nb);
      for (int j = 0; j < n; ++j) {
        int r = nb[j];
        if (below(a, r, s) && dAS[r] != AS[r] && !wn_as[r]) {
          wn_as[r] = 1;
          wn_as_list.push_back(r);
          break;
        }
      }
    }
    d_nfc = (int)wn_ds_list.size();
    d_nfc1 = (int)wn_as_list.size();
    emit(PH_WRONG_NBR, d_nfc, d_nfc1);
  }

  // fixpath (:4046-4206).
  void fixpath(int start, int direction) {
    int nb[14];
    int cur = start, t = -1, fl = -1;
    for (long long steps = 0; steps <= (long long)g.N; ++steps) {
      int ni = cur, nd = cur;
      int n = g.nbrs(cur, nb);
      for (int j = 0; j < n; ++j) {
        int r = nb[j];
        if (direction == 0) {
          if (f[ni] < f[r] || (f[ni] == f[r] && ni < r)) ni = r;
          if (a[nd] < a[r] || (a[nd] == a[r] && nd < r)) nd = r;
        } else {
          if (f[ni] > f[r] || (f[ni] == f[r] && ni > r)) ni = r;
          if (a[nd] > a[r] || (a[nd] == a[r] && nd > r)) nd = r;
        }
      }
      if (ni != nd) {
        t = ni;
        fl = nd;
        break;
      }
      if (ni == cur) break;
      cur = ni;
    }
    if (fl == t) return;
    int target = direction == 0 ? fl : t;
    amax(target, step_delta(target));
  }

  // r_loops (:4210-4227).
  void r_loops() {
    init_delta();
    for (int v : wn_ds_list) fixpath(v, 0);
    for (int v : wn_as_list) fixpath(v, 1);
    apply();
  }

  // get_wrong_index_max (:3113-3141).
  void wrong_index_max() {
    std::fill(wr_max.begin(), wr_max.end(), 0);
    std::fill(wr_max2.begin(), wr_max2.end(), 0);
    pmax1.clear();
    pmax2.clear();
    for (size_t i = 0; i < sad2.size(); ++i) {
      const int* o = &orow2[i * kRow];
      const int* d = &drow2[i * kRow];
      if (o[14] == 0) continue;
      if (o[0] != d[0] && !wr_max[o[0]]) {
        wr_max[o[0]] = 1;
        pmax1.push_back(o[0]);
        pmax1.push_back(d[0]);
      }
      int k = o[14] - 1;
      if (o[k] != d[k] && !wr_max2[o[k]]) {
        wr_max2[o[k]] = 1;
        pmax2.push_back(o[k]);
        pmax2.push_back(d[k]);
      }
    }
    d_wmc = (int)pmax1.size() / 2;
    d_wmc2 = (int)pmax2.size() / 2;
  }

  // get_wrong_index_min (:3143-3171).
  void wrong_index_min() {
    std::fill(wr_min.begin(), wr_min.end(), 0);
    std::fill(wr_min2.begin(), wr_min2.end(), 0);
    pmin1.clear();
    pmin2.clear();
    for (size_t i = 0; i < sad1.size(); ++i) {
      const int* o = &orow1[i * kRow];
      const int* d = &drow1[i * kRow];
      if (o[14] == 0) continue;
      if (o[0] != d[0] && !wr_min[o[0]]) {
        wr_min[o[0]] = 1;
        pmin1.push_back(o[0]);
        pmin1.push_back(d[0]);
      }
      int k = o[14] - 1;
      if (o[k] != d[k] && !wr_min2[o[k]]) {
        wr_min2[o[k]] = 1;
        pmin2.push_back(o[k]);
        pmin2.push_back(d[k]);
      }
    }
    d_wmin = (int)pmin1.size() / 2;
    d_wmin2 = (int)pmin2.size() / 2;
  }

  // s_loops (:3465-3487).
  void s_loops() {
    wrong_index_max();
    init_delta();
    h_wmc = d_wmc;
    h_wmc2 = d_wmc2;
    for (size_t p = 0; p < pmax1.size(); p += 2) {
      int fl = pmax1[p + 1];
      amax(fl, step_delta(fl));  // fix_wrong_index_max(0) (:3326-3344)
    }
    for (size_t p = 0; p < pmax2.size(); p += 2) {
      int t = pmax2[p];
      amax(t, step_delta(t));  // fix_wrong_index_max(1) (:3346-3364)
    }
    apply();
    emit(PH_SLOOPS, d_wmc, d_wmc2);
  }

  // s_loops_join (:3489-3512).
  void s_loops_join() {
    wrong_index_min();
    init_delta();
    h_wmin = d_wmin;
    h_wmin2 = d_wmin2;
    for (size_t p = 0; p < pmin1.size(); p += 2) {
      int t = pmin1[p];
      amax(t, step_delta(t));  // fix_wrong_index_min(0) (:3375-3391)
    }
    for (size_t p = 0; p < pmin2.size(); p += 2) {
      int fl = pmin2[p + 1];
      amax(fl, step_delta(fl));  // fix_wrong_index_min(1) (:3393-3410)
    }
    apply();
    emit(PH_SLOOPS_JOIN, d_wmin, d_wmin2);
  }

  // get_wrong_index_saddles (:3173-3218).
  void wrong_index_saddles() {
    psad.clear();
    for (size_t m = 0; m < maxima.size(); ++m) {
      int tl = largest[m];
      for (int i = max_off[m]; i < max_off[m + 1]; ++i) {
        int s = max_sad[i];
        if (a[s] > a[tl] || (a[s] == a[tl] && s > tl)) {
          psad.push_back(tl);
          psad.push_back(s);
          break;
        }
      }
    }
    d_wsc = (int)psad.size() / 2;
  }

  // get_wrong_index_saddles_join (:3220-3270).
  void wrong_index_saddles_join() {
    psadj.clear();
    for (size_t m = 0; m < minima.size(); ++m) {
      int ts = smallest[m];
      for (int i = min_off[m]; i < min_off[m + 1]; ++i) {
        int s = min_sad[i];
        if (a[s] < a[ts] || (a[s] == a[ts] && s < ts)) {
          psadj.push_back(ts);
          psadj.push_back(s);
          break;
        }
      }
    }
    d_wscj = (int)psadj.size() / 2;
  }

  // saddle_loops (:4229-4243).
  void saddle_loops() {
    wrong_index_saddles();
    init_delta();
    h_wsc = d_wsc;
    for (size_t p = 0; p < psad.size(); p += 2) {  // fix_wrong_index_saddle(0)
      int t = psad[p], fl = psad[p + 1];
      if (a[t] > a[fl] || (a[t] == a[fl] && t > fl)) continue;
      amax(fl, step_delta(fl));
    }
    apply();
    emit(PH_SADDLE, d_wsc);
  }

  // saddle_loops_join (:4245-4261).  fix_wrong_index_saddle(1) first stores
  // -bound/q non-atomically, then (edit_type 1) takes the atomic max with the
  // midpoint step (:3447-3458); the store-then-max sequence leaves
  // max(-bound/q, midpoint) whatever the interleaving, since every pair that
  // targets one vertex proposes the same midpoint.
  void saddle_loops_join() {
    wrong_index_saddles_join();
    init_delta();
    h_wscj = d_wscj;
    emit(PH_SADDLE_JOIN, d_wscj);
    if (d_wscj > 0) {
      for (size_t p = 0; p < psadj.size(); p += 2) {
        int t = psadj[p], fl = psadj[p + 1];
        if (a[t] < a[fl] || (a[t] == a[fl] && t < fl)) continue;
        if (delta[t] == sentinel) touched.push_back(t);
        T s = -bound / T(q);
        delta[t] = s;
        if (edit_type == 1) {
          T d = midpoint_delta(t);
          if (d > delta[t]) delta[t] = d;
        }
      }
      apply();
    }
  }

  void setup() {
    int N = g.N;
    otype.resize(N);
    olmask.resize(N);
#pragma omp parallel for schedule(static)
    for (int v = 0; v < N; ++v) otype[v] = (int8_t)classify(f, g, v, &olmask[v]);
    DS.resize(N);
    AS.resize(N);
    dDS.resize(N);
    dAS.resize(N);
    roots(f, g, DS.data(), AS.data());
    ext_index.assign(N, 0);
    for (int v = 0; v < N; ++v) {
      int t = otype[v];
      if (t == 2 || t == 3) sad2.push_back(v);
      if (t == 1 || t == 3) sad1.push_back(v);
      if (t == 4) maxima.push_back(v);
      if (t == 0) minima.push_back(v);
    }
    // computeMaxIndex then computeMinIndex share one array (:1928-1939).
    for (size_t i = 0; i < maxima.size(); ++i) ext_index[maxima[i]] = (int)i;
    for (size_t i = 0; i < minima.size(); ++i) ext_index[minima[i]] = (int)i;
    orow2.assign(sad2.size() * kRow, 0);
    orow1.assign(sad1.size() * kRow, 0);
    drow2.assign(sad2.size() * kRow, 0);
    drow1.assign(sad1.size() * kRow, 0);
    for (size_t i = 0; i < sad2.size(); ++i) asc_row(f, DS.data(), sad2[i], &orow2[i * kRow]);
    for (size_t i = 0; i < sad1.size(); ++i) desc_row(f, AS.data(), sad1[i], &orow1[i * kRow]);
    // computeMax_saddle_table / computeMin_saddle_table (:4806-4888).
    auto csr = [&](const std::vector<int>& sad, const std::vector<int>& rows, size_t next,
                   std::vector<int>& off, std::vector<int>& lst) {
      std::vector<int> cnt(next + 1, 0);
      for (size_t i = 0; i < sad.size(); ++i)
        for (int p = 0; p < rows[i * kRow + 14]; ++p) cnt[ext_index[rows[i * kRow + p]] + 1]++;
      off.assign(next + 1, 0);
      for (size_t m = 0; m < next; ++m) off[m + 1] = off[m] + cnt[m + 1];
      lst.assign(off[next], 0);
      std::vector<int> fill(off.begin(), off.end() - 1);
      for (size_t i = 0; i < sad.size(); ++i)
        for (int p = 0; p < rows[i * kRow + 14]; ++p)
          lst[fill[ext_index[rows[i * kRow + p]]]++] = sad[i];
    };
    csr(sad2, orow2, maxima.size(), max_off, max_sad);
    csr(sad1, orow1, minima.size(), min_off, min_sad);
    // findLargestSaddlePerMax / findSmallestSaddlePerMin (:4890-4940).
    largest.assign(maxima.size(), -1);
    for (size_t m = 0; m < maxima.size(); ++m) {
      int best = -1;
      for (int i = max_off[m]; i < max_off[m + 1]; ++i) {
        int s = max_sad[i];
        if (best < 0 || f[s] > f[best] || (f[s] == f[best] && s > best)) best = s;
      }
      largest[m] = best;
    }
    smallest.assign(minima.size(), -1);
    for (size_t m = 0; m < minima.size(); ++m) {
      int best = -1;
      for (int i = min_off[m]; i < min_off[m + 1]; ++i) {
        int s = min_sad[i];
        if (best < 0 || f[s] < f[best] || (f[s] == f[best] && s < best)) best = s;
      }
      smallest[m] = best;
    }
    delta.assign(N, sentinel);
    counter.assign(N, -1);
    wn_ds.assign(N, 0);
    wn_as.assign(N, 0);
    wr_max.assign(N, 0);
    wr_max2.assign(N, 0);
    wr_min.assign(N, 0);
    wr_min2.assign(N, 0);
  }

  // Order-independent value checksum (sum of mixed (bits, id) words), the same
  // on the CPU and in the CUDA trace.
  void checksum_emit() {
    uint64_t acc = 0;
    for (int v = 0; v < g.N; ++v) {
      uint64_t bits = 0;
      std::memcpy(&bits, &a[v], sizeof(T));
      uint64_t z = bits + 0x9e3779b97f4a7c15ull * (uint64_t)(v + 1);
      z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
      z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
      acc += z ^ (z >> 31);
    }
    emit(PH_CHECKSUM, (int)(acc & 0x7fffffff), (int)((acc >> 31) & 0x7fffffff));
  }

  // One "manifold block" of the outer loop: manifolds, rows, wrong neighbours.
  void manifold_block() {
    manifolds();
    wrong_neighbors();
  }

  // Mismatch census of the current decompressed field: the eleven loop-test
  // counters (order of the loop test :5603-5605) evaluated once, with no
  // edit.  The third block of the outer loop (:5872-5979) evaluates the
  // wrong-extremum and wrong-saddle counters only when the wrong-neighbour
  // counts are zero, and the join ones only with preserve_join_tree; the
  // census evaluates all of them.
  void census(int* out) {
    setup();
    detect();
    manifold_block();
    wrong_index_max();
    wrong_index_saddles();
    wrong_index_min();
    wrong_index_saddles_join();
    const int c[11] = {d_nfc, d_nfc1, d_cfmax, d_cfmin, d_cfsad, d_wmc,
                       d_wmc2, d_wsc, d_wmin, d_wmin2, d_wscj};
    std::memcpy(out, c, sizeof(c));
  }

  // main() (:5508-5997), preserve_join_tree as configured.
  int run(int max_outer, bool final_join, bool preserve_join, int* outer_out, int* counters) {
    setup();
    c_loops();
    if (capped) return 1;
    manifold_block();
    int h_nfc = d_nfc, h_nfc1 = d_nfc1;
    h_wmc = 0;  // :5562-5563
    h_wmc2 = 0;
    if (h_nfc == 0) {
      s_loops();
      h_wmc = d_wmc;  // :5570
      if (h_wmc == 0) saddle_loops();
    }
    if (h_nfc1 == 0 && preserve_join) {
      s_loops_join();
      h_wmin = d_wmin;
      if (h_wmin == 0) saddle_loops_join();
    }
    // :5589-5599: every host counter re-read.
    h_nfc = d_nfc;
    h_nfc1 = d_nfc1;
    int h_cfmax = d_cfmax, h_cfmin = d_cfmin, h_cfsad = d_cfsad;
    h_wmin = d_wmin;
    h_wmc = d_wmc;
    h_wmin2 = d_wmin2;
    h_wmc2 = d_wmc2;
    h_wsc = d_wsc;
    h_wscj = d_wscj;
    int outer = 0;
    auto any = [&] {
      return h_nfc > 0 || h_nfc1 > 0 || h_cfmax > 0 || h_cfmin > 0 || h_cfsad > 0 ||
             h_wmc > 0 || h_wmc2 > 0 || h_wsc > 0 || h_wmin > 0 || h_wmin2 > 0 || h_wscj > 0;
    };
    while (any()) {
      if (outer >= max_outer) {
        capped = true;
        break;
      }
      ++outer;
      // Block 1 (:5622-5747).
      c_loops();
      if (capped) break;
      r_loops();
      manifold_block();
      h_nfc = d_nfc;
      h_nfc1 = d_nfc1;
      if (h_nfc == 0) {
        s_loops();
        if (h_wmc == 0) saddle_loops();
      }
      if (h_nfc1 == 0 && preserve_join) {
        s_loops_join();
        h_wmin = d_wmin;
        if (h_wmin == 0) saddle_loops_join();
      }
      // Block 2 (:5749-5870).
      c_loops();
      if (capped) break;
      manifold_block();
      h_nfc = d_nfc;
      h_nfc1 = d_nfc1;
      if (h_nfc == 0) {
        s_loops();
        h_wmc = d_wmc;
        if (h_wmc == 0) saddle_loops();
      }
      if (h_nfc1 == 0 && preserve_join) {
        s_loops_join();
        h_wmin = d_wmin;
        if (h_wmin == 0) saddle_loops_join();
      }
      // Block 3 (:5872-5979): detection only.
      c_loops();
      if (capped) break;
      manifold_block();
      h_nfc = d_nfc;
      h_nfc1 = d_nfc1;
      if (h_nfc == 0) {
        wrong_index_max();
        wrong_index_saddles();
        h_wsc = d_wsc;
        h_wmc = d_wmc;
        h_wmc2 = d_wmc2;
        emit(PH_DETECT3, h_wsc, h_wmc, h_wmc2);
      }
      if (h_nfc1 == 0 && preserve_join) {
        wrong_index_min();
        wrong_index_saddles_join();
        h_wscj = d_wscj;
        h_wmin2 = d_wmin2;
        h_wmin = d_wmin;
      }
      detect();
      h_cfmax = d_cfmax;
      h_cfmin = d_cfmin;
      h_cfsad = d_cfsad;
      emit(PH_OUTER, outer);
      checksum_emit();
    }
    // Counters at loop exit (the loop test :5603-5605).
    if (counters) {
      int c[11] = {h_nfc, h_nfc1, h_cfmax, h_cfmin, h_cfsad, h_wmc,
                   h_wmc2, h_wsc, h_wmin, h_wmin2, h_wscj};
      std::memcpy(counters, c, sizeof(c));
    }
    if (!capped && final_join) saddle_loops_join();  // unconditional (:5997)
    if (outer_out) *outer_out = outer;
    return capped ? 1 : 0;
  }
};

template <class T>
int correct_t(const T* f, T* a, int W, int H, int D, const oracle_params* p, oracle_report* rep,
              int* trace, int trace_cap, int32_t* counter_out) {
  Corrector<T> c;
  c.g = {W, H, D, W * H * D};
  c.f = f;
  c.a = a;
  c.bound = (T)p->bound;
  c.thr = (T)p->thr;
  c.q = p->q;
  c.edit_type = p->edit_type;
  c.sentinel = T(-4.0) * c.bound;  // init_delta (:2572)
  c.max_cloop_rounds = p->max_cloop_rounds;
  c.wn_lag = p->wn_lag;
  c.trace = trace;
  c.trace_cap = trace_cap;
  std::vector<T> a0(a, a + c.g.N);
  int outer = 0;
  int counters[11] = {0};
  int st = c.run(p->max_outer, p->final_join != 0, p->preserve_join != 0, &outer, counters);
  if (rep) {
    rep->status = st;
    rep->outer_iters = outer;
    rep->cloop_rounds = c.cloop_rounds;
    rep->manifold_rounds = c.manifold_rounds;
    long long e = 0;
    for (int v = 0; v < c.g.N; ++v) e += std::memcmp(&a0[v], &a[v], sizeof(T)) != 0;
    rep->edited = e;
    std::memcpy(rep->counters, counters, sizeof(counters));
  }
  if (counter_out) std::memcpy(counter_out, c.counter.data(), sizeof(int) * c.g.N);
  return st;
}

// ---------------------------------------------------------------------------
// Edit stream of a correction (cost :4557-4675 for edit_type 0,
// floating_point_cost :4677-4797 for edit_type 1), without the files and
// the zstd step.  A voxel is edited when the corrected value differs from the
// decompressed one (decp_data_copy[i] != decp_data[i]).
//  * edit_type 0: index stream = every voxel's edit counter (0 when not
//    edited) packed three bits per voxel by encodeTo3BitBitmap (:4282-4312);
//    edits = the snapped voxels' (counter == q) lossless edits
//    -(decp - (input - bound)), in id order.
//  * edit_type 1: index stream = the edited voxels' ids delta-coded
//    (get_diff_index :4315-4323) as int32; edits = every edited voxel's
//    -(decp - (input - bound)), in id order.
// The reference computes the 3-bit stream but writes the first N bytes of the
// int32 counter array instead, and writes the first n bytes of the n-entry
// int32 delta array; the streams here are the ones its code computes, whole.
// PSNR follows calculateMSE / calculatePSNR (:4263-4280) with the original's
// value range.
// ---------------------------------------------------------------------------
template <class T>
int encode_t(const T* f, const T* d0, const T* d1, const int32_t* counter, long long N, double bnd,
             int q, int edit_type, uint8_t* index_out, long long index_cap, T* edits_out,
             long long edits_cap, oracle_edit_report* r) {
  const T bound = (T)bnd;
  std::vector<T> edits;
  long long edited = 0;
  std::vector<uint8_t> index;
  if (edit_type == 0) {
    std::vector<int> idx((size_t)N, 0);
    for (long long i = 0; i < N; ++i) {
      if (d0[i] != d1[i]) {
        idx[i] = counter[i];
        if (idx[i] == q) edits.push_back(-(d0[i] - (f[i] - bound)));
        ++edited;
      }
    }
    // encodeTo3BitBitmap: LSB-first, bits of a value that do not fit the
    // current byte start the next one.
    uint8_t cur = 0;
    int bit = 0;
    for (int v : idx) {
      if (v < 0 || v > 7) return -2;  // the reference returns an empty stream
      cur |= (uint8_t)(v << bit);
      bit += 3;
      if (bit >= 8) {
        index.push_back(cur);
        bit -= 8;
        cur = (uint8_t)(v >> (3 - bit));
      }
    }
    if (bit > 0) index.push_back(cur);
  } else {
    std::vector<int> ids;
    for (long long i = 0; i < N; ++i) {
      if (d0[i] != d1[i]) {
        ids.push_back((int)i);
        edits.push_back(-(d0[i] - (f[i] - bound)));
        ++edited;
      }
    }
    std::vector<int> diffs;
    if (!ids.empty()) diffs.push_back(ids[0]);
    for (size_t k = 1; k < ids.size(); ++k) diffs.push_back(ids[k] - ids[k - 1]);
    index.resize(diffs.size() * sizeof(int));
    if (!diffs.empty()) std::memcpy(index.data(), diffs.data(), index.size());
  }
  if ((long long)index.size() > index_cap || (long long)(edits.size() * sizeof(T)) > edits_cap)
    return -3;
  if (!index.empty()) std::memcpy(index_out, index.data(), index.size());
  if (!edits.empty()) std::memcpy(edits_out, edits.data(), edits.size() * sizeof(T));
  double lo = (double)f[0], hi = (double)f[0], s0 = 0.0, s1 = 0.0;
  for (long long i = 0; i < N; ++i) {
    lo = std::min(lo, (double)f[i]);
    hi = std::max(hi, (double)f[i]);
    s0 += std::pow((double)f[i] - (double)d0[i], 2);
    s1 += std::pow((double)f[i] - (double)d1[i], 2);
  }
  auto psnr = [&](double sse) {
    const double mse = sse / (double)N;
    if (mse == 0) return std::numeric_limits<double>::infinity();
    return -20.0 * std::log10(std::sqrt(mse) / (hi - lo));
  };
  r->index_bytes = (long long)index.size();
  r->edit_bytes = (long long)(edits.size() * sizeof(T));
  r->edited = edited;
  r->n_edits = (long long)edits.size();
  r->psnr_before = psnr(s0);
  r->psnr_after = psnr(s1);
  return 0;
}

bool dims_ok(int W, int H, int D) {
  // Saddle rows hold 15 ints per saddle, indexed with int offsets.
  return W > 0 && H > 0 && D > 0 && (long long)W * H * D * 15 < (1ll << 31);
}

// ---------------------------------------------------------------------------
// Merge-tree persistence pairs by the elder rule, with a union-find over the
// vertices in the tree's order: an independent check of the extremum-graph
// pairing (constructPersistencePairs, src/ExtreM.cpp:1863-1918) that the
// library runs.  Split tree: vertices by (value, id) descending; a vertex
// without an earlier neighbour starts a component (a maximum); a vertex
// joining several components pairs the younger components' maxima with
// itself.  Join tree: the same in ascending order (minima, 1-saddles).
// Output by extremum rank (maxima ascending, minima descending in value
// then id): (partner vertex, extremum vertex); the global extremum's partner
// is the opposite global extremum.
// ---------------------------------------------------------------------------
template <class T>
void elder_pairs(const T* f, const Grid& g, bool split, std::vector<int>& out,
                 std::vector<int>* parents = nullptr) {
  const int N = g.N;
  std::vector<int> order(N);
  for (int v = 0; v < N; ++v) order[v] = v;
  auto before = [&](int a, int b) {  // a comes first in the tree's order
    return split ? (f[a] > f[b] || (f[a] == f[b] && a > b)) : (f[a] < f[b] || (f[a] == f[b] && a < b));
  };
  std::sort(order.begin(), order.end(), before);
  std::vector<int> parent(N, -1), eldest(N, -1), pos(N);
  for (int k = 0; k < N; ++k) pos[order[k]] = k;
  auto find = [&](int x) {
    while (parent[x] != x) {
      parent[x] = parent[parent[x]];
      x = parent[x];
    }
    return x;
  };
  std::vector<int> ext;           // extrema in processing order
  std::vector<int> partner(N, -1);
  std::vector<int> merged_into(N, -1);  // the eldest of the surviving component
  for (int k = 0; k < N; ++k) {
    const int v = order[k];
    int ids[14];
    const int n = g.nbrs(v, ids);
    int roots[14], nr = 0;
    for (int j = 0; j < n; ++j) {
      const int u = ids[j];
      if (pos[u] >= k) continue;
      const int r = find(u);
      bool dup = false;
      for (int q = 0; q < nr; ++q) dup |= roots[q] == r;
      if (!dup) roots[nr++] = r;
    }
    if (nr == 0) {
      parent[v] = v;
      eldest[v] = v;
      ext.push_back(v);
      continue;
    }
    int keep = roots[0];  // the component whose extremum came first survives
    for (int q = 1; q < nr; ++q)
      if (pos[eldest[roots[q]]] < pos[eldest[keep]]) keep = roots[q];
    for (int q = 0; q < nr; ++q)
      if (roots[q] != keep) {
        partner[eldest[roots[q]]] = v;
        merged_into[eldest[roots[q]]] = eldest[keep];
        parent[roots[q]] = keep;
      }
    parent[v] = keep;
  }
  // Ranks: ascending in the tree's order = reverse of the processing order.
  out.clear();
  if (parents) parents->clear();
  const int opposite = order[N - 1];
  for (int i = (int)ext.size() - 1; i >= 0; --i) {
    const int e = ext[i];
    out.push_back(i == 0 ? opposite : partner[e]);
    out.push_back(e);
    // The branch an extremum joins: the elder rule's survivor at its merge
    // vertex, which is alive there by construction (constructMergeTree's
    // compressed parent, src/ExtreM.cpp:1863-1918); the global extremum its own.
    if (parents) parents->push_back(i == 0 ? e : merged_into[e]);
  }
}

}  // namespace

extern "C" {

// Persistence pairs of a field (see elder_pairs): 2 ints per maximum into
// max_pairs and per minimum into min_pairs; returns 0 and the counts, or -1
// on bad arguments, -3 when a buffer (caps in ints) is too small.
int oracle_persistence_pairs(const void* f, int dtype, int W, int H, int D, int32_t* max_pairs,
                             long long max_cap, int32_t* min_pairs, long long min_cap,
                             long long* n_max, long long* n_min) {
  if (!dims_ok(W, H, D) || !f) return -1;
  Grid g{W, H, D, W * H * D};
  std::vector<int> mx, mn;
  if (dtype == 0) {
    elder_pairs((const float*)f, g, true, mx);
    elder_pairs((const float*)f, g, false, mn);
  } else {
    elder_pairs((const double*)f, g, true, mx);
    elder_pairs((const double*)f, g, false, mn);
  }
  *n_max = (long long)mx.size() / 2;
  *n_min = (long long)mn.size() / 2;
  if ((long long)mx.size() > max_cap || (long long)mn.size() > min_cap) return -3;
  std::memcpy(max_pairs, mx.data(), mx.size() * 4);
  std::memcpy(min_pairs, mn.data(), mn.size() * 4);
  return 0;
}

// The same pairs plus, per extremum, the extremum whose branch it joins at
// its partner vertex (one int per extremum into max_parent / min_parent,
// caps in ints as for the pairs).
int oracle_persistence_tree(const void* f, int dtype, int W, int H, int D, int32_t* max_pairs,
                            long long max_cap, int32_t* min_pairs, long long min_cap,
                            int32_t* max_parent, int32_t* min_parent, long long* n_max,
                            long long* n_min) {
  if (!dims_ok(W, H, D) || !f) return -1;
  Grid g{W, H, D, W * H * D};
  std::vector<int> mx, mn, px, pn;
  if (dtype == 0) {
    elder_pairs((const float*)f, g, true, mx, &px);
    elder_pairs((const float*)f, g, false, mn, &pn);
  } else {
    elder_pairs((const double*)f, g, true, mx, &px);
    elder_pairs((const double*)f, g, false, mn, &pn);
  }
  *n_max = (long long)px.size();
  *n_min = (long long)pn.size();
  if ((long long)mx.size() > max_cap || (long long)mn.size() > min_cap) return -3;
  std::memcpy(max_pairs, mx.data(), mx.size() * 4);
  std::memcpy(min_pairs, mn.data(), mn.size() * 4);
  std::memcpy(max_parent, px.data(), px.size() * 4);
  std::memcpy(min_parent, pn.data(), pn.size() * 4);
  return 0;
}

// Threads of the dense passes (detection, manifolds, rows); results do not
// depend on it.
int oracle_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

// LUT in the reference's LUT.bin layout (24 800 int32).
int oracle_lut(int32_t* out, int n) {
  if (n < kLutSize) return -1;
  const Lut& L = lut();
  for (int i = 0; i < kLutSize; ++i) out[i] = L.table[i];
  return kLutSize;
}

// Per-vertex type and lower-star mask of a field.  dtype 0 = float32, 1 = float64.
int oracle_classify(const void* f, int dtype, int W, int H, int D, int8_t* type, uint16_t* lmask) {
  if (!dims_ok(W, H, D)) return -1;
  Grid g{W, H, D, W * H * D};
  for (int v = 0; v < g.N; ++v)
    type[v] = (int8_t)(dtype == 0 ? classify((const float*)f, g, v, &lmask[v])
                                  : classify((const double*)f, g, v, &lmask[v]));
  return 0;
}

// Full steepest-ascent / steepest-descent roots of every vertex.
int oracle_roots(const void* f, int dtype, int W, int H, int D, int32_t* ds, int32_t* as) {
  if (!dims_ok(W, H, D)) return -1;
  Grid g{W, H, D, W * H * D};
  if (dtype == 0) roots((const float*)f, g, ds, as);
  else roots((const double*)f, g, ds, as);
  return 0;
}

// Full correction, in place on decp.  trace (optional) receives 4-int records;
// counter_out (optional, N int32) the final edit counters (delta_counter).
int oracle_correct(const void* f, void* decp, int dtype, int W, int H, int D,
                   const oracle_params* p, oracle_report* rep, int32_t* trace, int trace_cap,
                   int32_t* counter_out) {
  if (!dims_ok(W, H, D) || !p || p->q <= 0) return -1;
  if (dtype == 0)
    return correct_t((const float*)f, (float*)decp, W, H, D, p, rep, trace, trace_cap,
                     counter_out);
  return correct_t((const double*)f, (double*)decp, W, H, D, p, rep, trace, trace_cap,
                   counter_out);
}

// Mismatch census of `decp` against the original `f` (Corrector::census):
// out receives the eleven loop-test counters.
int oracle_census(const void* f, const void* decp, int dtype, int W, int H, int D, double thr,
                  int wn_lag, int32_t* out) {
  if (!dims_ok(W, H, D) || !out) return -1;
  auto run = [&](auto* tag) {
    using T = std::remove_pointer_t<decltype(tag)>;
    const T* ff = static_cast<const T*>(f);
    std::vector<T> a(static_cast<const T*>(decp), static_cast<const T*>(decp) + (size_t)W * H * D);
    Corrector<T> c;
    c.g = {W, H, D, W * H * D};
    c.f = ff;
    c.a = a.data();
    c.bound = T(0);
    c.thr = (T)thr;
    c.q = 1;
    c.edit_type = 1;
    c.wn_lag = wn_lag;
    c.sentinel = T(0);
    c.trace = nullptr;
    c.trace_cap = 0;
    c.census(out);
  };
  if (dtype == 0) run((float*)nullptr);
  else run((double*)nullptr);
  return 0;
}

// Edit stream of a correction (see encode_t).  Returns 0, -1 on bad
// arguments, -2 for a counter outside 0..7 (edit_type 0), -3 when a stream
// exceeds its buffer.
int oracle_encode(const void* f, const void* decp0, const void* fixed, const int32_t* counter,
                  int dtype, long long n, double bound, int q, int edit_type, uint8_t* index_out,
                  long long index_cap, void* edits_out, long long edits_cap,
                  oracle_edit_report* rep) {
  if (!f || !decp0 || !fixed || n <= 0 || !rep || (edit_type == 0 && !counter)) return -1;
  if (dtype == 0)
    return encode_t((const float*)f, (const float*)decp0, (const float*)fixed, counter, n, bound,
                    q, edit_type, index_out, index_cap, (float*)edits_out, edits_cap, rep);
  return encode_t((const double*)f, (const double*)decp0, (const double*)fixed, counter, n, bound,
                  q, edit_type, index_out, index_cap, (double*)edits_out, edits_cap, rep);
}

}  // extern "C"

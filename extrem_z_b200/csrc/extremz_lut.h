// Critical-point lookup table, built on the host at library load.
//
// Follows the reference's table (src/ExtreM_cuda.cu:263-467 calculateLUT,
// :3280-3318 generateLookupTable, :84-113 keys/lutOffsets, src/LUT.bin): for
// each of the 27 boundary configurations of a grid with every dimension >= 3,
// and each split of its valid neighbours into lower/upper (bit k of the index =
// k-th valid neighbour, in direction order, is upper), the vertex type from the
// number of connected components of the lower and upper link:
//   0 minimum, 1 1-saddle, 2 2-saddle, 3 both, 4 maximum, 5 regular.
// Two link vertices are connected when their offset is itself one of the 14
// directions.  Sections are grouped by neighbour count and ordered by the
// representative vertex of each configuration in a 4x4x4 grid -- the layout of
// LUT.bin, so the table can be checked against it entry by entry.
#pragma once

#include <algorithm>
#include <cstdint>
#include <vector>

#include "extremz_common.cuh"

namespace extremz {

struct HostTables {
  int8_t lut[kLutSize];
  int key_offset[64];  // boundary code -> LUT offset or -1
  int key_mask[kNumKeys];
};

inline int link_components(int nodes_mask, const int adj[kNumDirs]) {
  int comps = 0, left = nodes_mask;
  while (left) {
    int comp = left & -left;
    for (;;) {
      int grow = comp;
      for (int d = 0; d < kNumDirs; ++d)
        if (comp >> d & 1) grow |= adj[d] & nodes_mask;
      if (grow == comp) break;
      comp = grow;
    }
    left &= ~comp;
    ++comps;
  }
  return comps;
}

inline void build_tables(HostTables& t) {
  int adj[kNumDirs];
  for (int a = 0; a < kNumDirs; ++a) {
    adj[a] = 0;
    for (int b = 0; b < kNumDirs; ++b) {
      if (a == b) continue;
      int dx = dir_x(b) - dir_x(a), dy = dir_y(b) - dir_y(a), dz = dir_z(b) - dir_z(a);
      for (int c = 0; c < kNumDirs; ++c)
        if (dir_x(c) == dx && dir_y(c) == dy && dir_z(c) == dz) adj[a] |= 1 << b;
    }
  }
  struct Rep { int id, mask, count; };
  std::vector<Rep> reps;
  const int cls[3] = {0, 1, 3};
  for (int cz : cls)
    for (int cy : cls)
      for (int cx : cls) {
        int mask = 0;
        for (int d = 0; d < kNumDirs; ++d) {
          int nx = cx + dir_x(d), ny = cy + dir_y(d), nz = cz + dir_z(d);
          if (nx >= 0 && nx < 4 && ny >= 0 && ny < 4 && nz >= 0 && nz < 4) mask |= 1 << d;
        }
        reps.push_back({cx + 4 * cy + 16 * cz, mask, __builtin_popcount(mask)});
      }
  std::sort(reps.begin(), reps.end(), [](const Rep& a, const Rep& b) {
    return a.count != b.count ? a.count < b.count : a.id < b.id;
  });
  int offsets[kNumKeys];
  int off = 0;
  for (int k = 0; k < kNumKeys; ++k) {
    const int mask = reps[k].mask, n = reps[k].count;
    t.key_mask[k] = mask;
    offsets[k] = off;
    int valid[kNumDirs];
    for (int d = 0, j = 0; d < kNumDirs; ++d)
      if (mask >> d & 1) valid[j++] = d;
    for (int cfg = 0; cfg < (1 << n); ++cfg) {
      int up = 0, lo = 0;
      for (int j = 0; j < n; ++j) ((cfg >> j & 1) ? up : lo) |= 1 << valid[j];
      int lc = link_components(lo, adj), uc = link_components(up, adj);
      int8_t ty = 0;
      if (lc == 0 && uc == 1) ty = 0;
      else if (lc == 1 && uc == 0) ty = 4;
      else if (lc == 1 && uc == 1) ty = 5;
      else if (lc > 1 && uc > 1) ty = 3;
      else if (lc > 1) ty = 1;
      else if (uc > 1) ty = 2;
      t.lut[off + cfg] = ty;
    }
    off += 1 << n;
  }
  for (int bc = 0; bc < 64; ++bc) {
    int mask = 0;
    for (int d = 0; d < kNumDirs; ++d)
      if (dir_valid(d, bc)) mask |= 1 << d;
    t.key_offset[bc] = -1;
    for (int k = 0; k < kNumKeys; ++k)
      if (t.key_mask[k] == mask) t.key_offset[bc] = offsets[k];
  }
}

}  // namespace extremz

// Runs the reference's constructPersistencePairs and constructMergeTree
// (src/ExtreM.cpp :2132-2249 and :1863-1918, compiled from the reference
// checkout's own source) on a given extremum graph -- test infrastructure
// only, the checker of the numpy restatement in oracle/merge_tree.py.
//
//   ref_mergetree <in.i32> <out.i32>
// in:  nMax, nSaddle, N, globalMin, Maximum[nMax], saddles2[nSaddle],
//      rows[nSaddle][46] (entries, [44] = count, [45] = vertex), order[N]
// out: nMax, pairs[nMax][2], triplets after the pairing [nMax][2], triplets
//      after constructMergeTree [nMax][2], then per branch its vertex count
//      and (order, vertex) per vertex.
//
// The header-declaration fix is the one of ref_cpu_harness.cpp.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <iomanip>
#include <limits>
#include <numeric>
#include <queue>
#include <sstream>

#define directions extremz_header_directions
#include "api/ExtreM.h"
#undef directions
#include "ExtreM.cpp"

static std::vector<int> read_all(const char* path) {
  std::vector<int> v;
  FILE* f = std::fopen(path, "rb");
  if (!f) return v;
  int x;
  while (std::fread(&x, 4, 1, f) == 1) v.push_back(x);
  std::fclose(f);
  return v;
}

int main(int argc, char** argv) {
  if (argc != 3) return 2;
  std::vector<int> in = read_all(argv[1]);
  if (in.size() < 4) return 3;
  size_t k = 0;
  const int nMax = in[k++], nSad = in[k++], N = in[k++], gmin = in[k++];
  if (in.size() != 4 + (size_t)nMax + nSad + (size_t)nSad * 46 + N || nMax < 1) return 3;
  std::vector<int> maximum(in.begin() + k, in.begin() + k + nMax);
  k += nMax;
  std::vector<int> sad(in.begin() + k, in.begin() + k + nSad);
  k += nSad;
  std::vector<std::array<int, 46>> rows(nSad);
  for (int i = 0; i < nSad; ++i)
    for (int q = 0; q < 46; ++q) rows[i][q] = in[k++];
  std::vector<int> order(in.begin() + k, in.begin() + k + N);

  std::vector<std::pair<int, int>> pairs(nMax), triplets(nMax);
  constructPersistencePairs(pairs, triplets, rows, maximum.data(), sad.data(), nMax, gmin);
  std::vector<std::pair<int, int>> paired = triplets;
  std::vector<Branch> branches(nMax);
  constructMergeTree(branches, triplets, maximum, sad, order.data());

  std::vector<int> out;
  out.push_back(nMax);
  for (auto& p : pairs) { out.push_back(p.first); out.push_back(p.second); }
  for (auto& p : paired) { out.push_back(p.first); out.push_back(p.second); }
  for (auto& p : triplets) { out.push_back(p.first); out.push_back(p.second); }
  for (auto& b : branches) {
    out.push_back((int)b.vertices.size());
    for (auto& v : b.vertices) { out.push_back(v.first); out.push_back(v.second); }
  }
  FILE* f = std::fopen(argv[2], "wb");
  if (!f) return 4;
  std::fwrite(out.data(), 4, out.size(), f);
  std::fclose(f);
  return 0;
}

// libExtreMz.so: the reference's CPU host API (include/api/ExtreM.h) over the
// C ABI of libextremz.so, so that a program written against that header -- the
// reference driver main.cpp first of all -- links and runs unchanged, with its
// correction done on the GPU.
//
// How the reference's correction sequence (main.cpp:65-446) maps here:
//   * getdata reads the original field, computes bound = (max - min) * er as
//     the reference does (src/ExtreM.cpp:95-141) and fills decp_data with the
//     decompressed field: the file named by $EXTREMZ_DECP_FILE when set, else
//     the linear quantiser round(f / 2eb) * 2eb (SZ3 is not part of this
//     build; with its output in that file the layer corrects it as given).
//   * The first c_loops call runs the whole correction of decp_data on the GPU
//     (extremz_correct_host, in place): the reference GPU path's semantics over
//     the 14-neighbour stencil, with the join tree preserved, as main.cpp
//     preserves it (main.cpp:21), and no final join-saddle pass (main.cpp has
//     none).  The field main.cpp hands over already carries its own edits
//     (global extrema and original saddles lowered to f - bound,
//     main.cpp:74-75, :122-131).
//   * Every other correction-sequence function evaluates what it reports on
//     the current field exactly: the loop-test counters come from the
//     library's mismatch census (extremz_mismatch_census), the wrong split /
//     join neighbours from the steepest-path roots of both fields
//     (extremz_classify) with the caller's flag arrays, so main.cpp's loop
//     test sees the corrected field's true state and ends.  If a correction
//     stopped at its round cap, the next c_loops / r_loops call resumes it
//     from the current field.
//   * classifyAllVertices, ComputeDescending/AscendingManifold, computeCP and
//     compute_MergeT run the library's classification, steepest-path roots
//     and merge-tree pairing (extremz_persistence_tree) on the GPU.
// Errors end the process with a message: the reference's API has no error
// channel (its functions are void).
#include "extrem_api.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <numeric>

#include "../../include/extremz.h"

// ----------------------------------------------------------------- globals --
extern "C" {
// The 14 directions of the stencil, in the reference's order
// (src/ExtreM.cpp:16-21, src/ExtreM_cuda.cu:155-162); the header declares 78.
int directions[78] = {1, 0, 0,  -1, 0, 0,  0, 1, 0,  0, -1, 0,  0, 0, 1,  0, 0, -1,
                      -1, 1, 0, 1, -1, 0, 0, 1, 1,  0, -1, -1, -1, 0, 1, 1, 0, -1,
                      -1, 1, 1, 1, -1, -1};
int direction_to_index_mapping[26][3];
double* d_deltaBuffer = nullptr;
int width = 0, height = 0, depth = 0, maxNeighbors = 14, num_Elements = 0,
    number_of_false_cases = 0;
std::atomic_int count_f_max{0}, count_f_min{0}, count_f_saddle{0};
int wrong_max_counter = 0, globalMin = 0, dec_globalMin = 0, wrong_max_counter_2 = 0,
    wrong_saddle_counter = 0;
int wrong_saddle_counter_join = 0;
int *adjacency = nullptr, *dec_vertex_type = nullptr, *vertex_type = nullptr, *all_max = nullptr,
    *all_min = nullptr, *all_saddle = nullptr;
double *decp_data = nullptr, *input_data = nullptr, *decp_data_copy = nullptr;
double bound = 0.0;
int *or_saddle_max_map = nullptr, *wrong_neighbors = nullptr, *wrong_neighbors1 = nullptr,
    *wrong_neighbors_index = nullptr, *wrong_rank_max = nullptr, *wrong_rank_max_index = nullptr,
    *wrong_rank_saddle = nullptr, *wrong_rank_saddle_index = nullptr, *wrong_rank_max_2 = nullptr,
    *wrong_rank_max_index_2 = nullptr;
int *wrong_rank_ds_saddle = nullptr, *wrong_rank_ds_saddle_index = nullptr;
int *or_saddle_min_map = nullptr, *wrong_neighbors_ds = nullptr,
    *wrong_neighbors_ds_index = nullptr, *wrong_rank_min = nullptr, *wrong_rank_min_index = nullptr,
    *wrong_rank_min_2 = nullptr, *wrong_rank_min_index_2 = nullptr;
int number_of_false_cases1 = 0, wrong_min_counter = 0, wrong_min_counter_2 = 0;
std::vector<std::array<int, 46>> saddleTriplets, dec_saddleTriplets;
std::vector<std::array<int, 46>> saddle1Triplets, dec_saddle1Triplets;
std::vector<std::vector<int>> vertex_cells;
std::vector<int> saddles2, maximum, dec_saddles2, dec_maximum, delta_counter;
std::vector<int> saddles1, minimum, dec_saddles1, dec_minimum;
std::unordered_map<int, int> largestSaddlesForMax, dec_largestSaddlesForMax;
std::unordered_map<int, int> smallestSaddlesForMin, dec_smallestSaddlesForMin;
int *lowerStars = nullptr, *upperStars = nullptr, *dec_lowerStars = nullptr,
    *dec_upperStars = nullptr;
int *wrong_rank_saddle_join = nullptr, *wrong_rank_saddle_join_index = nullptr;
}

// ------------------------------------------------------------------ state --
namespace {

[[noreturn]] void fail(const char* what, int status) {
  std::fprintf(stderr, "libExtreMz: %s failed: %s (%s)\n", what, extremz_status_string(status),
               extremz_last_cuda_error());
  std::exit(2);
}

void cuda_ok(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    std::fprintf(stderr, "libExtreMz: %s failed: %s\n", what, cudaGetErrorString(e));
    std::exit(2);
  }
}

// A device buffer for the duration of one call.
struct DevBuf {
  void* p = nullptr;
  explicit DevBuf(size_t bytes) { cuda_ok(cudaMalloc(&p, bytes ? bytes : 1), "cudaMalloc"); }
  ~DevBuf() { cudaFree(p); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
};

struct Layer {
  extremz_ctx* ctx = nullptr;
  int device = 0;
  bool corrected = false;  // the first c_loops call has run the correction
  int status = EXTREMZ_OK;
  long long version = 0;  // bumped whenever this layer changes decp_data
  // Roots of the original field's steepest paths, and of decp_data at
  // dec_version; census of decp_data at census_version.
  std::vector<int> ods, oas, dds, das;
  const double* orig_of = nullptr;
  long long dec_version = -1, census_version = -1;
  int census[11] = {0};
};

Layer& layer() {
  static Layer L;
  return L;
}

extremz_ctx* ctx() {
  Layer& L = layer();
  if (!L.ctx) {
    const char* dev = std::getenv("EXTREMZ_DEVICE");
    L.device = dev ? std::atoi(dev) : 0;
    cuda_ok(cudaSetDevice(L.device), "cudaSetDevice");
    const int st = extremz_ctx_create(L.device, &L.ctx);
    if (st != EXTREMZ_OK) fail("extremz_ctx_create", st);
  }
  return L.ctx;
}

long long voxels() { return (long long)width * height * depth; }

void check_dims() {
  if (width <= 0 || height <= 0 || depth <= 0 || voxels() != num_Elements) {
    std::fprintf(stderr, "libExtreMz: width*height*depth (%d*%d*%d) must equal num_Elements (%d)\n",
                 width, height, depth, num_Elements);
    std::exit(2);
  }
}

// Types and roots of a host field (any output may be null).
void classify_host(const double* field, int8_t* type, int* ds, int* as) {
  check_dims();
  const size_t n = (size_t)voxels();
  DevBuf f(n * 8), t(n), d(n * 4), a(n * 4);
  cuda_ok(cudaMemcpy(f.p, field, n * 8, cudaMemcpyHostToDevice), "copy in");
  const int st = extremz_classify(ctx(), f.p, EXTREMZ_F64, width, height, depth,
                                  static_cast<int8_t*>(t.p), static_cast<int32_t*>(d.p),
                                  static_cast<int32_t*>(a.p), nullptr);
  if (st != EXTREMZ_OK) fail("extremz_classify", st);
  if (type) cuda_ok(cudaMemcpy(type, t.p, n, cudaMemcpyDeviceToHost), "copy out");
  if (ds) cuda_ok(cudaMemcpy(ds, d.p, n * 4, cudaMemcpyDeviceToHost), "copy out");
  if (as) cuda_ok(cudaMemcpy(as, a.p, n * 4, cudaMemcpyDeviceToHost), "copy out");
}

// Roots of the original field (input_data) and of decp_data, cached.
void ensure_roots() {
  Layer& L = layer();
  const size_t n = (size_t)voxels();
  if (L.orig_of != input_data || L.ods.size() != n) {
    L.ods.resize(n);
    L.oas.resize(n);
    classify_host(input_data, nullptr, L.ods.data(), L.oas.data());
    L.orig_of = input_data;
  }
  if (L.dec_version != L.version || L.dds.size() != n) {
    L.dds.resize(n);
    L.das.resize(n);
    classify_host(decp_data, nullptr, L.dds.data(), L.das.data());
    L.dec_version = L.version;
  }
}

// The eleven loop-test counters of decp_data against input_data, cached.
const int* census() {
  Layer& L = layer();
  if (L.census_version == L.version) return L.census;
  check_dims();
  const size_t n = (size_t)voxels();
  DevBuf f(n * 8), g(n * 8);
  cuda_ok(cudaMemcpy(f.p, input_data, n * 8, cudaMemcpyHostToDevice), "copy in");
  cuda_ok(cudaMemcpy(g.p, decp_data, n * 8, cudaMemcpyHostToDevice), "copy in");
  const int st = extremz_mismatch_census(ctx(), f.p, g.p, EXTREMZ_F64, width, height, depth, 0.0,
                                         L.census, nullptr);
  if (st != EXTREMZ_OK) fail("extremz_mismatch_census", st);
  L.census_version = L.version;
  return L.census;
}

// The correction of decp_data in place (from its current values).
void run_correction() {
  check_dims();
  Layer& L = layer();
  extremz_params p;
  extremz_default_params(&p);
  p.bound = bound;
  p.preserve_join = 1;  // main.cpp:21
  p.final_join = 0;     // main.cpp has no final join-saddle pass
  extremz_report rep;
  const int st = extremz_correct_host(ctx(), input_data, decp_data, EXTREMZ_F64, width, height,
                                      depth, &p, &rep, nullptr);
  if (st != EXTREMZ_OK && st != EXTREMZ_ROUND_CAP) fail("extremz_correct_host", st);
  L.status = st;
  L.corrected = true;
  ++L.version;
  if (st == EXTREMZ_ROUND_CAP)
    std::fprintf(stderr, "libExtreMz: the correction stopped at its round cap; the next "
                         "c_loops / r_loops call resumes it\n");
}

bool above(const double* a, int u, int v) { return a[u] > a[v] || (a[u] == a[v] && u > v); }
bool below(const double* a, int u, int v) { return a[u] < a[v] || (a[u] == a[v] && u < v); }

// Neighbour of v in direction d, or -1 outside the grid.
int neighbour(int v, int d) {
  const int x = v % width, y = (v / width) % height, z = v / (width * height);
  const int nx = x + directions[3 * d], ny = y + directions[3 * d + 1],
            nz = z + directions[3 * d + 2];
  if (nx < 0 || nx >= width || ny < 0 || ny >= height || nz < 0 || nz >= depth) return -1;
  return nx + (ny + nz * height) * width;
}

int stencil() { return std::min(std::max(maxNeighbors, 1), 14); }

}  // namespace

// ------------------------------------------------------- field and helpers --
void Branch::print() const {
  for (const auto& v : vertices) std::cout << "(" << v.first << ", " << v.second << ") ";
  std::cout << std::endl;
}

extern "C" {

void saveArrayToBin(const double* arr, size_t size, const std::string& filename) {
  std::ofstream out(filename, std::ios::binary);
  if (!out) {
    std::cerr << "Error opening file for writing: " << filename << std::endl;
    return;
  }
  out.write(reinterpret_cast<const char*>(arr), (std::streamsize)(size * sizeof(double)));
}

// The reference builds the 2-D triangle star of its CPU classification here
// (src/ExtreM.cpp:1585-1595); the GPU classification needs none, so
// vertex_cells is left as the caller sized it.
void get_vertex_traingle() {}

static bool read_exact(const std::string& path, double* out, long long n, const char* what) {
  std::ifstream file(path, std::ios::binary | std::ios::ate);
  if (!file) {
    std::cerr << "Cannot open file: " << path << std::endl;
    return false;
  }
  const std::streamsize size = file.tellg();
  if (size != (std::streamsize)(n * (long long)sizeof(double))) {
    std::cerr << what << " file size does not match expected data size." << std::endl;
    return false;
  }
  file.seekg(0, std::ios::beg);
  file.read(reinterpret_cast<char*>(out), size);
  return (bool)file;
}

void getdata(const std::string& filename, const double er, int data_size, std::string type) {
  (void)type;
  if (!read_exact(filename, input_data, data_size, "Input")) return;
  const auto mm = std::minmax_element(input_data, input_data + data_size);
  bound = (*mm.second - *mm.first) * er;
  const char* decp_file = std::getenv("EXTREMZ_DECP_FILE");
  if (decp_file && *decp_file) {
    if (!read_exact(decp_file, decp_data, data_size, "Decompressed")) return;
  } else {
    // Linear quantiser round(f / 2eb) * 2eb; a value the rounding leaves
    // outside the bound steps one ulp toward f.
    const double step = 2.0 * bound;
    for (int i = 0; i < data_size; ++i) {
      double q = bound > 0 ? std::nearbyint(input_data[i] / step) * step : input_data[i];
      if (std::fabs(input_data[i] - q) > bound) q = std::nextafter(q, input_data[i]);
      decp_data[i] = q;
    }
  }
  if (decp_data_copy) std::copy(decp_data, decp_data + data_size, decp_data_copy);
  Layer& L = layer();
  L.corrected = false;
  L.orig_of = nullptr;
  ++L.version;
}

void getSortedIndexes(const double* vec, int* indexes) {
  std::iota(indexes, indexes + num_Elements, 0);
  std::sort(indexes, indexes + num_Elements,
            [vec](int i, int j) { return vec[i] < vec[j] || (vec[i] == vec[j] && i < j); });
}

void computeAdjacency() {
  const int m = std::min(std::max(maxNeighbors, 0), 14);
  for (int v = 0; v < num_Elements; ++v)
    for (int d = 0; d < m; ++d) adjacency[(size_t)v * m + d] = neighbour(v, d);
}

// Vertex types of heightMap by the library's classification (the 14-neighbour
// lookup table, classifyVertex_CUDA src/ExtreM_cuda.cu:3720-3911), and each
// vertex's lower / upper neighbours among the first maxNeighbors directions,
// with their count at slot maxNeighbors, as the reference's rows are laid out.
void classifyAllVertices(int* vertex_type_out, const double* heightMap, int* lower, int* upper,
                         int type) {
  (void)type;
  const size_t n = (size_t)voxels();
  std::vector<int8_t> t(n);
  classify_host(heightMap, t.data(), nullptr, nullptr);
  for (size_t v = 0; v < n; ++v) vertex_type_out[v] = t[v];
  const int m = std::min(std::max(maxNeighbors, 0), 14);
  if (!lower || !upper) return;
  for (int v = 0; v < (int)n; ++v) {
    int* lo = lower + (size_t)v * (m + 1);
    int* up = upper + (size_t)v * (m + 1);
    int nl = 0, nu = 0;
    for (int d = 0; d < m; ++d) {
      const int r = neighbour(v, d);
      if (r < 0) continue;
      if (below(heightMap, r, v)) lo[nl++] = r;
      else up[nu++] = r;
    }
    lo[m] = nl;
    up[m] = nu;
  }
}

int ComputeDescendingManifold(const double* offset, const int* vt, int* DS_M) {
  (void)vt;
  classify_host(offset, nullptr, DS_M, nullptr);
  return 0;
}

int ComputeAscendingManifold(const double* offset, const int* vt, int* AS_M) {
  (void)vt;
  classify_host(offset, nullptr, nullptr, AS_M);
  return 0;
}

// Critical-point lists from vertex types, ordered as the reference orders
// them (src/ExtreM.cpp:1920-2040): 2-saddles and minima descending, 1-saddles
// and maxima ascending in (value, id).  A 2-saddle's row holds the local
// indices (into `maximum`) of the maxima its upper neighbours ascend to,
// distinct and ascending, with their count at [44]; a 1-saddle's row the
// minima its lower neighbours descend to; [45] is the saddle's vertex id.
void computeCP(std::vector<std::pair<int, int>>& maximaTriplets,
               std::vector<std::pair<int, int>>& minimumTriplets,
               std::vector<std::array<int, 46>>& sad2_rows,
               std::vector<std::array<int, 46>>& sad1_rows, const double* offset,
               const int* desManifold, const int* ascManifold, const int* vertex_type_tmp,
               std::vector<int>& sad2, std::vector<int>& sad1, std::vector<int>& minima,
               std::vector<int>& maxima, int& global_min, int translation) {
  (void)maximaTriplets;
  (void)minimumTriplets;
  sad2.clear();
  sad1.clear();
  minima.clear();
  maxima.clear();
  for (int v = 0; v < num_Elements; ++v) {
    const int t = vertex_type_tmp[v];
    if (t == 2 || t == 3) sad2.push_back(v);
    if (t == 1 || t == 3) sad1.push_back(v);
    if (t == 4) maxima.push_back(v);
    if (t == 0) minima.push_back(v);
  }
  auto up = [offset](int a, int b) { return above(offset, a, b); };
  auto down = [offset](int a, int b) { return below(offset, a, b); };
  std::sort(sad2.begin(), sad2.end(), up);
  std::sort(sad1.begin(), sad1.end(), down);
  std::sort(maxima.begin(), maxima.end(), down);
  std::sort(minima.begin(), minima.end(), up);
  std::unordered_map<int, int> max_local, min_local;
  for (size_t i = 0; i < maxima.size(); ++i) max_local[maxima[i]] = (int)i;
  for (size_t i = 0; i < minima.size(); ++i) min_local[minima[i]] = (int)i;
  auto rows = [&](const std::vector<int>& sads, std::vector<std::array<int, 46>>& out,
                  const int* labels, const std::unordered_map<int, int>& local, bool upper) {
    out.assign(sads.size(), std::array<int, 46>{});
    for (size_t i = 0; i < sads.size(); ++i) {
      const int s = sads[i];
      std::vector<int> r;
      for (int d = 0; d < 14; ++d) {
        const int nb = neighbour(s, d);
        if (nb < 0 || (upper ? !above(offset, nb, s) : !below(offset, nb, s))) continue;
        const auto it = local.find(labels[nb]);
        if (it != local.end()) r.push_back(it->second);
      }
      std::sort(r.begin(), r.end());
      r.erase(std::unique(r.begin(), r.end()), r.end());
      for (size_t k = 0; k < r.size(); ++k) out[i][k] = r[k];
      out[i][44] = (int)r.size();
      out[i][45] = s;
    }
  };
  rows(sad2, sad2_rows, desManifold, max_local, true);
  rows(sad1, sad1_rows, ascManifold, min_local, false);
  if (translation == 0) return;
  int g = 0;
  for (int v = 1; v < num_Elements; ++v)
    if (below(offset, v, g)) g = v;
  global_min = g;
}

// Per extremum (local index), the row index of the last saddle row that
// reaches it, rows in the order the caller keeps them.
void computelargestSaddlesForMax(const int nMax, const std::vector<std::array<int, 46>>& rows,
                                 std::unordered_map<int, int>& out, const std::vector<int>* list) {
  (void)nMax;
  (void)list;
  out.clear();
  for (size_t i = 0; i < rows.size(); ++i)
    for (int k = 0; k < rows[i][44]; ++k) out[rows[i][k]] = (int)i;
}

void computesmallestSaddlesForMin(const int nMin, const std::vector<std::array<int, 46>>& rows,
                                  std::unordered_map<int, int>& out, const std::vector<int>* list) {
  computelargestSaddlesForMax(nMin, rows, out, list);
}

// The reference fills its saddle-to-extremum maps here for its own s_loops
// (src/ExtreM.cpp:2373-2403); the GPU correction keeps its own.
void compute_Max_for_Saddle(int saddle, const double* offset) {
  (void)saddle;
  (void)offset;
}
void compute_Min_for_Saddle(int saddle, const double* offset) {
  (void)saddle;
  (void)offset;
}

// ------------------------------------------------------------ correction --
// The first call corrects decp_data (see the top of this file); a later call
// resumes a correction that stopped at its round cap.  Either way the
// critical-point counters are then those of the current field.
void c_loops(std::string type) {
  (void)type;
  Layer& L = layer();
  if (!L.corrected || L.status == EXTREMZ_ROUND_CAP) run_correction();
  const int* c = census();
  count_f_max = c[2];
  count_f_min = c[3];
  count_f_saddle = c[4];
}

void r_loops(std::string type) {
  (void)type;
  Layer& L = layer();
  if (!L.corrected || L.status == EXTREMZ_ROUND_CAP) run_correction();
}

// The first upper (split) or lower (join) neighbour of the saddle, in
// direction order, whose steepest-path root differs between the original and
// the current field and which no earlier call flagged: flagged, appended to
// the index list and counted, as src/ExtreM.cpp:2405-2450 does.
static void wrong_neighbour(int saddle, int& count, const double* offset, bool split) {
  ensure_roots();
  const Layer& L = layer();
  int* flags = split ? wrong_neighbors : wrong_neighbors_ds;
  int* list = split ? wrong_neighbors_index : wrong_neighbors_ds_index;
  const std::vector<int>& now = split ? L.dds : L.das;
  const std::vector<int>& orig = split ? L.ods : L.oas;
  for (int d = 0; d < 14; ++d) {
    const int n = neighbour(saddle, d);
    if (n < 0 || (split ? !above(offset, n, saddle) : !below(offset, n, saddle))) continue;
    if (now[n] == orig[n] || (flags && flags[n])) continue;
    if (flags) flags[n] = 1;
    if (list) list[count] = n;
    ++count;
    return;
  }
}

void get_wrong_split_neighbors(int saddle, int& num_false_cases, const double* offset) {
  wrong_neighbour(saddle, num_false_cases, offset, true);
}

void get_wrong_join_neighbors(int saddle, int& num_false_cases, const double* offset) {
  wrong_neighbour(saddle, num_false_cases, offset, false);
}

void get_false_criticle_points() {
  const int* c = census();
  count_f_max = c[2];
  count_f_min = c[3];
  count_f_saddle = c[4];
}

void get_wrong_index_max() {
  const int* c = census();
  wrong_max_counter = c[5];
  wrong_max_counter_2 = c[6];
}

void get_wrong_index_min() {
  const int* c = census();
  wrong_min_counter = c[8];
  wrong_min_counter_2 = c[9];
}

void get_wrong_index_saddles() { wrong_saddle_counter = census()[7]; }

void get_wrong_index_saddles_join() { wrong_saddle_counter_join = census()[10]; }

void s_loops(std::string type) {
  (void)type;
  get_wrong_index_max();
}

void s_loops_join(std::string type) {
  (void)type;
  get_wrong_index_min();
}

void saddle_loops(std::string type) {
  (void)type;
  get_wrong_index_saddles();
}

void saddle_loops_join(std::string type) {
  (void)type;
  get_wrong_index_saddles_join();
}

// ------------------------------------------------------------ merge tree --
// Branch decomposition of the split tree of `offset` (constructPersistence-
// Pairs + constructMergeTree, src/ExtreM.cpp:1863-1918, 2132-2249, as
// compute_MergeT :2930-2952 calls them), from the library's pairing
// (extremz_persistence_tree), one branch per maximum in ascending (value, id)
// order, the global maximum last.  A branch holds its maximum, the merge
// vertices of the branches that join it and its own merge vertex (the global
// minimum for the global maximum's branch), as (order, vertex id) pairs sorted
// descending; order is the vertex's rank in (value, id).  maximaTriplets[b]
// becomes (merge vertex, branch joined).
void compute_MergeT(std::vector<Branch>& branches, const std::vector<int> sad2,
                    const std::vector<int> maxima, std::vector<std::pair<int, int>>& maximaTriplets,
                    std::vector<std::array<int, 46>>& rows, const double* offset,
                    const int data_size, const int global_min) {
  (void)sad2;
  (void)maxima;
  (void)rows;
  (void)global_min;
  check_dims();
  const size_t n = (size_t)data_size;
  DevBuf f(n * 8), mp(n * 8), np_(n * 8), mpar(n * 4), npar(n * 4);
  cuda_ok(cudaMemcpy(f.p, offset, n * 8, cudaMemcpyHostToDevice), "copy in");
  long long nmax = 0, nmin = 0;
  const int st = extremz_persistence_tree(
      ctx(), f.p, EXTREMZ_F64, width, height, depth, static_cast<int32_t*>(mp.p), 2ll * n,
      static_cast<int32_t*>(np_.p), 2ll * n, static_cast<int32_t*>(mpar.p),
      static_cast<int32_t*>(npar.p), &nmax, &nmin, nullptr);
  if (st != EXTREMZ_OK) fail("extremz_persistence_tree", st);
  std::vector<int> pairs(2 * (size_t)nmax), parent((size_t)nmax);
  if (nmax) {
    cuda_ok(cudaMemcpy(pairs.data(), mp.p, pairs.size() * 4, cudaMemcpyDeviceToHost), "copy out");
    cuda_ok(cudaMemcpy(parent.data(), mpar.p, parent.size() * 4, cudaMemcpyDeviceToHost),
            "copy out");
  }
  // Rank of every vertex in (value, id).
  std::vector<int> sorted(n), order(n);
  std::iota(sorted.begin(), sorted.end(), 0);
  std::sort(sorted.begin(), sorted.end(), [offset](int a, int b) { return below(offset, a, b); });
  for (size_t i = 0; i < n; ++i) order[sorted[i]] = (int)i;
  const int nb = (int)nmax;
  std::unordered_map<int, int> branch_of;  // maximum vertex -> branch
  for (int b = 0; b < nb; ++b) branch_of[pairs[2 * b + 1]] = b;
  std::vector<int> par(nb), sad(nb);
  for (int b = 0; b < nb; ++b) {
    sad[b] = pairs[2 * b];
    const auto it = branch_of.find(parent[b]);
    par[b] = it == branch_of.end() ? b : it->second;
  }
  if (nb) par[nb - 1] = nb - 1;
  // A parent whose own merge vertex lies above the branch's (it merged
  // first) hands the branch on to its parent, until nothing moves.
  for (bool moved = true; moved;) {
    moved = false;
    for (int b = 0; b < nb; ++b) {
      const int p = par[b], q = par[p];
      if (q != p && p != nb - 1 && order[sad[p]] > order[sad[b]]) {
        par[b] = q;
        moved = true;
      }
    }
  }
  branches.assign(nb, Branch());
  maximaTriplets.assign(nb, std::make_pair(-1, -1));
  for (int b = 0; b < nb; ++b) {
    const int mx = pairs[2 * b + 1];
    branches[b].vertices.emplace_back(order[mx], mx);
    maximaTriplets[b] = std::make_pair(sad[b], par[b]);
    if (par[b] != b) {
      branches[b].vertices.emplace_back(order[sad[b]], sad[b]);
      branches[b].parentBranch = &branches[par[b]];
      branches[par[b]].vertices.emplace_back(order[sad[b]], sad[b]);
    } else {
      branches[b].vertices.emplace_back(-1, sad[b]);
    }
  }
  for (auto& br : branches) std::sort(br.vertices.begin(), br.vertices.end(), std::greater<>());
}

}  // extern "C"

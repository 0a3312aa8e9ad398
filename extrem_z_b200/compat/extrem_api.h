// Host API of the reference's CPU library, restated for the compatibility
// layer libExtreMz.so (extrem_api.cpp), which implements it over the C ABI
// of libextremz.so.
//
// A program written against the reference's include/api/ExtreM.h -- its
// driver main.cpp first of all -- links against libExtreMz.so unchanged: the
// names, types and linkage below are the ones that header declares
// (include/api/ExtreM.h:10-123), so that both declarations agree.  The
// reference header declares `directions[78]` while its library defines 42
// entries (src/ExtreM.cpp:16); here the array has the declared 78 entries,
// the first 42 holding the 14 directions, so the unmodified header compiles
// and links against this layer.
#ifndef EXTREMZ_COMPAT_EXTREM_API_H
#define EXTREMZ_COMPAT_EXTREM_API_H

#include <stddef.h>

#include <array>
#include <atomic>
#include <cstdint>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

// One branch of a merge tree: (order, vertex id) pairs, the extremum first
// after sorting, and the branch it joins (include/api/ExtreM.h:10-15).
struct Branch {
  std::vector<std::pair<int, int>> vertices;
  Branch* parentBranch = nullptr;
  void print() const;
};

extern "C" {
// Field, neighbourhood and bound (include/api/ExtreM.h:18-29).
extern int directions[78], direction_to_index_mapping[26][3];
extern double* d_deltaBuffer;
extern int width, height, depth, maxNeighbors, num_Elements, number_of_false_cases;
extern std::atomic_int count_f_max, count_f_min, count_f_saddle;
extern int wrong_max_counter, globalMin, dec_globalMin, wrong_max_counter_2,
    wrong_saddle_counter;
extern int wrong_saddle_counter_join;
extern int *adjacency, *dec_vertex_type, *vertex_type, *all_max, *all_min, *all_saddle;
extern double *decp_data, *input_data, *decp_data_copy;
extern double bound;

// Work arrays of the correction loops, allocated by the caller
// (include/api/ExtreM.h:30-41).
extern int *or_saddle_max_map, *wrong_neighbors, *wrong_neighbors1, *wrong_neighbors_index,
    *wrong_rank_max, *wrong_rank_max_index, *wrong_rank_saddle, *wrong_rank_saddle_index,
    *wrong_rank_max_2, *wrong_rank_max_index_2;
extern int *wrong_rank_ds_saddle, *wrong_rank_ds_saddle_index;
extern int *or_saddle_min_map, *wrong_neighbors_ds, *wrong_neighbors_ds_index, *wrong_rank_min,
    *wrong_rank_min_index, *wrong_rank_min_2, *wrong_rank_min_index_2;
extern int number_of_false_cases1, wrong_min_counter, wrong_min_counter_2;
extern std::vector<std::array<int, 46>> saddleTriplets, dec_saddleTriplets;
extern std::vector<std::array<int, 46>> saddle1Triplets, dec_saddle1Triplets;
extern std::vector<std::vector<int>> vertex_cells;
extern std::vector<int> saddles2, maximum, dec_saddles2, dec_maximum, delta_counter;
extern std::vector<int> saddles1, minimum, dec_saddles1, dec_minimum;
extern std::unordered_map<int, int> largestSaddlesForMax, dec_largestSaddlesForMax;
extern std::unordered_map<int, int> smallestSaddlesForMin, dec_smallestSaddlesForMin;
extern int *lowerStars, *upperStars, *dec_lowerStars, *dec_upperStars;
extern int *wrong_rank_saddle_join, *wrong_rank_saddle_join_index;

// The correction sequence (include/api/ExtreM.h:43-123).
void saveArrayToBin(const double* arr, size_t size, const std::string& filename);
void get_vertex_traingle();
void getdata(const std::string& filename, const double er, int data_size, std::string type);
int ComputeDescendingManifold(const double* offset, const int* vertex_type, int* DS_M);
int ComputeAscendingManifold(const double* offset, const int* vertex_type, int* AS_M);
void classifyAllVertices(int* vertex_type, const double* heightMap, int* lowerStars,
                         int* upperStars, int type);
void computeAdjacency();
void c_loops(std::string type);
void computeCP(std::vector<std::pair<int, int>>& maximaTriplets,
               std::vector<std::pair<int, int>>& minimumTriplets,
               std::vector<std::array<int, 46>>& saddleTriplets,
               std::vector<std::array<int, 46>>& saddle1Triplets, const double* offset,
               const int* desManifold, const int* ascManifold, const int* vertex_type_tmp,
               std::vector<int>& saddles2, std::vector<int>& saddles1, std::vector<int>& minimum,
               std::vector<int>& maximum, int& globalMin, int translation);
void getSortedIndexes(const double* vec, int* indexes);
void compute_Max_for_Saddle(int saddle, const double* offset);
void compute_Min_for_Saddle(int saddle, const double* offset);
void get_wrong_split_neighbors(int saddle, int& num_false_cases, const double* offset);
void get_wrong_join_neighbors(int saddle, int& num_false_cases, const double* offset);
void get_false_criticle_points();
void r_loops(std::string type);
void s_loops(std::string type);
void s_loops_join(std::string type);
void get_wrong_index_max();
void get_wrong_index_min();
void get_wrong_index_saddles();
void get_wrong_index_saddles_join();
void saddle_loops(std::string type);
void saddle_loops_join(std::string type);
void compute_MergeT(std::vector<Branch>& branches, const std::vector<int> saddles2,
                    const std::vector<int> maximum,
                    std::vector<std::pair<int, int>>& maximaTriplets,
                    std::vector<std::array<int, 46>>& saddleTriplets, const double* offset,
                    const int data_size, const int globalMin);
void computelargestSaddlesForMax(const int nMax,
                                 const std::vector<std::array<int, 46>>& saddleTriplets,
                                 std::unordered_map<int, int>& largestSaddlesForMax,
                                 const std::vector<int>* saddles2);
void computesmallestSaddlesForMin(const int nMin,
                                  const std::vector<std::array<int, 46>>& saddleTriplets,
                                  std::unordered_map<int, int>& smallestSaddlesForMin,
                                  const std::vector<int>* minimum);
}

#endif  // EXTREMZ_COMPAT_EXTREM_API_H

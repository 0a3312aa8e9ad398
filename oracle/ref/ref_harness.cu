// Runs the reference GPU correction (src/ExtreM_cuda.cu, compiled unmodified
// from the reference checkout) on a given field and writes its corrected field
// -- test harness only, the checker for the oracle.
//
//   ref_gpu <orig.f64> <W> <H> <D> <er> <sim> <q> <edit_type> <out.f64>
// with the decompressed field in $EXTREMZ_REF_DECP, LUT.bin in the working
// directory and ../stat_result writable (the reference writes timings there).
//
// The reference's main() computes the correction, then calls cost() /
// floating_point_cost(), which write to fixed cluster paths and throw when
// those files are missing (src/ExtreM_cuda.cu:4626-4631, :4746-4751) before
// fixed.bin is saved.  The harness catches that and copies the corrected
// field out of the reference's own device buffer.
//
// Every cudaMalloc of the reference goes through a guard that pads the
// allocation on both sides: get_wrong_index_saddles reads decp_data[-1] for a
// maximum without saddles (src/ExtreM_cuda.cu:3197-3198).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <iomanip>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

static cudaError_t extremz_guarded_malloc(void** p, size_t n) {
  char* base = nullptr;
  cudaError_t e = ::cudaMalloc(reinterpret_cast<void**>(&base), n + 512);
  if (e == cudaSuccess) {
    cudaMemset(base, 0, 256);
    *p = base + 256;
  }
  return e;
}
#define cudaMalloc(p, n) extremz_guarded_malloc(reinterpret_cast<void**>(p), (n))
#define main extremz_reference_main
#include "ExtreM_cuda.cu"
#undef main
#undef cudaMalloc

// Host-only modes that run two helpers of the reference's edit-stream
// encoder on int32 input, for the oracle's golden vectors:
//   ref_gpu --encode3 <in.i32> <out.u8>   encodeTo3BitBitmap (:4282-4312)
//   ref_gpu --diff    <in.i32> <out.i32>  get_diff_index<int> (:4315-4323)
static int helper_mode(int argc, char** argv) {
  FILE* fi = std::fopen(argv[2], "rb");
  if (!fi) return 6;
  std::vector<int> in;
  int v;
  while (std::fread(&v, sizeof(int), 1, fi) == 1) in.push_back(v);
  std::fclose(fi);
  FILE* fo = std::fopen(argv[3], "wb");
  if (!fo) return 6;
  if (std::string(argv[1]) == "--encode3") {
    std::vector<uint8_t> out = encodeTo3BitBitmap(in);
    if (!out.empty()) std::fwrite(out.data(), 1, out.size(), fo);
  } else {
    std::vector<int> out = get_diff_index<int>(in);
    std::fwrite(out.data(), sizeof(int), out.size(), fo);
  }
  std::fclose(fo);
  return 0;
}

int main(int argc, char** argv) {
  if (argc == 4 && (std::string(argv[1]) == "--encode3" || std::string(argv[1]) == "--diff"))
    return helper_mode(argc, argv);
  if (argc != 10) {
    std::fprintf(stderr, "usage: %s orig W H D er sim q edit_type out\n", argv[0]);
    return 2;
  }
  std::string dims = std::string(argv[1]) + "," + argv[2] + "," + argv[3] + "," + argv[4];
  std::vector<std::string> a = {"ExtreM_cuda", dims, argv[5], "sz3", argv[6], argv[7], argv[8]};
  std::vector<char*> av;
  for (auto& s : a) av.push_back(const_cast<char*>(s.c_str()));
  int rc = 0;
  try {
    rc = extremz_reference_main((int)av.size(), av.data());
  } catch (const std::exception& e) {
    std::fprintf(stderr, "reference main stopped after the correction: %s\n", e.what());
  }
  if (rc != 0) {
    std::fprintf(stderr, "reference main returned %d\n", rc);
    return 4;
  }
  double* dptr = nullptr;
  if (cudaMemcpyFromSymbol(&dptr, decp_data, sizeof(double*)) != cudaSuccess) return 5;
  std::vector<double> out((size_t)num_Elements_host);
  if (cudaMemcpy(out.data(), dptr, out.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
    return 5;
  FILE* fh = std::fopen(argv[9], "wb");
  if (!fh) return 6;
  std::fwrite(out.data(), sizeof(double), out.size(), fh);
  std::fclose(fh);
  return 0;
}

// Stand-in for the SZ3 API used by the reference's getdata (test harness only).
//
// SZ3 is a third-party dependency that is not vendored with the reference and
// pinned nowhere.  The harness needs the reference's correction to run on a
// decompressed field that this repository also feeds to its own corrector, so
// SZ_decompress here returns that field: the raw float64 file named by the
// environment variable EXTREMZ_REF_DECP.  SZ_compress only records the size.
// The four zstd entry points that an unused reference function names are
// declared and stubbed so that the program links.
#pragma once
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace SZ3 {
enum ALGO { ALGO_LORENZO_REG = 0, ALGO_INTERP_LORENZO = 1, ALGO_INTERP = 2 };
enum EB { EB_ABS = 0, EB_REL = 1 };
struct Config {
  size_t dims[3];
  int cmprAlgo = ALGO_INTERP_LORENZO;
  int errorBoundMode = EB_REL;
  double relErrorBound = 0.0;
  double absErrorBound = 0.0;
  explicit Config(size_t n) : dims{n, 1, 1} {}
  Config(size_t d, size_t h, size_t w) : dims{d, h, w} {}
  size_t num() const { return dims[0] * dims[1] * dims[2]; }
};
}  // namespace SZ3

template <class T>
char* SZ_compress(const SZ3::Config& conf, const T* data, size_t& cmpSize) {
  (void)data;
  cmpSize = conf.num() * sizeof(T);
  char* out = new char[8];
  std::memcpy(out, &cmpSize, sizeof(size_t) < 8 ? sizeof(size_t) : 8);
  return out;
}

template <class T>
void SZ_decompress(const SZ3::Config& conf, const char* cmp, size_t cmpSize, T*& out) {
  (void)cmp;
  (void)cmpSize;
  const char* path = std::getenv("EXTREMZ_REF_DECP");
  if (!path) {
    std::fprintf(stderr, "EXTREMZ_REF_DECP is not set\n");
    std::exit(3);
  }
  FILE* fh = std::fopen(path, "rb");
  if (!fh) {
    std::fprintf(stderr, "cannot open %s\n", path);
    std::exit(3);
  }
  if (!out) out = new T[conf.num()];
  size_t got = std::fread(out, sizeof(T), conf.num(), fh);
  std::fclose(fh);
  if (got != conf.num()) {
    std::fprintf(stderr, "short read of %s\n", path);
    std::exit(3);
  }
}

inline size_t ZSTD_compressBound(size_t n) { return n + 64; }
inline size_t ZSTD_compress(void*, size_t, const void*, size_t, int) { return 0; }
inline unsigned ZSTD_isError(size_t) { return 1; }
inline const char* ZSTD_getErrorName(size_t) { return "zstd stub"; }

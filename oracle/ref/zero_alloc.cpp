// Optional link-in for the reference CPU program: every operator new returns
// zero-filled memory.  The reference reads heap memory that it never wrote
// (the tempArray of computeCP, src/ExtreM.cpp:2004-2012, holds entries only for
// the extrema it lists, but findAscPaths reads it at every steepest-ascent
// root, :1617); with this link-in those reads return 0 on every run instead of
// whatever the allocator hands back.  Test infrastructure only.
#include <cstdlib>
#include <new>

static void* zero_alloc(std::size_t n) {
  void* p = std::calloc(n ? n : 1, 1);
  if (!p) throw std::bad_alloc();
  return p;
}
void* operator new(std::size_t n) { return zero_alloc(n); }
void* operator new[](std::size_t n) { return zero_alloc(n); }
void operator delete(void* p) noexcept { std::free(p); }
void operator delete[](void* p) noexcept { std::free(p); }
void operator delete(void* p, std::size_t) noexcept { std::free(p); }
void operator delete[](void* p, std::size_t) noexcept { std::free(p); }

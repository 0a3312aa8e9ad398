// Builds the reference's CPU correction (src/ExtreM.cpp and main.cpp of the
// reference checkout, compiled from their own sources) into one program --
// test infrastructure only, used to record how that path behaves on 2-D
// fields.
//
// include/api/ExtreM.h declares `directions[78]` while src/ExtreM.cpp:16
// defines it with 42 elements, so the unmodified pair does not compile.  The
// harness includes the header first with that one declarator renamed; the
// header's include guard then keeps src/ExtreM.cpp from declaring it again.
// Nothing else is changed.  SZ3 is replaced by the stand-in header next to
// this file (the decompressed field comes from $EXTREMZ_REF_DECP).
//
//   ref_cpu "<orig.f64>,W,H,D" <er> <compressor-id>    (writes fixed.bin)
#include <algorithm>
#include <chrono>
#include <cmath>
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

#define main extremz_cpu_reference_main
#include "main.cpp"
#undef main

int main(int argc, char** argv) { return extremz_cpu_reference_main(argc, argv); }

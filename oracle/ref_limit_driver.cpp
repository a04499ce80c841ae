// Test infrastructure (the checker, not the product): the reference's own
// limit<T> (ctas src/common/external.world.cpp:69-90), which turns a float
// image into integer samples for the 8- and 16-bit image writers
// (external.world.cpp:743, 1659).  external.world.cpp itself needs TIFF, HDF5
// and Magick++, which are absent, so oracle/Makefile extracts that one
// template from the file where it lies into _ref/limit_extract.inc and this
// driver compiles it with the reference's own flags, after the reference's
// matrix header (Map = ArrayF<2>, a blitz::Array<float, 2>), as
// external.world.cpp reaches it.
#include <climits>
#include <cstdint>
#include <limits>

#include "matrix.world.h"

using namespace std;

#include "limit_extract.inc"

namespace {

template <class T>
void run(const float *img, long rows, long cols, float mincon, float maxcon, void *out) {
  Map m(const_cast<float *>(img), blitz::shape(rows, cols), blitz::neverDeleteData);
  const blitz::Array<T, 2> r = limit<T>(m, mincon, maxcon);
  T *o = static_cast<T *>(out);
  for (long y = 0; y < rows; y++)
    for (long x = 0; x < cols; x++) o[y * cols + x] = r(y, x);
}

}  // namespace

extern "C" {

// bpp: 8, -8, 16, -16 (negative = signed), the sample types of the 8- and
// 16-bit writers (external.world.cpp:689-692).  Returns 0, or -1 for another
// bpp.
int ref_limit(const float *img, long rows, long cols, int bpp, float mincon, float maxcon,
              void *out) {
  switch (bpp) {
    case 8: run<unsigned char>(img, rows, cols, mincon, maxcon, out); return 0;
    case -8: run<char>(img, rows, cols, mincon, maxcon, out); return 0;
    case 16: run<unsigned short>(img, rows, cols, mincon, maxcon, out); return 0;
    case -16: run<short>(img, rows, cols, mincon, maxcon, out); return 0;
    default: return -1;
  }
}

}  // extern "C"

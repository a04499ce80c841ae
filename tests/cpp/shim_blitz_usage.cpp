// The C++ mirror of the reconstruction interface used with the reference's own
// array type, blitz::Array<float,2> (the `Map` of matrix.world.h:127-129), the
// way the ctas tools use CTrec: construction from an array's shape and a
// per-thread clone (ct.cpp:178-191), the filter-once / backproject-many calls
// of the axis tool including recr.resize(rec->recShape()) (axis.cpp:143-155),
// and recCrop (ct.h:276-279, used as in lct.cpp:876-877).  Built against the
// reference's Blitz++ headers where they are available.  Exit status 0 when
// sino() + repeat() equals reconstruct() bit for bit and the crop has the
// shape recShape() gives.
#include <blitz/array.h>

#include <cmath>
#include <cstdio>

#include "ctas_ct.hpp"

using namespace ctas_b200;
typedef blitz::Array<float, 2> BMap;

int main() {
  BMap sino(180, 256);
  for (int n = 0; n < 180; n++)
    for (int k = 0; k < 256; k++)
      sino(n, k) = 1.0f + 0.25f * std::sin(0.05f * (float)(k + 3 * n)) * std::exp(-0.0001f * (k - 128) * (k - 128));
  try {
    CTrec canon(sino.shape(), Contrast::ABS, 180.0f, Filter("RAMP"));
    CTrec rec(canon);
    rec.setPhysics(0.0f, 0.0f);
    BMap once(sino.copy()), slice;
    rec.reconstruct(once, slice, -1.5f);

    BMap _sino(sino.copy());
    rec.sino(_sino);
    BMap recr;
    recr.resize(rec.recShape());
    rec.repeat(recr, -1.5f);
    if (recr.extent(0) != 256 || recr.extent(1) != 256) return 2;
    for (int j = 0; j < 256; j++)
      for (int i = 0; i < 256; i++)
        if (recr(j, i) != slice(j, i)) return 3;

    const RecCrop crp = rec.recCrop(-1.5f);
    const RecShape oosh = crp.shape(recr.extent(0), recr.extent(1));
    BMap cropped(recr(blitz::Range(crp.rows.begin(), crp.rows.end(recr.extent(0)) - 1),
                      blitz::Range::all()));
    blitz::TinyVector<ssize_t, 2> as_shape = rec.recShape(-1.5f);
    if (cropped.extent(0) != oosh.rows || as_shape(0) != oosh.rows || oosh.rows != 254) return 4;
  } catch (const CtasErr &e) {
    std::fprintf(stderr, "CtasErr %d: %s\n", e.code, e.what());
    return 1;
  }
  std::printf("ok\n");
  return 0;
}

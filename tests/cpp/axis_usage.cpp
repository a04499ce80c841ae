// Uses the C++ mirror of the axis search the way the axis tool does
// (axis.cpp:117-170): raxis with each algorithm on one sinogram, then the
// average gradient at the centre.
// Usage: axis_usage <N> <W> <max_dev> <in.f32>
//   in.f32 holds an N x W float32 transmission sinogram; prints five numbers:
//   the axis positions for algorithms 0..3 ("err" where raxis throws) and the
//   average gradient at 0.5 (W-1).
#include <cstdio>
#include <cstdlib>

#include "ctas_ct.hpp"

using namespace ctas_b200;

int main(int argc, char **argv) {
  if (argc != 5) {
    std::fprintf(stderr, "usage: %s N W max_dev in.f32\n", argv[0]);
    return 2;
  }
  const long N = std::atol(argv[1]), W = std::atol(argv[2]);
  const float max_dev = (float)std::atof(argv[3]);
  Map sino(N, W);
  FILE *f = std::fopen(argv[4], "rb");
  if (!f || std::fread(sino.data(), sizeof(float), (size_t)(N * W), f) != (size_t)(N * W)) return 3;
  std::fclose(f);
  try {
    for (int algo = 0; algo < 4; algo++) {
      try {
        std::printf("%.6f ", raxis(sino, 180.0f, max_dev, algo));
      } catch (const CtasErr &) {  // e.g. an estimate beyond max_dev
        std::printf("err ");
      }
    }
    AverageGradient ag(sino, 180.0f);
    std::printf("%.9g\n", ag.apply(0.5f * (W - 1)));
    try {
      raxis(sino, 90.0f, max_dev, 1);  // arc below 180 degrees must throw
      return 5;
    } catch (const CtasErr &e) {
      if (e.code != CTAS_E_ARG) return 6;
    }
  } catch (const CtasErr &e) {
    std::fprintf(stderr, "CtasErr %d: %s\n", e.code, e.what());
    return 1;
  }
  return 0;
}

// Uses the C++ mirror of ts_add the way the ts tool does (ts.cpp:209-217):
// one call per projection image, the result accumulated across calls.
// Usage: ts_usage <rows> <pixels> <n> <in.f32> <out.f32>
//   in.f32 holds n rows x pixels absorption images taken at angles
//   -0.3 + 0.6 i / (n - 1); out.f32 receives the result image.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "ctas_ct.hpp"

using namespace ctas_b200;

int main(int argc, char **argv) {
  if (argc != 6) {
    std::fprintf(stderr, "usage: %s rows pixels n in.f32 out.f32\n", argv[0]);
    return 2;
  }
  const long rows = std::atol(argv[1]), pix = std::atol(argv[2]), n = std::atol(argv[3]);
  std::vector<float> all((size_t)(rows * pix * n));
  FILE *f = std::fopen(argv[4], "rb");
  if (!f || std::fread(all.data(), sizeof(float), all.size(), f) != all.size()) return 3;
  std::fclose(f);
  Map proj(rows, pix), result(rows, pix);
  try {
    for (long i = 0; i < n; i++) {
      for (long k = 0; k < rows * pix; k++) proj.data()[k] = all[(size_t)(i * rows * pix + k)];
      const float angle = -0.3f + 0.6f * (float)i / (float)(n > 1 ? n - 1 : 1);
      ts_add(proj, result, Filter(), 1.5f, Contrast("ABS"), angle, 12);
    }
  } catch (const CtasErr &e) {
    std::fprintf(stderr, "CtasErr %d: %s\n", e.code, e.what());
    return 1;
  }
  FILE *o = std::fopen(argv[5], "wb");
  std::fwrite(result.data(), sizeof(float), (size_t)(rows * pix), o);
  std::fclose(o);
  return 0;
}

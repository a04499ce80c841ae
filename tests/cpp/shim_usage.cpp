// Uses the C++ mirror of the ctas reconstruction interface the way the ct
// tool uses CTrec (ct.cpp:178-202): one canonical object, a per-thread clone,
// setPhysics, reconstruct, then repeat with another centre.
// Usage: shim_usage <N> <W> <center> <in.f32> <out.f32>
//   in.f32 holds N*W float32 samples; out.f32 receives two W*W slices
//   (reconstruct at <center>, then repeat at -<center>).
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "ctas_ct.hpp"

using namespace ctas_b200;

int main(int argc, char **argv) {
  if (argc != 6) {
    std::fprintf(stderr, "usage: %s N W center in.f32 out.f32\n", argv[0]);
    return 2;
  }
  const long N = std::atol(argv[1]), W = std::atol(argv[2]);
  const float center = (float)std::atof(argv[3]);
  Map sino(N, W), slice, slice2;
  FILE *f = std::fopen(argv[4], "rb");
  if (!f || std::fread(sino.data(), sizeof(float), (size_t)(N * W), f) != (size_t)(N * W)) return 3;
  std::fclose(f);
  try {
    Filter ft("HANN");
    Filter parsed;
    if (!_conversion(&parsed, "hamming")) return 4;
    CTrec canon(std::array<long, 2>{N, W}, Contrast("PHS"), 180.0f, ft);
    CTrec rec(canon);
    rec.setPhysics(0.0f, 0.0f);
    rec.reconstruct(sino, slice, center);
    rec.repeat(slice2, -center);
    try {
      rec.repeat(slice2, (float)W);  // |center| >= W/2 must throw
      return 5;
    } catch (const CtasErr &e) {
      if (e.code != CTAS_E_CENTER) return 6;
    }
  } catch (const CtasErr &e) {
    std::fprintf(stderr, "CtasErr %d: %s\n", e.code, e.what());
    return 1;
  }
  FILE *o = std::fopen(argv[5], "wb");
  std::fwrite(slice.data(), sizeof(float), (size_t)(W * W), o);
  std::fwrite(slice2.data(), sizeof(float), (size_t)(W * W), o);
  std::fclose(o);
  std::printf("ok\n");
  return 0;
}

// The ct tool's slice loop (ct.cpp:156-206) over a volume of sinograms, with
// the C++ mirror: CTrec set up as RecInThread does, then one streamed call
// that reads sinograms from a raw float32 file and writes the slices as bpp
// samples (the tool's -i/-m/-M) to another.
// Usage: volume_usage <slices> <projections> <pixels> <center> <bpp> <min> <max> <in.f32> <out>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "ctas_ct.hpp"

using namespace ctas_b200;

int main(int argc, char **argv) {
  if (argc != 10) {
    std::fprintf(stderr, "usage: %s slices projections pixels center bpp min max in.f32 out\n",
                 argv[0]);
    return 2;
  }
  const long S = std::atol(argv[1]), N = std::atol(argv[2]), W = std::atol(argv[3]);
  const float center = (float)std::atof(argv[4]);
  const int bpp = std::atoi(argv[5]);
  const float mincon = (float)std::atof(argv[6]), maxcon = (float)std::atof(argv[7]);
  FILE *in = std::fopen(argv[8], "rb");
  FILE *out = std::fopen(argv[9], "wb");
  if (!in || !out) return 3;
  const long sb = ctas_vol_sample_bytes(bpp);
  try {
    CTrec rec(std::array<int64_t, 2>{N, W}, Contrast("PHS"), 180, Filter("HANN"));
    rec.setPhysics(0, 0);
    reconstruct_volume(
        rec, S, center,
        [&](int64_t first, int64_t count, float *sinos) {
          std::fseek(in, (long)(first * N * W * sizeof(float)), SEEK_SET);
          if (std::fread(sinos, sizeof(float), (size_t)(count * N * W), in) !=
              (size_t)(count * N * W))
            throw CtasErr(CTAS_E_IO, "short read");
        },
        [&](int64_t first, int64_t count, const void *slices) {
          std::fseek(out, (long)(first * W * W * sb), SEEK_SET);
          std::fwrite(slices, (size_t)sb, (size_t)(count * W * W), out);
        },
        bpp, mincon, maxcon);
  } catch (const CtasErr &e) {
    std::fprintf(stderr, "CtasErr %d: %s\n", e.code, e.what());
    return 1;
  }
  std::fclose(in);
  std::fclose(out);
  return 0;
}

// Exercises the header-only C++ mirror (include/bimp/bimp.hpp) the way the
// reference's demo uses bimp::Context (example_bimp.cpp:37-65): image in,
// std::vector<KeyPoint> out.  Reads a raw grey image (width height file),
// writes one "x y size response octave" line per keypoint to stdout.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "bimp/bimp.hpp"

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s width height image.raw [lambdas...]\n", argv[0]);
    return 2;
  }
  const int w = std::atoi(argv[1]), h = std::atoi(argv[2]);
  std::vector<unsigned char> img(static_cast<size_t>(w) * h);
  FILE* f = std::fopen(argv[3], "rb");
  if (!f || std::fread(img.data(), 1, img.size(), f) != img.size()) {
    std::fprintf(stderr, "cannot read %s\n", argv[3]);
    return 2;
  }
  std::fclose(f);
  std::vector<float> lambdas;
  for (int i = 4; i < argc; ++i) lambdas.push_back(static_cast<float>(std::atof(argv[i])));
  if (lambdas.empty()) lambdas = bimp::cuda::makeLambdasLog(4, 64, 2);
  try {
    bimp::ImageView v;
    v.data = img.data();
    v.rows = h;
    v.cols = w;
    v.step = static_cast<size_t>(w);
    bimp::Context ctx(v, lambdas);
    ctx.capacity = 1 << 20;
    const std::vector<bimp::KeyPoint> pts = ctx.getKeypointsAndDownload();
    for (const auto& k : pts)
      std::printf("%.9g %.9g %.9g %.9g %d %d %.1f\n", k.pt.x, k.pt.y, k.size, k.response, k.octave, k.class_id,
                  k.angle);
    std::fprintf(stderr, "%zu keypoints\n", pts.size());
  } catch (const bimp::Error& e) {
    std::fprintf(stderr, "bimp error %d: %s\n", e.code(), e.what());
    return 1;
  }
  return 0;
}

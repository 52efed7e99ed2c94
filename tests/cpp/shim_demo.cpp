// Exercises the header-only C++ mirror (include/bimp/bimp.hpp) the way the
// reference's demo uses bimp::Context (example_bimp.cpp:37-65): image in,
// std::vector<KeyPoint> out.  Reads a raw uint8 image (width height channels
// file; channels 1 = grey, 3 = BGR) and writes to stdout:
//   one "kp x y size response octave class_id angle" line per keypoint (from
//   the device 7 x n matrix of Context::getKeypoints(), downloaded);
//   "ctx width height found" (the uploaded image's size, as Context::width());
//   "lowlevel found same" (bimp::cuda::getKeypoints on the context's device
//   image: its count, and 1 if its records equal the context's);
//   one "resp scale data_w data_h maxD sumD sumS" line per scale
//   (Context::downloadResultsToCPU());
//   "color n sum" for a BGR image (Context::getColorFeatures()).
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "bimp/bimp.hpp"

int main(int argc, char** argv) {
  if (argc < 5) {
    std::fprintf(stderr, "usage: %s width height channels image.raw [lambdas...]\n", argv[0]);
    return 2;
  }
  const int w = std::atoi(argv[1]), h = std::atoi(argv[2]), ch = std::atoi(argv[3]);
  std::vector<unsigned char> img(static_cast<size_t>(w) * h * ch);
  FILE* f = std::fopen(argv[4], "rb");
  if (!f || std::fread(img.data(), 1, img.size(), f) != img.size()) {
    std::fprintf(stderr, "cannot read %s\n", argv[4]);
    return 2;
  }
  std::fclose(f);
  std::vector<float> lambdas;
  for (int i = 5; i < argc; ++i) lambdas.push_back(static_cast<float>(std::atof(argv[i])));
  if (lambdas.empty()) lambdas = bimp::cuda::makeLambdasLog(4, 64, 2);
  try {
    bimp::ImageView v;
    v.data = img.data();
    v.rows = h;
    v.cols = w;
    v.channels = ch;
    v.step = static_cast<size_t>(w) * ch;
    bimp::Context ctx(v, lambdas);
    ctx.capacity = 1 << 20;
    bimp::DeviceMat& kp = ctx.getKeypoints();
    const std::vector<bimp::KeyPoint> pts = bimp::utils::downloadKeypoints(kp);
    for (const auto& k : pts)
      std::printf("kp %.9g %.9g %.9g %.9g %d %d %.1f\n", k.pt.x, k.pt.y, k.size, k.response, k.octave, k.class_id,
                  k.angle);
    std::printf("ctx %d %d %d\n", ctx.width(), ctx.height(), ctx.found);
    // the lower-level pair on the context's device image (GpuMat getKeypoints(GpuMat&, CudaStuff&))
    int found = 0;
    bimp::DeviceMat low = bimp::cuda::getKeypoints(ctx.current_image.data, ctx.current_image.step, ctx.cuda_data,
                                                   1 << 20, &found);
    const std::vector<bimp::KeyPoint> pts2 = bimp::utils::downloadKeypoints(low);
    bool same = pts2.size() == pts.size();
    for (size_t i = 0; same && i < pts.size(); ++i)
      same = pts2[i].pt.x == pts[i].pt.x && pts2[i].pt.y == pts[i].pt.y && pts2[i].response == pts[i].response;
    std::printf("lowlevel %d %d\n", found, same ? 1 : 0);
    for (const auto& r : ctx.downloadResultsToCPU()) {
      double mx = -1e300, sd = 0, ss = 0;
      for (float x : r.h_ResultDouble) {
        mx = x > mx ? x : mx;
        sd += x;
      }
      for (float x : r.h_ResultSingle) ss += x;
      std::printf("resp %d %d %d %.9g %.9g %.9g\n", r.info.margin, r.info.data_w, r.info.data_h, mx, sd, ss);
    }
    if (ch == 3) {
      const std::vector<float> feats = ctx.getColorFeatures();
      double sum = 0;
      for (float x : feats) sum += x;
      std::printf("color %zu %.9g\n", feats.size() / 24, sum);
    }
    std::fprintf(stderr, "%zu keypoints\n", pts.size());
  } catch (const bimp::Error& e) {
    std::fprintf(stderr, "bimp error %d: %s\n", e.code(), e.what());
    return 1;
  }
  return 0;
}

// bimp/bimp.hpp -- header-only C++ mirror of the daniel-koudouna/cuda-bimp
// keypoint API over the C ABI (bimp_b200.h).
//
//   bimp::cuda::CudaStuff(int w, int h, std::vector<float> lambdas)
//        bimp/include/detection/cuda_bimp.hpp:92-100
//   int bimp::cuda::getKeypoints(device image, CudaStuff&, device 7 x N out)
//        bimp/include/detection/cuda_bimp.hpp:111
//   bimp::cuda::makeLambdasLog / makeLambdasLin / snapTransformSize
//        bimp/include/detection/cuda_bimp.hpp:140,146
//   bimp::utils::downloadKeypoints / uploadKeypoints
//        bimp/include/detection/utils.hpp:30-32
//   bimp::Context(image), getKeypointsAndDownload(), loadImage(), width(),
//   height()        bimp/include/detection/bimp.hpp:19-51
//
// Without OpenCV the header defines a layout-compatible bimp::KeyPoint and a
// plain image view; with -DBIMP_WITH_OPENCV it uses cv::KeyPoint and accepts
// cv::Mat.  Errors throw bimp::Error carrying the C status code (the
// reference exit()s instead).  Link with -lbimp_b200.
#pragma once

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "bimp_b200.h"

#ifdef BIMP_WITH_OPENCV
#include <opencv2/core.hpp>
#endif

namespace bimp {

#ifdef BIMP_WITH_OPENCV
using KeyPoint = cv::KeyPoint;
#else
struct Point2f {
  float x, y;
};
// Field-for-field stand-in of cv::KeyPoint.
struct KeyPoint {
  Point2f pt;
  float size;
  float angle;
  float response;
  int octave;
  int class_id;
};
#endif
static_assert(sizeof(KeyPoint) == sizeof(bimp_keypoint), "KeyPoint must match the C record");

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string& what) : std::runtime_error(what), code_(code) {}
  int code() const { return code_; }

 private:
  int code_;
};

inline void check(int rc, const char* where) {
  if (rc != BIMP_OK) throw Error(rc, std::string(where) + ": " + bimp_last_error());
}

// Grey uint8 host image (stand-in for a CV_8UC1 cv::Mat).
struct ImageView {
  const uint8_t* data = nullptr;
  int rows = 0, cols = 0;
  size_t step = 0;   // bytes per row
};

namespace cuda {

constexpr int KP_VECTOR_LENGTH = BIMP_KP_VECTOR_LENGTH;
constexpr int KP_MAX_POINTS = BIMP_KP_MAX_POINTS;

inline int snapTransformSize(int n) { return bimp_snap_transform_size(n); }

inline std::vector<float> makeLambdasLog(float start, float end, int scalesPerOctave) {
  int n = 0;
  check(bimp_make_lambdas_log(start, end, scalesPerOctave, nullptr, 0, &n), "makeLambdasLog");
  std::vector<float> v(static_cast<size_t>(n));
  check(bimp_make_lambdas_log(start, end, scalesPerOctave, v.data(), n, &n), "makeLambdasLog");
  return v;
}

inline std::vector<float> makeLambdasLin(float start, float end, int numScales) {
  std::vector<float> v(static_cast<size_t>(numScales > 0 ? numScales : 0));
  int n = 0;
  check(bimp_make_lambdas_lin(start, end, numScales, v.data(), numScales, &n), "makeLambdasLin");
  v.resize(static_cast<size_t>(n));
  return v;
}

// Filter bank and per-frame buffers for one image size on the current device.
class CudaStuff {
 public:
  CudaStuff(int width, int height, std::vector<float> lambdas, const bimp_params* params = nullptr) {
    check(bimp_ctx_create(&ctx_, width, height, lambdas.data(), static_cast<int>(lambdas.size()), params),
          "CudaStuff");
    const int n = bimp_ctx_num_scales(ctx_);
    ks.resize(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) check(bimp_ctx_scale_info(ctx_, i, &ks[static_cast<size_t>(i)]), "CudaStuff");
    width_ = width;
    height_ = height;
  }
  ~CudaStuff() { bimp_ctx_destroy(ctx_); }
  CudaStuff(const CudaStuff&) = delete;
  CudaStuff& operator=(const CudaStuff&) = delete;
  CudaStuff(CudaStuff&& o) noexcept : ks(std::move(o.ks)), ctx_(o.ctx_), width_(o.width_), height_(o.height_) {
    o.ctx_ = nullptr;
  }

  bimp_context* handle() const { return ctx_; }
  int width() const { return width_; }
  int height() const { return height_; }

  std::vector<bimp_scale_info> ks;   // per-scale geometry (CudaKernels fields)

 private:
  bimp_context* ctx_ = nullptr;
  int width_ = 0, height_ = 0;
};

// int getKeypoints(GpuMat& input, GpuMat& output, CudaStuff& cs): device grey
// image in, keypoints into the device 7 x ld matrix `d_out`.  Returns the
// number found; like the reference, only the first `capacity` are written.
inline int getKeypoints(const uint8_t* d_image, size_t pitch, CudaStuff& cs, float* d_out, size_t ld,
                        int capacity = KP_MAX_POINTS, void* stream = nullptr) {
  int n = 0;
  const int rc = bimp_detect_device(cs.handle(), d_image, pitch, cs.width(), cs.height(), d_out, ld, capacity, &n,
                                    stream);
  if (rc != BIMP_OK && rc != BIMP_ERR_CAPACITY) check(rc, "getKeypoints");
  return n;
}

}  // namespace cuda

namespace utils {

// downloadKeypoints (utils.cpp:130-150).
inline std::vector<KeyPoint> downloadKeypoints(const float* d_kp, size_t ld, int n, void* stream = nullptr) {
  std::vector<KeyPoint> out(static_cast<size_t>(n));
  check(bimp_download_keypoints(d_kp, ld, n, reinterpret_cast<bimp_keypoint*>(out.data()), stream),
        "downloadKeypoints");
  return out;
}

// uploadKeypoints (utils.cpp:109-128).
inline void uploadKeypoints(const std::vector<KeyPoint>& points, float* d_kp, size_t ld, void* stream = nullptr) {
  check(bimp_upload_keypoints(reinterpret_cast<const bimp_keypoint*>(points.data()), static_cast<int>(points.size()),
                              d_kp, ld, stream),
        "uploadKeypoints");
}

}  // namespace utils

// bimp::Context for the keypoint path: the bank is makeLambdasLog(4, 64, 2)
// (bimp.cpp:8); keypoints are computed on first request and cached until
// loadImage() (bimp.cpp:61-73, 106-117).
class Context {
 public:
  explicit Context(const ImageView& image, std::vector<float> lambdas = cuda::makeLambdasLog(4, 64, 2),
                   const bimp_params* params = nullptr)
      : cuda_data(image.cols, image.rows, std::move(lambdas), params) {
    loadImage(image);
  }
#ifdef BIMP_WITH_OPENCV
  explicit Context(const cv::Mat& gray) : Context(view(gray)) {}
  void loadImage(const cv::Mat& gray) { loadImage(view(gray)); }
#endif

  void loadImage(const ImageView& image) {
    if (image.cols != cuda_data.width() || image.rows != cuda_data.height())
      throw Error(BIMP_ERR_INVALID, "loadImage: size differs from the context's");
    image_ = image;
    has_changed_keypoints = true;
  }

  std::vector<KeyPoint> getKeypointsAndDownload() {
    if (has_changed_keypoints) {
      keypoints_.resize(static_cast<size_t>(capacity));
      int n = 0;
      const int rc = bimp_detect_host(cuda_data.handle(), image_.data, image_.step, image_.cols, image_.rows,
                                      reinterpret_cast<bimp_keypoint*>(keypoints_.data()), capacity, &n, nullptr);
      if (rc != BIMP_OK && rc != BIMP_ERR_CAPACITY) check(rc, "getKeypointsAndDownload");
      keypoints_.resize(static_cast<size_t>(n < capacity ? n : capacity));
      found = n;
      has_changed_keypoints = false;
    }
    return keypoints_;
  }

  int width() const { return cuda_data.width(); }
  int height() const { return cuda_data.height(); }

  cuda::CudaStuff cuda_data;
  bool has_changed_keypoints = true;
  int capacity = cuda::KP_MAX_POINTS;   // keypoint limit, as KP_MAX_POINTS
  int found = 0;                        // count before truncation to `capacity`

 private:
#ifdef BIMP_WITH_OPENCV
  static ImageView view(const cv::Mat& m) {
    if (m.type() != CV_8UC1) throw Error(BIMP_ERR_INVALID, "Context expects a CV_8UC1 image");
    ImageView v;
    v.data = m.data;
    v.rows = m.rows;
    v.cols = m.cols;
    v.step = m.step;
    return v;
  }
#endif
  ImageView image_;
  std::vector<KeyPoint> keypoints_;
};

}  // namespace bimp

// bimp/bimp.hpp -- header-only C++ mirror of the daniel-koudouna/cuda-bimp
// keypoint API over the C ABI (bimp_b200.h).
//
//   bimp::cuda::CudaStuff(int w, int h, std::vector<float> lambdas)
//        bimp/include/detection/cuda_bimp.hpp:92-100
//   int bimp::cuda::getKeypoints(device image, CudaStuff&, device 7 x N out)
//        bimp/include/detection/cuda_bimp.hpp:111
//   bimp::cuda::getGPUImage(image, grayscale)
//        bimp/include/detection/cuda_bimp.hpp:119, bimp/src/cuda_bimp.cu:156-180
//   bimp::cuda::makeLambdasLog / makeLambdasLin / snapTransformSize
//        bimp/include/detection/cuda_bimp.hpp:140,146
//   bimp::utils::downloadKeypoints / uploadKeypoints
//        bimp/include/detection/utils.hpp:30-32
//   bimp::Context(image), getKeypoints(), getKeypointsAndDownload(),
//   getResponses(), downloadResultsToCPU(), loadImage(host or device image),
//   width(), height()      bimp/include/detection/bimp.hpp:19-51,
//                          bimp/src/bimp.cpp:7-129
//   (the colour histogram of addColorFeatures, bimp/src/bimp.cpp:42-43, as
//   Context::getColorFeatures(); SURF descriptors and matching are not part
//   of this library)
//
// Without OpenCV the header defines a layout-compatible bimp::KeyPoint, a
// host image view and an owning device matrix (bimp::DeviceMat, the stand-in
// for cv::cuda::GpuMat: rows x cols elements, `step` bytes per row); with
// -DBIMP_WITH_OPENCV it uses cv::KeyPoint and accepts cv::Mat.  Errors throw
// bimp::Error carrying the C status code (the reference exit()s instead).
// Link with -lbimp_b200.
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

// uint8 host image (stand-in for a CV_8UC1 or CV_8UC3 BGR cv::Mat).
struct ImageView {
  const uint8_t* data = nullptr;
  int rows = 0, cols = 0;
  size_t step = 0;     // bytes per row
  int channels = 1;    // 1 (grey) or 3 (BGR)
};

// Owning device matrix, the stand-in for cv::cuda::GpuMat: rows x cols
// elements of elem_size bytes, `step` bytes per row.  `cols` may be set below
// the allocated width (as GpuMat::colRange keeps the step).
class DeviceMat {
 public:
  DeviceMat() = default;
  DeviceMat(int rows, int cols, size_t elem_size) { create(rows, cols, elem_size); }
  ~DeviceMat() { release(); }
  DeviceMat(const DeviceMat&) = delete;
  DeviceMat& operator=(const DeviceMat&) = delete;
  DeviceMat(DeviceMat&& o) noexcept { *this = std::move(o); }
  DeviceMat& operator=(DeviceMat&& o) noexcept {
    if (this != &o) {
      release();
      data = o.data; step = o.step; rows = o.rows; cols = o.cols; elem = o.elem; alloc_cols = o.alloc_cols;
      o.data = nullptr; o.rows = o.cols = o.alloc_cols = 0; o.step = 0;
    }
    return *this;
  }
  // GpuMat::create: keeps the allocation when it already has this shape.
  void create(int rows_, int cols_, size_t elem_size) {
    if (data && rows == rows_ && alloc_cols == cols_ && elem == elem_size) {
      cols = cols_;
      return;
    }
    release();
    const size_t row_bytes = static_cast<size_t>(cols_) * elem_size;
    const size_t pitch = (row_bytes + 255) / 256 * 256;
    void* p = nullptr;
    check(bimp_device_alloc(&p, pitch * static_cast<size_t>(rows_)), "DeviceMat::create");
    data = static_cast<uint8_t*>(p);
    step = pitch;
    rows = rows_;
    cols = alloc_cols = cols_;
    elem = elem_size;
  }
  void release() {
    if (data) bimp_device_free(data);
    data = nullptr;
    rows = cols = alloc_cols = 0;
    step = 0;
  }
  bool empty() const { return data == nullptr || rows == 0 || cols == 0; }
  template <typename T>
  T* ptr(int y = 0) const { return reinterpret_cast<T*>(data + static_cast<size_t>(y) * step); }
  // GpuMat::upload / download of rows x cols elements.
  void upload(const void* host, size_t host_step) {
    check(bimp_copy_2d(data, step, host, host_step, static_cast<size_t>(cols) * elem, static_cast<size_t>(rows),
                       nullptr),
          "DeviceMat::upload");
  }
  void download(void* host, size_t host_step) const {
    check(bimp_copy_2d(host, host_step, data, step, static_cast<size_t>(cols) * elem, static_cast<size_t>(rows),
                       nullptr),
          "DeviceMat::download");
  }

  uint8_t* data = nullptr;
  size_t step = 0;
  int rows = 0, cols = 0;
  size_t elem = 1;

 private:
  int alloc_cols = 0;
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
// input_width / input_height (default: the same) are the size of the images a
// detection takes; larger inputs are filtered on the top-left window of each
// pyramid level, as the reference's Context does for upscaled small images
// (bimp_ctx_create_for_input).
class CudaStuff {
 public:
  CudaStuff(int width, int height, std::vector<float> lambdas, const bimp_params* params = nullptr,
            int input_width = 0, int input_height = 0) {
    in_width_ = input_width > 0 ? input_width : width;
    in_height_ = input_height > 0 ? input_height : height;
    check(bimp_ctx_create_for_input(&ctx_, width, height, in_width_, in_height_, lambdas.data(),
                                    static_cast<int>(lambdas.size()), params),
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
  CudaStuff(CudaStuff&& o) noexcept
      : ks(std::move(o.ks)), ctx_(o.ctx_), width_(o.width_), height_(o.height_), in_width_(o.in_width_),
        in_height_(o.in_height_) {
    o.ctx_ = nullptr;
  }

  bimp_context* handle() const { return ctx_; }
  int width() const { return width_; }
  int height() const { return height_; }
  int input_width() const { return in_width_; }
  int input_height() const { return in_height_; }

  std::vector<bimp_scale_info> ks;   // per-scale geometry (CudaKernels fields)

 private:
  bimp_context* ctx_ = nullptr;
  int width_ = 0, height_ = 0, in_width_ = 0, in_height_ = 0;
};

// int getKeypoints(GpuMat& input, GpuMat& output, CudaStuff& cs): device grey
// image in, keypoints into the device 7 x ld matrix `d_out`.  Returns the
// number found; like the reference, only the first `capacity` are written.
inline int getKeypoints(const uint8_t* d_image, size_t pitch, CudaStuff& cs, float* d_out, size_t ld,
                        int capacity = KP_MAX_POINTS, void* stream = nullptr) {
  int n = 0;
  const int rc = bimp_detect_device(cs.handle(), d_image, pitch, cs.input_width(), cs.input_height(), d_out, ld,
                                    capacity, &n, stream);
  if (rc != BIMP_OK && rc != BIMP_ERR_CAPACITY) check(rc, "getKeypoints");
  return n;
}

// GpuMat getKeypoints(GpuMat& input, CudaStuff& cs), bimp/src/cuda_bimp.cu:129-140:
// a fresh 7 x capacity device matrix whose `cols` is set to the keypoints
// kept (as the reference's colRange view); more than `capacity` found are
// truncated, as the reference warns and truncates.  `found` (optional)
// receives the count before truncation.
inline DeviceMat getKeypoints(const uint8_t* d_image, size_t pitch, CudaStuff& cs, int capacity = KP_MAX_POINTS,
                              int* found = nullptr) {
  DeviceMat kp(KP_VECTOR_LENGTH, capacity, sizeof(float));
  const int n = getKeypoints(d_image, pitch, cs, kp.ptr<float>(), kp.step / sizeof(float), capacity);
  if (found) *found = n;
  kp.cols = n < capacity ? n : capacity;
  return kp;
}

// getGPUImage(cv::Mat&, bool grayscale), bimp/src/cuda_bimp.cu:156-180: the
// host image uploaded, upscaled when a side is below 350 pixels, and for a
// 3-channel BGR image with grayscale set converted to grey.
inline DeviceMat getGPUImage(const ImageView& in, bool grayscale = true) {
  if (!in.data || in.rows < 1 || in.cols < 1 || (in.channels != 1 && in.channels != 3))
    throw Error(BIMP_ERR_INVALID, "getGPUImage: expected a grey or BGR uint8 image");
  int ow = 0, oh = 0;
  check(bimp_min_size_dims(in.cols, in.rows, &ow, &oh, nullptr), "getGPUImage");
  DeviceMat src(in.rows, in.cols * in.channels, 1);
  src.upload(in.data, in.step);
  const int out_ch = (grayscale && in.channels == 3) ? 1 : in.channels;
  DeviceMat dst(oh, ow * out_ch, 1);
  check(bimp_gpu_image(src.data, src.step, in.cols, in.rows, in.channels, grayscale ? 1 : 0, dst.data, dst.step,
                       nullptr),
        "getGPUImage");
  return dst;
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
// The same for a 7 x n device matrix (the GpuMat overload of the reference).
inline std::vector<KeyPoint> downloadKeypoints(const DeviceMat& kp) {
  return downloadKeypoints(kp.ptr<float>(), kp.step / sizeof(float), kp.cols);
}

// uploadKeypoints (utils.cpp:109-128).
inline void uploadKeypoints(const std::vector<KeyPoint>& points, float* d_kp, size_t ld, void* stream = nullptr) {
  check(bimp_upload_keypoints(reinterpret_cast<const bimp_keypoint*>(points.data()), static_cast<int>(points.size()),
                              d_kp, ld, stream),
        "uploadKeypoints");
}

}  // namespace utils

// One scale's responses (the geometry and result fields of the reference's
// CudaKernels): the summed keypoint map D (k.d_ResultDouble) and the
// single-stopped map S (k.d_ResultSingle), data_h x data_w floats on the
// device; the host copies are filled by Context::downloadResultsToCPU().
struct ScaleResponses {
  bimp_scale_info info{};
  DeviceMat d_ResultDouble, d_ResultSingle;
  std::vector<float> h_ResultDouble, h_ResultSingle;
};

// bimp::Context for the keypoint path (bimp.cpp:7-129).  As in the
// reference: the bank is makeLambdasLog(4, 64, 2) (bimp.cpp:8); the image
// goes through getGPUImage (grey, upscaled when a side is below 350 pixels;
// the colour image is kept for the colour histogram); CudaStuff is built from
// the image's own size (bimp.cpp:7-8), so for an upscaled image each scale
// filters the top-left window of its pyramid level (bimp_ctx_create_for_input
// reproduces this); keypoints are computed on first request and cached until
// loadImage() (bimp.cpp:61-73, 106-117).  width()/height() are those of the
// uploaded (possibly upscaled) image, as current_image's in the reference.
class Context {
 public:
  explicit Context(const ImageView& image, std::vector<float> lambdas = cuda::makeLambdasLog(4, 64, 2),
                   const bimp_params* params = nullptr)
      : cuda_data(image.cols, image.rows, std::move(lambdas), params, min_size(image).first,
                  min_size(image).second) {
    loadImage(image);
  }
#ifdef BIMP_WITH_OPENCV
  explicit Context(const cv::Mat& image) : Context(view(image)) {}
  void loadImage(const cv::Mat& image) { loadImage(view(image)); }
#endif

  // loadImage(cv::Mat): through getGPUImage; the result must have the size
  // the context was built for.
  void loadImage(const ImageView& image) {
    DeviceMat grey = cuda::getGPUImage(image, true);
    if (grey.cols != cuda_data.input_width() || grey.rows != cuda_data.input_height())
      throw Error(BIMP_ERR_INVALID, "loadImage: size differs from the context's");
    current_image = std::move(grey);
    if (image.channels == 3) current_image_color = cuda::getGPUImage(image, false);
    else current_image_color.release();
    has_changed_keypoints = true;
  }
  // loadImage(cv::cuda::GpuMat): a grey device image of the context's size
  // (copied; the reference shares the GpuMat).
  void loadImage(const uint8_t* d_grey, size_t pitch, int cols, int rows) {
    if (cols != cuda_data.input_width() || rows != cuda_data.input_height())
      throw Error(BIMP_ERR_INVALID, "loadImage: size differs from the context's");
    current_image.create(rows, cols, 1);
    check(bimp_copy_2d(current_image.data, current_image.step, d_grey, pitch, static_cast<size_t>(cols),
                       static_cast<size_t>(rows), nullptr),
          "loadImage");
    current_image_color.release();
    has_changed_keypoints = true;
  }

  // cv::cuda::GpuMat& getKeypoints(): the device 7 x n SURF-layout matrix
  // (rows X, Y, LAPLACIAN, OCTAVE, SIZE, ANGLE, HESSIAN; n <= capacity).
  DeviceMat& getKeypoints() {
    if (has_changed_keypoints) {
      current_keypoints.create(cuda::KP_VECTOR_LENGTH, capacity, sizeof(float));
      found = cuda::getKeypoints(current_image.data, current_image.step, cuda_data, current_keypoints.ptr<float>(),
                                 current_keypoints.step / sizeof(float), capacity);
      current_keypoints.cols = found < capacity ? found : capacity;
      has_changed_keypoints = false;
    }
    return current_keypoints;
  }

  std::vector<KeyPoint> getKeypointsAndDownload() { return utils::downloadKeypoints(getKeypoints()); }

  // getResponses(): per scale the geometry and the D and S maps of the
  // current image (detecting first if needed).
  std::vector<ScaleResponses> getResponses() {
    getKeypoints();
    std::vector<ScaleResponses> out(cuda_data.ks.size());
    for (size_t s = 0; s < out.size(); ++s) {
      ScaleResponses& r = out[s];
      r.info = cuda_data.ks[s];
      r.d_ResultDouble.create(r.info.data_h, r.info.data_w, sizeof(float));
      r.d_ResultSingle.create(r.info.data_h, r.info.data_w, sizeof(float));
      check(bimp_dense_map(cuda_data.handle(), static_cast<int>(s), 0, r.d_ResultDouble.ptr<float>(),
                           r.d_ResultDouble.step / sizeof(float), nullptr),
            "getResponses");
      check(bimp_dense_map(cuda_data.handle(), static_cast<int>(s), 1, r.d_ResultSingle.ptr<float>(),
                           r.d_ResultSingle.step / sizeof(float), nullptr),
            "getResponses");
    }
    return out;
  }

  // downloadResultsToCPU() (bimp.cpp:75-80, cuda_bimp.cu downloadResultsToCPU):
  // the responses with their host copies filled.
  std::vector<ScaleResponses> downloadResultsToCPU() {
    std::vector<ScaleResponses> out = getResponses();
    for (ScaleResponses& r : out) {
      const size_t n = static_cast<size_t>(r.info.data_w) * r.info.data_h;
      r.h_ResultDouble.resize(n);
      r.h_ResultSingle.resize(n);
      r.d_ResultDouble.download(r.h_ResultDouble.data(), sizeof(float) * r.info.data_w);
      r.d_ResultSingle.download(r.h_ResultSingle.data(), sizeof(float) * r.info.data_w);
    }
    return out;
  }

  // The 24-bin colour histogram of every current keypoint over the colour
  // image (addColorFeatures, bimp/src/bimp.cpp:42-43): n x 24 floats, row
  // major.  Needs a 3-channel (BGR) image.
  std::vector<float> getColorFeatures() {
    if (current_image_color.empty()) throw Error(BIMP_ERR_INVALID, "getColorFeatures: the image has no colour");
    DeviceMat& kp = getKeypoints();
    const int n = kp.cols;
    std::vector<float> out(static_cast<size_t>(n) * 24);
    if (n == 0) return out;
    DeviceMat desc(n, 24, sizeof(float));
    check(bimp_color_features(kp.ptr<float>(), kp.step / sizeof(float), n, current_image_color.data,
                              current_image_color.step, current_image.cols, current_image.rows,
                              desc.ptr<float>(), desc.step / sizeof(float), nullptr),
          "getColorFeatures");
    desc.download(out.data(), 24 * sizeof(float));
    return out;
  }

  int width() const { return current_image.cols; }
  int height() const { return current_image.rows; }

  cuda::CudaStuff cuda_data;
  DeviceMat current_image, current_image_color, current_keypoints;
  bool has_changed_keypoints = true;
  int capacity = cuda::KP_MAX_POINTS;   // keypoint limit, as KP_MAX_POINTS
  int found = 0;                        // count before truncation to `capacity`

 private:
  static std::pair<int, int> min_size(const ImageView& image) {
    int w = 0, h = 0;
    check(bimp_min_size_dims(image.cols, image.rows, &w, &h, nullptr), "Context");
    return {w, h};
  }
#ifdef BIMP_WITH_OPENCV
  static ImageView view(const cv::Mat& m) {
    if (m.depth() != CV_8U || (m.channels() != 1 && m.channels() != 3))
      throw Error(BIMP_ERR_INVALID, "Context expects a CV_8UC1 or CV_8UC3 image");
    ImageView v;
    v.data = m.data;
    v.rows = m.rows;
    v.cols = m.cols;
    v.step = m.step;
    v.channels = m.channels();
    return v;
  }
#endif
};

}  // namespace bimp

// Minimal stand-ins for the OpenCV 3.x types that the reference's kernel
// header (bimp/include/detection/cuda_bimp.cuh, through cuda_bimp.hpp) names.
// They let that header compile unmodified for the reference harness; they are
// declarations of this repository's own, carry no OpenCV code, and are used
// only by the oracle's reference build (test infrastructure).
//
// Only PtrStepSz has behaviour, because the reference kernels index through
// it: ptr(y) is the address of row y (`step` bytes apart) and (y, x) the
// element, which is how the kernels address their matrices.
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

#ifndef CV_PI
#define CV_PI 3.1415926535897932384626433832795
#endif

namespace cv {
typedef unsigned char uchar;

class Mat {};
template <typename T>
class Mat_ {};
class KeyPoint {};
class Scalar {
 public:
  Scalar() {}
  explicit Scalar(double) {}
};

namespace cuda {
class GpuMat {};

template <typename T>
struct PtrStepSz {
  T* data;
  size_t step;   // bytes between rows
  int cols;
  int rows;
  __host__ __device__ PtrStepSz() : data(nullptr), step(0), cols(0), rows(0) {}
  __host__ __device__ PtrStepSz(int rows_, int cols_, T* data_, size_t step_)
      : data(data_), step(step_), cols(cols_), rows(rows_) {}
  __host__ __device__ T* ptr(int y = 0) { return reinterpret_cast<T*>(reinterpret_cast<char*>(data) + y * step); }
  __host__ __device__ const T* ptr(int y = 0) const {
    return reinterpret_cast<const T*>(reinterpret_cast<const char*>(data) + y * step);
  }
  __host__ __device__ T& operator()(int y, int x) { return ptr(y)[x]; }
  __host__ __device__ const T& operator()(int y, int x) const { return ptr(y)[x]; }
};
}  // namespace cuda
}  // namespace cv

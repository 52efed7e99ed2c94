// Stand-in for OpenCV's SURF_CUDA keypoint row layout, the only name the
// reference's kernel header takes from this OpenCV header.  Row ids as in
// OpenCV's cv::cuda::SURF_CUDA::KeypointLayout (X, Y, LAPLACIAN, OCTAVE,
// SIZE, ANGLE, HESSIAN).  Test infrastructure for the oracle's reference
// build only.
#pragma once

#include "../opencv.hpp"

namespace cv {
namespace cuda {
struct SURF_CUDA {
  enum KeypointLayout { X_ROW = 0, Y_ROW, LAPLACIAN_ROW, OCTAVE_ROW, SIZE_ROW, ANGLE_ROW, HESSIAN_ROW, ROWS_COUNT };
};
}  // namespace cuda
}  // namespace cv

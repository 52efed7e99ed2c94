// Input preprocessing and the colour-histogram descriptor.
//
//   bimp_min_size_dims / bimp_gpu_image   getGPUImage, bimp/src/cuda_bimp.cu:156-180
//   bimp_color_features                   addColorFeatures_kernel,
//                                         bimp/include/detection/cuda_bimp.cuh:8-71
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>

#include "bimp_b200.h"
#include "bimp_internal.h"

namespace bimp_b200 {

// cv::resize INTER_LINEAR source index and 11-bit fixed-point weights of one
// destination coordinate: f = (d + 0.5) * scale - 0.5 in float, clamped to
// the first / last source sample at the borders.
__device__ __forceinline__ void lin_coef(int d, double scale, int n, int& s0, int& s1, int& a0, int& a1) {
  float f = (float)((d + 0.5) * scale - 0.5);
  int s = (int)floorf(f);
  f -= (float)s;
  if (s < 0) { f = 0.f; s = 0; }
  if (s >= n - 1) { f = 0.f; s = n - 1; }
  s0 = s;
  s1 = min(s + 1, n - 1);
  a0 = __float2int_rn((1.f - f) * 2048.f);
  a1 = __float2int_rn(f * 2048.f);
}

// One channel of the bilinear upscale: horizontal taps in int, vertical
// blend with the 16-bit multiply-high rounding of OpenCV's 8-bit path.
__device__ __forceinline__ int lin_sample(const uint8_t* __restrict__ src, size_t pitch, int cn, int c, int sy0, int sy1,
                                          int b0, int b1, int sx0, int sx1, int a0, int a1) {
  const int h0 = src[(size_t)sy0 * pitch + sx0 * cn + c] * a0 + src[(size_t)sy0 * pitch + sx1 * cn + c] * a1;
  const int h1 = src[(size_t)sy1 * pitch + sx0 * cn + c] * a0 + src[(size_t)sy1 * pitch + sx1 * cn + c] * a1;
  const int y = ((b0 * (h0 >> 4)) >> 16) + ((b1 * (h1 >> 4)) >> 16);
  const int v = (y + 2) >> 2;
  return v < 0 ? 0 : (v > 255 ? 255 : v);
}

// getGPUImage: optional upscale of a BGR or grey image, then BGR -> grey with
// the 14-bit fixed-point weights of the CUDA colour conversion
// (Y = (1868 B + 9617 G + 4899 R + 8192) >> 14), or the resized BGR image.
__global__ void k_gpu_image(const uint8_t* __restrict__ src, size_t spitch, int sw, int sh, int cn,
                            uint8_t* __restrict__ dst, size_t dpitch, int dw, int dh, int gray, double scale) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= dw || y >= dh) return;
  int px[3];
  if (dw == sw && dh == sh) {
    for (int c = 0; c < cn; ++c) px[c] = src[(size_t)y * spitch + x * cn + c];
  } else {
    int sx0, sx1, a0, a1, sy0, sy1, b0, b1;
    lin_coef(x, scale, sw, sx0, sx1, a0, a1);
    lin_coef(y, scale, sh, sy0, sy1, b0, b1);
    for (int c = 0; c < cn; ++c) px[c] = lin_sample(src, spitch, cn, c, sy0, sy1, b0, b1, sx0, sx1, a0, a1);
  }
  if (cn == 1) {
    dst[(size_t)y * dpitch + x] = (uint8_t)px[0];
  } else if (gray) {
    dst[(size_t)y * dpitch + x] = (uint8_t)((px[0] * 1868 + px[1] * 9617 + px[2] * 4899 + 8192) >> 14);
  } else {
    for (int c = 0; c < cn; ++c) dst[(size_t)y * dpitch + x * cn + c] = (uint8_t)px[c];
  }
}

// addColorFeatures_kernel: 8-bin histograms of B, G and R over a
// 2p x 2p window, p = (int)(log2(size)/2), at (int)x, (int)y.  As in the
// reference the channel bytes are read as signed char and the bins are the
// open intervals (31.875 k, 31.875 (k+1)); every visited pixel adds 3 to the
// normaliser; desc = 0.5 * count / visited.  The reference's window test
// admits iy == rows and ix == cols (one past the image); reads there are
// skipped here.
__global__ void k_color_features(const float* __restrict__ kp, size_t kld, int n, const uint8_t* __restrict__ bgr,
                                 size_t pitch, int w, int h, float* __restrict__ desc, size_t dld) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float x = kp[BIMP_X_ROW * kld + i];
  const float y = kp[BIMP_Y_ROW * kld + i];
  const float size = kp[BIMP_SIZE_ROW * kld + i];
  const int bins = 8;
  const float thresh = (float)(255.0 / (1.0 * bins));
  float cnt[24];
#pragma unroll
  for (int k = 0; k < 24; ++k) cnt[k] = 0.f;
  const int im_x = (int)x, im_y = (int)y;
  const int pixels = (int)(log2((double)size) / 2.0);
  int found = 0;
  for (int iy = im_y - pixels; iy < im_y + pixels; ++iy) {
    if (iy < 0 || iy > h) continue;
    for (int ix = im_x - pixels; ix < im_x + pixels; ++ix) {
      if (ix < 0 || ix > w) continue;
      found += 3;
      if (iy >= h || ix >= w) continue;
      const uint8_t* p = bgr + (size_t)iy * pitch + 3 * ix;
      const signed char ch[3] = {(signed char)p[0], (signed char)p[1], (signed char)p[2]};
#pragma unroll
      for (int c = 0; c < 3; ++c) {
#pragma unroll
        for (int k = 0; k < bins; ++k)
          if ((float)ch[c] > thresh * k && (float)ch[c] < thresh * (k + 1)) cnt[c * bins + k] += 1.f;
      }
    }
  }
  float* d = desc + (size_t)i * dld;
#pragma unroll
  for (int k = 0; k < 24; ++k) d[k] = (float)((0.5 * cnt[k]) / (found * 1.0));
}

}  // namespace bimp_b200

using namespace bimp_b200;

namespace {
int xfail(int code, const std::string& m) {
  record_error(m);
  return code;
}
}  // namespace

extern "C" int bimp_min_size_dims(int width, int height, int* out_w, int* out_h, double* scale) {
  if (!out_w || !out_h || width <= 0 || height <= 0) return xfail(BIMP_ERR_INVALID, "bad size");
  const int kMin = 350;   // cuda_bimp.cu:158
  double sf = 1.0;
  if (height < kMin && width >= kMin)
    sf = static_cast<float>(kMin / (1.0 * height));
  else if (width < kMin)
    sf = static_cast<float>(kMin / (1.0 * width));
  *out_w = sf == 1.0 ? width : static_cast<int>(std::nearbyint(width * sf));
  *out_h = sf == 1.0 ? height : static_cast<int>(std::nearbyint(height * sf));
  if (scale) *scale = sf;
  return BIMP_OK;
}

extern "C" int bimp_gpu_image(const uint8_t* d_src, size_t src_pitch, int width, int height, int channels,
                              int grayscale, uint8_t* d_dst, size_t dst_pitch, void* stream) {
  if (!d_src || !d_dst || (channels != 1 && channels != 3)) return xfail(BIMP_ERR_INVALID, "bad image arguments");
  int ow = 0, oh = 0;
  double sf = 1.0;
  int rc = bimp_min_size_dims(width, height, &ow, &oh, &sf);
  if (rc != BIMP_OK) return rc;
  const int ocn = (grayscale || channels == 1) ? 1 : channels;
  if (src_pitch < (size_t)width * channels || dst_pitch < (size_t)ow * ocn)
    return xfail(BIMP_ERR_INVALID, "pitch too small");
  dim3 b(32, 8), g((ow + 31) / 32, (oh + 7) / 8);
  k_gpu_image<<<g, b, 0, static_cast<cudaStream_t>(stream)>>>(d_src, src_pitch, width, height, channels, d_dst,
                                                               dst_pitch, ow, oh, grayscale ? 1 : 0, 1.0 / sf);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return xfail(BIMP_ERR_CUDA, cudaGetErrorString(e));
  return BIMP_OK;
}

extern "C" int bimp_color_features(const float* d_kp, size_t kp_ld, int n, const uint8_t* d_bgr, size_t bgr_pitch,
                                   int width, int height, float* d_desc, size_t desc_ld, void* stream) {
  if (n < 0 || (n > 0 && (!d_kp || !d_bgr || !d_desc || kp_ld < (size_t)n || desc_ld < 24 ||
                          bgr_pitch < (size_t)width * 3)))
    return xfail(BIMP_ERR_INVALID, "bad colour-feature arguments");
  if (n == 0) return BIMP_OK;
  k_color_features<<<(n + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(d_kp, kp_ld, n, d_bgr, bgr_pitch,
                                                                                    width, height, d_desc, desc_ld);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return xfail(BIMP_ERR_CUDA, cudaGetErrorString(e));
  return BIMP_OK;
}

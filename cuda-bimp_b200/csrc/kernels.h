// Launch interface of the BIMP kernels (kernels.cu).
#pragma once

#include <string>

#include <cuda_runtime.h>
#include <cstdint>

#include "bimp_internal.h"

namespace bimp_b200 {

// One pyramid step src (sw x sh, pitch sp) -> dst (dw x dh, pitch dp).
// Up to three pyrDown levels of one image from one source level.
struct PyrJob {
  const uint8_t* src;
  int sw, sh, sp;
  uint8_t* dst[3];
  int dw[3], dh[3], dp[3];
};

// One float pyramid step (same fields; for the transpose, src is the level-l
// gradient with pitch sp and dst the level-(l-1) gradient with pitch dp, while
// sw/sh stay the level-(l-1) size and dw/dh the level-l size).
struct PyrJobF {
  const float* src;
  int sw, sh, sp;
  float* dst;
  int dw, dh, dp;
};

// Keypoint destination of one image: a 7 x ld SURF-layout float matrix
// (rows X, Y, LAPLACIAN, OCTAVE, SIZE, ANGLE, HESSIAN), or with aos = 1 an
// array of bimp_keypoint records (7 words each, cv::KeyPoint field order).
struct KpOut {
  float* kp = nullptr;
  size_t ld = 0;
  int capacity = 0;
  int aos = 0;
  int* count = nullptr;   // where the NMS also writes the image's keypoint total (or null)
};

cudaError_t configure_kernels();
size_t gabor_smem_bytes();
// SM count of the current device (cached per device).
int num_sms();
size_t stencil_smem_bytes();

// `levels` (1..3) pyrDown steps per job in one launch; maxW/maxH: largest
// deepest-level size over the jobs
void launch_set_out(KpOut* d, const KpOut& v, cudaStream_t s);
// reset/resetWords: words the launch's first CTA zeroes before anything else
// of the detection runs (the map maxima and the fault word), or null.
void launch_pyr(const PyrJob* d_jobs, int njobs, int levels, int maxW, int maxH, cudaStream_t s,
                unsigned int* reset = nullptr, int resetWords = 0);
// d_fault: word that receives 1 if a bounded device wait expired.
// pipelined: the warp-specialised variant (k_gabor_tiles_ws), for work whose
// scales all have V <= pipelined_tile_max_valid(); otherwise the phased one
// pdl: launched with programmatic stream serialisation after the previous
// kernel of the detection sequence (see griddep_wait in kernels.cu)
void launch_gabor(const ScaleDev* d_sd, const TileWork* d_work, int nwork, int grid, unsigned int* d_fault,
                  cudaStream_t s, bool pipelined, bool pdl = false);
int pipelined_tile_max_valid();
// One TMA tensor map per scale entry over its complex-cell maps (x: cPitch
// columns, y: cRows rows, z: the 8 orientations; box 48 x 48 x 8 floats,
// zero fill outside), written to maps[e] (128-byte CUtensorMap blobs).
constexpr size_t kTensorMapBytes = 128;
struct alignas(64) TensorMapBlob {
  unsigned char bytes[kTensorMapBytes];
};
bool encode_c_maps(const ScaleDev* sds, int n, void* maps, std::string& err);

// Stencil output modes: D only (detection), D and S (responses), and the
// differentiable forward (D, T, R, ReLU states).
enum StencilMode { kStencilD = 0, kStencilDS = 1, kStencilAdj = 2 };
// Persistent stencil (one CTA per SM); an expired staging wait sets bit 1 of
// *d_fault.
void launch_stencil(const ScaleDev* d_sd, const int2* d_work, int nwork, unsigned int* d_fault, cudaStream_t s,
                    int mode = kStencilD, bool pdl = false);
// NMS in two launches (k_nms_decide, k_nms_emit): one CTA per group of up to
// kNmsRowsPerCta candidate rows of one image; d_ctaCount holds nctas ints
// (written by the first kernel, read by the second).
constexpr int kNmsRowsPerCta = 8;
struct NmsCta {
  int rowStart;   // first entry of the CTA's rows in the row list
  int nRows;      // 1..kNmsRowsPerCta
  int firstCta;   // first CTA of the image (its chain starts at 0)
  int image;
  int last;       // 1: the image's last CTA, which writes the image total
};
void launch_nms_two_pass(const ScaleDev* d_sd, const int2* d_rows, const NmsCta* d_ctas, int nctas, int* d_ctaCount,
                         int* d_totals, const KpOut* d_outs, cudaStream_t s, bool pdl = false);
void launch_nms(const ScaleDev* d_sd, const int2* d_rows, int nrows, int* d_counts, int* d_offsets,
                const int* d_imageRowStart, int nImages, int* d_totals, const KpOut* d_outs,
                cudaStream_t s);

// differentiable path and its adjoint
void launch_pyr_f(const PyrJobF* d_jobs, int njobs, int maxW, int maxH, cudaStream_t s);
void launch_pyr_f_adj(const PyrJobF* d_jobs, int njobs, int maxW, int maxH, cudaStream_t s);
// differentiable forward: the tile kernel on the float levels (one CTA per
// work item)
void launch_gabor_flt(const ScaleDev* d_sd, const TileWork* d_work, int nwork, unsigned int* d_fault,
                      cudaStream_t s, bool pipelined);
// detection-path tile kernel that also keeps e + i o (ScaleDev::Z) for the
// line/edge detector; one CTA per work item
void launch_gabor_keep_z(const ScaleDev* d_sd, const TileWork* d_work, int nwork, unsigned int* d_fault,
                         cudaStream_t s);
// line/edge detection on one scale (d_sd: that scale's descriptor, with Z)
void launch_detect_le(const ScaleDev* d_sd, int dataW, int dataH, const float* d_ch, int chLd, float* d_result,
                      float* d_ori, int8_t* d_type, int ld, cudaStream_t s);
void launch_masked_loss(const ScaleDev* d_sd, const int2* d_work, int nwork, double* d_loss, double* d_gparams,
                        cudaStream_t s);
void launch_stencil_bwd(const ScaleDev* d_sd, const int2* d_work, int nwork, cudaStream_t s);
// tile backward, recomputing the responses; `grid` persistent CTAs (at most
// nwork), d_xscratch holds grid x kSpecHalf float2 (one tile spectrum per CTA)
void launch_gabor_bwd(const ScaleDev* d_sd, const TileWork* d_work, int nwork, int grid, float2* d_xscratch,
                      double* d_gparams, cudaStream_t s);

}  // namespace bimp_b200

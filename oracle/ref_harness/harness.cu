// Reference harness (test infrastructure; part of the oracle, never of the
// product): runs the reference's own BIMP device kernels, compiled unmodified
// from bimp/include/detection/cuda_bimp.cuh of daniel-koudouna/cuda-bimp, on
// one scale of one image, in the order of DoFullGPUFiltering
// (bimp/src/cuda_bimp.cu:462-559) and cuda_gpu_keypoints
// (bimp/src/cuda_bimp.cu:714-743), with cuFFT doing the reference's R2C/C2R
// transforms.
//
// Kernels taken from the reference header as they are:
//   FilterSimpleCells_kernel     cuda_bimp.cuh:226-248
//   complexResponse_kernel       cuda_bimp.cuh:165-180
//   endStoppedResponse_kernel    cuda_bimp.cuh:436-467
//   inhibitionResponse_kernel    cuda_bimp.cuh:469-502
//   inhibitKeypoints_kernel      cuda_bimp.cuh:504-517
//   identifyKeypoints_kernel     cuda_bimp.cuh:86-148
// and thrust::max_element for the map maximum (cuda_bimp.cu:960-966).
//
// What this harness supplies itself, because the reference's code for it
// needs OpenCV-CUDA or CUDA<=11 texture references:
//   * the uint8 pyramid level (the caller passes it: cv::cuda::pyrDown is not
//     available), converted with the factor 255/65536 of convertTo
//     (cuda_bimp.cu:481; exact in float);
//   * the padded image and the padded kernels, by the index maps of
//     padDataClampToBorder / padKernel (convolutionFFT2D.cuh:31-85):
//     data rows/cols, then kernelY/kernelX clamp-to-last, then index 0; kernel
//     centre at (0, 0) with wrap;
//   * the 3x3 dilate with the centre masked out and the subtraction
//     (cuda_bimp.cu:73-85, 730-733): only pixels more than (int)lambda from the
//     border are ever used, so the border rule does not matter;
//   * the Gabor taps and stencil offsets (host arithmetic, passed in).
//
// The complex-cell buffers get slack rows after the fftH x fftW torus holding
// its first elements again (flat index wrapped modulo fftH*fftW).  The
// reference's stencils read one row (and, when fftW == dataW, one more
// element) past the data by flat address; where that is past the torus the
// reference reads whatever its (larger, shared) buffer holds, and this
// harness makes it the wrapped torus, the choice the oracle makes.
#include <cuda_runtime.h>
#include <cufft.h>
#include <thrust/device_ptr.h>
#include <thrust/extrema.h>

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "cuda_bimp.cuh"

namespace {

std::string g_err;

struct Fail {};

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    g_err = std::string(what) + ": " + cudaGetErrorString(e);
    throw Fail();
  }
}
void ckf(cufftResult r, const char* what) {
  if (r != CUFFT_SUCCESS) {
    g_err = std::string(what) + ": cufft error " + std::to_string((int)r);
    throw Fail();
  }
}

// padDataClampToBorder's source index (convolutionFFT2D.cuh:56-85).
__host__ __device__ inline int pad_src_index(int t, int n, int k_half) {
  return t < n ? t : (t < n + k_half ? n - 1 : 0);
}

__global__ void k_level_to_float(const uint8_t* __restrict__ lvl, int pitch, float* __restrict__ out, int W, int H) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x < W && y < H) out[y * W + x] = (float)lvl[(size_t)y * pitch + x] * (255.0f / 65536.0f);
}

__global__ void k_pad_data(const float* __restrict__ d, float* __restrict__ p, int W, int H, int fftW, int fftH,
                           int kX, int kY) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x < fftW && y < fftH) p[y * fftW + x] = d[pad_src_index(y, H, kY) * W + pad_src_index(x, W, kX)];
}

// 8-neighbour maximum (centre excluded) and loc = D - dil; border pixels
// take the in-range neighbours only.
__global__ void k_dilate_subtract(const float* __restrict__ D, float* __restrict__ loc, int W, int H) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= W || y >= H) return;
  float m = -INFINITY;
  for (int dy = -1; dy <= 1; ++dy)
    for (int dx = -1; dx <= 1; ++dx) {
      if (!dx && !dy) continue;
      const int yy = y + dy, xx = x + dx;
      if (yy >= 0 && yy < H && xx >= 0 && xx < W) m = fmaxf(m, D[yy * W + xx]);
    }
  loc[y * W + x] = D[y * W + x] - m;
}

template <typename T>
struct DevBuf {
  T* p = nullptr;
  explicit DevBuf(size_t n) { ck(cudaMalloc(&p, sizeof(T) * (n ? n : 1)), "cudaMalloc"); }
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
};

struct Plan {
  cufftHandle h = 0;
  bool ok = false;
  Plan(int fftH, int fftW, cufftType t) {
    ckf(cufftPlan2d(&h, fftH, fftW, t), "cufftPlan2d");
    ok = true;
  }
  ~Plan() {
    if (ok) cufftDestroy(h);
  }
};

}  // namespace

extern "C" {

const char* bref_last_error(void) { return g_err.c_str(); }

// One scale.  level: host uint8, at least dataH rows x dataW columns at
// `pitch` bytes.  even/odd: host taps, 8 x kW x kW (row-major).  es/inh:
// 8 x 2 ints, the end-stop and inhibition offsets (row, col) per
// orientation (cuda_bimp.cu:533-550).  Outputs (host): D and S, dataH x
// dataW (k.d_ResultDouble / k.d_ResultSingle); C (may be null), 8 x fftH x
// fftW complex cells; kp, 7 x cap floats (SURF_CUDA rows, int rows 2 and 3),
// unordered (atomic slots); *count the total found.  Returns 0 or -1
// (message in bref_last_error()).
int bref_scale(const uint8_t* level, int pitch, int dataW, int dataH, int fftW, int fftH, int kW, int kX,
               const float* even, const float* odd, const int* es, const int* inh, float lambda_level,
               float pyrstep, float* D_out, float* S_out, float* C_out, float* kp_out, int cap, int* count) {
  try {
    if (!level || !even || !odd || !es || !inh || !D_out || !S_out || !kp_out || !count || cap <= 0 || dataW < 3 ||
        dataH < 3 || pitch < dataW || fftW < dataW || fftH < dataH || kW > fftW || kW > fftH || (fftW & 1)) {
      g_err = "bad arguments";
      return -1;
    }
    const int W = dataW, H = dataH;
    const size_t N = (size_t)W * H, F = (size_t)fftW * fftH, Fh = (size_t)fftH * (fftW / 2 + 1);
    const size_t slack = 2 * (size_t)fftW + 64;
    // level -> float data -> padded image -> spectrum (cuda_bimp.cu:473-499)
    DevBuf<uint8_t> dLvl((size_t)pitch * H);
    ck(cudaMemcpy(dLvl.p, level, (size_t)pitch * H, cudaMemcpyHostToDevice), "level upload");
    DevBuf<float> dData(N), dPad(F);
    DevBuf<cufftComplex> dSpec(Fh);
    const dim3 b2(32, 8);
    k_level_to_float<<<dim3((W + 31) / 32, (H + 7) / 8), b2>>>(dLvl.p, pitch, dData.p, W, H);
    k_pad_data<<<dim3((fftW + 31) / 32, (fftH + 7) / 8), b2>>>(dData.p, dPad.p, W, H, fftW, fftH, kX, kX);
    ck(cudaGetLastError(), "pad");
    Plan fwd(fftH, fftW, CUFFT_R2C), inv(fftH, fftW, CUFFT_C2R);
    ckf(cufftExecR2C(fwd.h, dPad.p, dSpec.p), "R2C data");
    // kernel spectra (cuda_bimp.cu:338-349): centre at (0, 0) with wrap
    std::vector<DevBuf<cufftComplex>*> kse, kso;
    struct Cleanup {
      std::vector<DevBuf<cufftComplex>*>* a;
      std::vector<DevBuf<cufftComplex>*>* b;
      ~Cleanup() {
        for (auto* p : *a) delete p;
        for (auto* p : *b) delete p;
      }
    } cleanup{&kse, &kso};
    {
      std::vector<float> hp(F);
      DevBuf<float> dKp(F);
      for (int o = 0; o < 8; ++o) {
        for (int eo = 0; eo < 2; ++eo) {
          const float* taps = (eo ? odd : even) + (size_t)o * kW * kW;
          std::fill(hp.begin(), hp.end(), 0.f);
          for (int y = 0; y < kW; ++y)
            for (int x = 0; x < kW; ++x) {
              const int py = ((y - kX) % fftH + fftH) % fftH, px = ((x - kX) % fftW + fftW) % fftW;
              hp[(size_t)py * fftW + px] = taps[y * kW + x];
            }
          ck(cudaMemcpy(dKp.p, hp.data(), sizeof(float) * F, cudaMemcpyHostToDevice), "kernel upload");
          auto* spec = new DevBuf<cufftComplex>(Fh);
          (eo ? kso : kse).push_back(spec);
          ckf(cufftExecR2C(fwd.h, dKp.p, spec->p), "R2C kernel");
        }
      }
    }
    // per orientation: multiply, two C2R, complex magnitude (cuda_bimp.cu:504-524)
    DevBuf<cufftComplex> dRe(Fh), dRo(Fh);
    DevBuf<float> dE(F), dO(F);
    std::vector<DevBuf<float>*> cplx;
    struct Cleanup2 {
      std::vector<DevBuf<float>*>* a;
      ~Cleanup2() {
        for (auto* p : *a) delete p;
      }
    } cleanup2{&cplx};
    for (int o = 0; o < 8; ++o) {
      cplx.push_back(new DevBuf<float>(F + slack));
      FilterSimpleCells_kernel<<<(int)((Fh + 255) / 256), 256>>>(dRe.p, dRo.p, kse[o]->p, kso[o]->p, dSpec.p, (int)Fh,
                                                                   1.0f / (float)(fftW * fftH));
      ck(cudaGetLastError(), "FilterSimpleCells_kernel");
      ckf(cufftExecC2R(inv.h, dRe.p, dE.p), "C2R even");
      ckf(cufftExecC2R(inv.h, dRo.p, dO.p), "C2R odd");
      complexResponse_kernel<<<(int)((F + 255) / 256), 256>>>(dE.p, dO.p, cplx[o]->p, (int)F);
      ck(cudaGetLastError(), "complexResponse_kernel");
      // slack: the torus continued by flat index
      for (size_t off = 0; off < slack; off += F) {
        const size_t n = std::min(F, slack - off);
        ck(cudaMemcpy(cplx[o]->p + F + off, cplx[o]->p, sizeof(float) * n, cudaMemcpyDeviceToDevice), "slack");
      }
    }
    // end-stopping, inhibition, summed map (cuda_bimp.cu:530-552)
    DevBuf<float> dD(N), dS(N), dT(N), dR(N), dLoc(N);
    ck(cudaMemset(dD.p, 0, sizeof(float) * N), "clear");
    ck(cudaMemset(dS.p, 0, sizeof(float) * N), "clear");
    ck(cudaMemset(dT.p, 0, sizeof(float) * N), "clear");
    ck(cudaMemset(dR.p, 0, sizeof(float) * N), "clear");
    const dim3 b32(32, 32), g32((W + 31) / 32, (H + 31) / 32);
    for (int o = 0; o < 8; ++o)
      endStoppedResponse_kernel<<<g32, b32>>>(dD.p, dS.p, cplx[o]->p, es[2 * o], es[2 * o + 1], W, H, fftW);
    for (int o = 0; o < 8; ++o)
      inhibitionResponse_kernel<<<g32, b32>>>(dT.p, dR.p, cplx[o]->p, cplx[(o + 4) % 8]->p, inh[2 * o],
                                              inh[2 * o + 1], W, H, fftW);
    inhibitKeypoints_kernel<<<g32, b32>>>(dD.p, dS.p, dT.p, dR.p, W, H, W);
    ck(cudaGetLastError(), "stencil kernels");
    // keypoints (cuda_bimp.cu:714-743)
    thrust::device_ptr<float> dp = thrust::device_pointer_cast(dD.p);
    const float mx = *thrust::max_element(dp, dp + N);
    const double thresh = mx * 0.104;
    k_dilate_subtract<<<dim3((W + 31) / 32, (H + 7) / 8), b2>>>(dD.p, dLoc.p, W, H);
    DevBuf<float> dKpts((size_t)7 * cap);
    DevBuf<int> dCount(1);
    ck(cudaMemset(dKpts.p, 0, sizeof(float) * 7 * cap), "clear");
    ck(cudaMemset(dCount.p, 0, sizeof(int)), "clear");
    cv::cuda::PtrStepSz<float> result(7, cap, dKpts.p, sizeof(float) * cap);
    cv::cuda::PtrStepSz<int> resultInts(7, cap, reinterpret_cast<int*>(dKpts.p), sizeof(float) * cap);
    cv::cuda::PtrStepSz<float> keypts(H, W, dD.p, sizeof(float) * W);
    cv::cuda::PtrStepSz<float> kLoc(H, W, dLoc.p, sizeof(float) * W);
    const int off = (int)lambda_level;
    const dim3 b16(16, 16), g16((W + 16) / 16, (H + 16) / 16);
    identifyKeypoints_kernel<<<g16, b16>>>(result, resultInts, keypts, kLoc, lambda_level, off, H, W, pyrstep,
                                           (float)thresh, dCount.p);
    ck(cudaGetLastError(), "identifyKeypoints_kernel");
    ck(cudaDeviceSynchronize(), "synchronize");
    ck(cudaMemcpy(D_out, dD.p, sizeof(float) * N, cudaMemcpyDeviceToHost), "D download");
    ck(cudaMemcpy(S_out, dS.p, sizeof(float) * N, cudaMemcpyDeviceToHost), "S download");
    if (C_out)
      for (int o = 0; o < 8; ++o)
        ck(cudaMemcpy(C_out + (size_t)o * F, cplx[o]->p, sizeof(float) * F, cudaMemcpyDeviceToHost), "C download");
    ck(cudaMemcpy(kp_out, dKpts.p, sizeof(float) * 7 * cap, cudaMemcpyDeviceToHost), "kp download");
    ck(cudaMemcpy(count, dCount.p, sizeof(int), cudaMemcpyDeviceToHost), "count download");
    return 0;
  } catch (Fail&) {
    return -1;
  }
}

}  // extern "C"

// Keypoint extraction from one summed keypoint map with no memory allocation.
//
// Some callers cannot allocate device memory while they run: real-time loops
// that must never enter the allocator (an allocation can block on a device
// synchronisation), or hosts whose device memory all belongs to a pool that
// the library may not touch.  They still need the threshold /
// non-maximum-suppression / compaction step.  This entry point runs it with
// all of its scratch (the scale descriptor, the per-row candidate counts and
// offsets, the maximum of the map) in one file-scope device array of fixed
// size, and calls no cudaMalloc, cudaFree or allocating library routine.  The
// caller passes the map and the keypoint destination.
//
// The array is shared by every call on a device and keeps the previous call's
// contents; each call first clears what has to start at zero.  Two calls
// whose work overlaps on the GPU (different streams, no ordering between
// them) race on the array.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "bimp_b200.h"
#include "bimp_internal.h"
#include "kernels.h"

namespace bimp_b200 {

// Largest map height the scratch array can serve (candidate rows per map).
constexpr int kNoAllocMaxRows = 16384;

struct NoAllocScratch {
  ScaleDev sd;
  KpOut out;
  int imgRowStart[2];
  int total;
  unsigned int maxKey;
  int2 rows[kNoAllocMaxRows];
  int counts[kNoAllocMaxRows];
  int offsets[kNoAllocMaxRows];
};

// One per device that loads the library; held until process exit.
static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

// Writes the descriptor, the row list and the zeroed maximum into the scratch.
__global__ void k_noalloc_setup(NoAllocScratch* s, ScaleDev sd, KpOut out, int nrows) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) {
    sd.maxKey = &s->maxKey;
    s->sd = sd;
    s->out = out;
    s->imgRowStart[0] = 0;
    s->imgRowStart[1] = nrows;
    s->total = 0;
    s->maxKey = 0u;
  }
  for (int r = t; r < nrows; r += gridDim.x * blockDim.x) s->rows[r] = make_int2(0, r);
}

__device__ __forceinline__ unsigned int noalloc_key(float f) {
  const unsigned int b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// max over the whole map (the quantity the threshold is 0.104 times).
__global__ void k_noalloc_max(const float* __restrict__ D, int ld, int W, int H, unsigned int* maxKey) {
  float m = -INFINITY;
  for (int y = blockIdx.y; y < H; y += gridDim.y)
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < W; x += gridDim.x * blockDim.x)
      m = fmaxf(m, D[(size_t)y * ld + x]);
#pragma unroll
  for (int k = 16; k > 0; k >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, k));
  if ((threadIdx.x & 31) == 0 && m > -INFINITY) atomicMax(maxKey, noalloc_key(m));
}

namespace {
std::mutex g_mu;
NoAllocScratch* g_ptr[128];

int na_fail(int code, const std::string& m) {
  record_error(m);
  return code;
}
}  // namespace

}  // namespace bimp_b200

using namespace bimp_b200;

extern "C" int bimp_extract_keypoints_noalloc(const float* d_map, size_t ld, int width, int height,
                                              float lambda_level, float pyrstep, double thresh_ratio,
                                              float* d_kp, size_t kp_ld, int capacity, int* d_count,
                                              void* stream) {
  if (!d_map || !d_count || width < 3 || height < 3 || ld < (size_t)width || capacity < 0 ||
      (capacity > 0 && (!d_kp || kp_ld < (size_t)capacity)) || !(lambda_level > 0.f) || !(pyrstep > 0.f))
    return na_fail(BIMP_ERR_INVALID, "bad arguments");
  // the kernels take the map's row pitch as an int
  if (ld > (size_t)INT_MAX) return na_fail(BIMP_ERR_INVALID, "map row pitch above INT_MAX floats");
  const int off = static_cast<int>(lambda_level);
  const int yEnd = std::min(height - off - 1, height - 2);
  const int nrows = std::max(0, yEnd - off);
  if (nrows > kNoAllocMaxRows)
    return na_fail(BIMP_ERR_UNSUPPORTED, "map has " + std::to_string(nrows) + " candidate rows; the fixed scratch "
                   "array holds " + std::to_string(kNoAllocMaxRows));
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return na_fail(BIMP_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= 128) return na_fail(BIMP_ERR_NO_DEVICE, "device index out of range");
  NoAllocScratch* s = nullptr;
  {
    // set-up once per device, with that device current: the symbol's device
    // address (the host-side name is only a stand-in)
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ptr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess) return na_fail(BIMP_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_ptr[dev] = static_cast<NoAllocScratch*>(p);
    }
    s = g_ptr[dev];
  }
  ScaleDev sd;
  std::memset(&sd, 0, sizeof(sd));
  sd.dataW = width;
  sd.dataH = height;
  sd.D = const_cast<float*>(d_map);
  sd.dPitch = static_cast<int>(ld);
  sd.off = off;
  sd.pyrstep = pyrstep;
  sd.kpSize = lambda_level * pyrstep;
  sd.kpOctave = static_cast<int>(lambda_level * pyrstep);
  sd.threshRatio = thresh_ratio;
  KpOut out;
  out.kp = d_kp;
  out.ld = kp_ld;
  out.capacity = capacity;
  out.aos = 0;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_noalloc_setup<<<std::max(1, std::min(64, (nrows + 255) / 256)), 256, 0, st>>>(s, sd, out, nrows);
  dim3 g((width + 255) / 256 < 8 ? (width + 255) / 256 : 8, std::min(height, 1024));
  k_noalloc_max<<<g, 256, 0, st>>>(d_map, static_cast<int>(ld), width, height, &s->maxKey);
  launch_nms(&s->sd, s->rows, nrows, s->counts, s->offsets, s->imgRowStart, 1, &s->total, &s->out, st);
  e = cudaMemcpyAsync(d_count, &s->total, sizeof(int), cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return na_fail(BIMP_ERR_CUDA, cudaGetErrorString(e));
  return BIMP_OK;
}

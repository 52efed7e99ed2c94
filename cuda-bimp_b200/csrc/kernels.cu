// BIMP device kernels for sm_100a.
//
//   k_pyr_down      uint8 Gaussian pyramid level (cv::cuda::pyrDown semantics)
//   k_gabor_tiles   overlap-save 128x128 tile FFT: image spectrum once per
//                   tile, then per orientation spectrum multiply + inverse
//                   FFT + complex magnitude; writes only the magnitude maps
//   k_stencil       end-stopped cells, tangential/radial inhibition and the
//                   summed keypoint map D (and S), all 8 orientations staged
//                   in shared memory; per-scale max(D)
//   k_nms_count     strict 8-neighbour maxima above 0.104*max per row
//   k_scan          exclusive scan of the row counts
//   k_nms_write     keypoint records in (scale, y, x) order
#include <cuda_runtime.h>
#include <cstdint>

#include "bimp_internal.h"
#include "fft128.cuh"
#include "kernels.h"

namespace bimp_b200 {

// ---------------------------------------------------------------------------
// pyramid
// ---------------------------------------------------------------------------
__device__ __forceinline__ int reflect101(int i, int n) {
  if (n == 1) return 0;
  const int period = 2 * n - 2;
  i = abs(i) % period;
  return i >= n ? period - i : i;
}

// dst(y,x) = rint(sum w_i w_j src(r101(2y+i), r101(2x+j)) / 256), w = 1 4 6 4 1.
// The weighted sum is an exact integer; ties round to even (cvt.rni).
__global__ void k_pyr_down(const PyrJob* __restrict__ jobs) {
  const PyrJob j = jobs[blockIdx.z];
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= j.dw || y >= j.dh) return;
  const int w5[5] = {1, 4, 6, 4, 1};
  int cols[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) cols[k] = reflect101(2 * x + k - 2, j.sw);
  int acc = 0;
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    const uint8_t* row = j.src + (size_t)reflect101(2 * y + i - 2, j.sh) * j.sp;
    int h = 0;
#pragma unroll
    for (int k = 0; k < 5; ++k) h += w5[k] * row[cols[k]];
    acc += w5[i] * h;
  }
  const int q = acc >> 8;
  const int v = (acc + 127 + (q & 1)) >> 8;
  j.dst[(size_t)y * j.dp + x] = (uint8_t)(v > 255 ? 255 : v);
}

// ---------------------------------------------------------------------------
// tiled FFT Gabor filtering
// ---------------------------------------------------------------------------
__constant__ float2 c_w128[kTile];   // exp(-2 pi i k / 128)

__device__ __forceinline__ int pmod(int a, int m) {
  const int r = a % m;
  return r < 0 ? r + m : r;
}

// Source row/col of padded-torus index t (convolutionFFT2D.cuh:56-85):
// data, then kHalf clamp-to-last entries, then clamp-to-first.
__device__ __forceinline__ int pad_src(int t, int nData, int kHalf) {
  return t < nData ? t : (t < nData + kHalf ? nData - 1 : 0);
}

// X[ky][kx] of the tile spectrum at permuted row position py and permuted
// column position p, from the Hermitian half Xh[py][slot].
__device__ __forceinline__ float2 spectrum_at(const float2* __restrict__ Xh, int py, int p) {
  const int a = p >> 3, b = p & 7;
  if (b < 4) return Xh[py * kXhCols + 4 * a + b];
  if (b == 4 && a == 0) return Xh[py * kXhCols + 64];
  const int slot = a > 0 ? 4 * (16 - a) + (7 - b) : (8 - b);
  const int c = py >> 3, d = py & 7;
  const int npy = c > 0 ? 8 * (16 - c) + (7 - d) : ((8 - d) & 7);
  const float2 v = Xh[npy * kXhCols + slot];
  return make_float2(v.x, -v.y);
}

__global__ void __launch_bounds__(kTileThreads, 1)
k_gabor_tiles(const ScaleDev* __restrict__ sds, const TileWork* __restrict__ work, int nwork) {
  extern __shared__ float4 smem4[];
  float2* W = reinterpret_cast<float2*>(smem4);      // kTile x kTileLD
  float2* Xh = W + kTile * kTileLD;                    // kTile x kXhCols
  float2* tw = Xh + kTile * kXhCols;                   // 8 x 17: w128^(n1*k2)
  int* rmap = reinterpret_cast<int*>(tw + 8 * 17);     // window row -> level row
  int* cmap = rmap + kTile;                            // window col -> level col
  const int t = threadIdx.x;

  if (t < 8 * 17) {
    const int n1 = t / 17, k2 = t % 17;
    tw[t] = k2 < 16 ? c_w128[(n1 * k2) & 127] : make_float2(0.f, 0.f);
  }

  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const TileWork item = work[w];
    const ScaleDev* sd = sds + item.entry;
    const int kX = sd->kX, V = sd->V;
    const int ty = item.tile / sd->tilesX, tx = item.tile - ty * sd->tilesX;
    const int R0 = ty * V, C0 = tx * V;
    const uint8_t* __restrict__ lvl = sd->lvl;
    const int lp = sd->lvlPitch;

    __syncthreads();   // previous tile finished with maps / work buffers
    if (t < kTile) {
      rmap[t] = pad_src(pmod(R0 - kX + t, sd->fftH), sd->dataH, kX);
    } else if (t < 2 * kTile) {
      const int i = t - kTile;
      cmap[i] = pad_src(pmod(C0 - kX + i, sd->fftW), sd->dataW, kX);
    }
    __syncthreads();

    // F1: x-dim pass A on packed rows z[r] = in[r] + i in[r+64], r < 64.
    // Pixel value 255*u8/65536 (convertTo, cuda_bimp.cu:481) enters as
    // (255*u8 - 32768)/65536 = value - 0.5, exactly; the 0.5 offset is put
    // back into the DC bin below.  Removing the mean keeps the butterflies'
    // intermediate magnitudes, and so their float rounding, small.
    {
      const int r = t >> 3, n1 = t & 7;
      const uint8_t* rowA = lvl + (size_t)rmap[r] * lp;
      const uint8_t* rowB = lvl + (size_t)rmap[r + 64] * lp;
      const float s = 1.0f / 65536.0f;
      float2 v[16];
#pragma unroll
      for (int m = 0; m < 16; ++m) {
        const int c = cmap[n1 + 8 * m];
        v[m] = make_float2(s * (float)(255 * (int)rowA[c] - 32768),
                           s * (float)(255 * (int)rowB[c] - 32768));
      }
      dft16<false>(v);
#pragma unroll
      for (int k2 = 0; k2 < 16; ++k2)
        W[r * kTileLD + phys(n1 + 8 * k2)] = c_mul(v[k2], tw[n1 * 17 + k2]);
    }
    __syncthreads();
    // F2: x-dim pass B
#pragma unroll
    for (int it = 0; it < 2; ++it) {
      const int j = t + it * kTileThreads;
      const int r = j >> 4, k2 = j & 15;
      float2 v[8];
#pragma unroll
      for (int n1 = 0; n1 < 8; ++n1) v[n1] = W[r * kTileLD + phys(8 * k2 + n1)];
      dft8<false>(v);
#pragma unroll
      for (int k1 = 0; k1 < 8; ++k1) W[r * kTileLD + phys(8 * k2 + k1)] = v[k1];
    }
    __syncthreads();
    // separation of the packed rows into the Hermitian half (kx = 0..64)
    for (int j = t; j < 64 * kXhCols; j += kTileThreads) {
      const int r = j / kXhCols, s = j - r * kXhCols;
      const int kx = s < 64 ? (s >> 2) + 16 * (s & 3) : 64;
      const int nk = (128 - kx) & 127;
      const float2 Z = W[r * kTileLD + phys(8 * (kx & 15) + (kx >> 4))];
      const float2 Zn = W[r * kTileLD + phys(8 * (nk & 15) + (nk >> 4))];
      Xh[r * kXhCols + s] = make_float2(0.5f * (Z.x + Zn.x), 0.5f * (Z.y - Zn.y));
      Xh[(r + 64) * kXhCols + s] = make_float2(0.5f * (Z.y + Zn.y), 0.5f * (Zn.x - Z.x));
    }
    __syncthreads();
    // F3: y-dim pass A on the 65 half columns
    for (int j = t; j < 8 * kXhCols; j += kTileThreads) {
      const int n1 = j / kXhCols, s = j - n1 * kXhCols;
      float2 v[16];
#pragma unroll
      for (int m = 0; m < 16; ++m) v[m] = Xh[(n1 + 8 * m) * kXhCols + s];
      dft16<false>(v);
#pragma unroll
      for (int k2 = 0; k2 < 16; ++k2)
        Xh[(n1 + 8 * k2) * kXhCols + s] = c_mul(v[k2], tw[n1 * 17 + k2]);
    }
    __syncthreads();
    // F4: y-dim pass B -> Xh rows in permuted ky order
    for (int j = t; j < 16 * kXhCols; j += kTileThreads) {
      const int k2 = j / kXhCols, s = j - k2 * kXhCols;
      float2 v[8];
#pragma unroll
      for (int n1 = 0; n1 < 8; ++n1) v[n1] = Xh[(8 * k2 + n1) * kXhCols + s];
      dft8<false>(v);
#pragma unroll
      for (int k1 = 0; k1 < 8; ++k1) Xh[(8 * k2 + k1) * kXhCols + s] = v[k1];
    }
    __syncthreads();
    if (t == 0) Xh[0].x += 0.5f * (float)(kTile * kTile);   // DC of the removed 0.5 offset
    __syncthreads();

    const int cRows = sd->cRows, cCols = sd->cCols, cPitch = sd->cPitch;
    for (int o = 0; o < kNumOri; ++o) {
      const float* __restrict__ G = sd->G + (size_t)o * kSpecFloats;
      float* __restrict__ Cout = sd->C + (size_t)o * sd->cStride;
      // I1: y-dim pass B' with the spectrum product Z = X * G
#pragma unroll
      for (int it = 0; it < 4; ++it) {
        const int j = t + it * kTileThreads;
        const int p = j & 127, k2 = j >> 7;
        float2 v[8];
#pragma unroll
        for (int k1 = 0; k1 < 8; ++k1) {
          const int py = 8 * k2 + k1;
          v[k1] = c_scale(spectrum_at(Xh, py, p), __ldg(G + py * kTile + p));
        }
        dft8<true>(v);
        const int pc = phys(p);
#pragma unroll
        for (int n1 = 0; n1 < 8; ++n1)
          W[(8 * k2 + n1) * kTileLD + pc] = c_mulc(v[n1], tw[n1 * 17 + k2]);
      }
      __syncthreads();
      // I2: y-dim pass A' -> natural y
#pragma unroll
      for (int it = 0; it < 2; ++it) {
        const int j = t + it * kTileThreads;
        const int p = j & 127, n1 = j >> 7;
        const int pc = phys(p);
        float2 v[16];
#pragma unroll
        for (int k2 = 0; k2 < 16; ++k2) v[k2] = W[(8 * k2 + n1) * kTileLD + pc];
        dft16<true>(v);
#pragma unroll
        for (int n2 = 0; n2 < 16; ++n2) W[(n1 + 8 * n2) * kTileLD + pc] = v[n2];
      }
      __syncthreads();
      // I3: x-dim pass B' on the rows holding valid outputs
      for (int j = t; j < V * 16; j += kTileThreads) {
        const int y = kX + (j >> 4), k2 = j & 15;
        float2 v[8];
#pragma unroll
        for (int k1 = 0; k1 < 8; ++k1) v[k1] = W[y * kTileLD + phys(8 * k2 + k1)];
        dft8<true>(v);
#pragma unroll
        for (int n1 = 0; n1 < 8; ++n1)
          W[y * kTileLD + phys(8 * k2 + n1)] = c_mulc(v[n1], tw[n1 * 17 + k2]);
      }
      __syncthreads();
      // I4: x-dim pass A' -> natural x; complex magnitude of valid outputs
      for (int j = t; j < V * 8; j += kTileThreads) {
        const int y = kX + (j >> 3), n1 = j & 7;
        float2 v[16];
#pragma unroll
        for (int k2 = 0; k2 < 16; ++k2) v[k2] = W[y * kTileLD + phys(8 * k2 + n1)];
        dft16<true>(v);
        const int gy = R0 + y - kX;
        if (gy < cRows) {
          float* dst = Cout + (size_t)gy * cPitch;
#pragma unroll
          for (int n2 = 0; n2 < 16; ++n2) {
            const int x = n1 + 8 * n2;
            const int gx = C0 + x - kX;
            if (x >= kX && x < kX + V && gx < cCols)
              dst[gx] = sqrtf(v[n2].x * v[n2].x + v[n2].y * v[n2].y);
          }
        }
      }
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------
// stencil: end-stopping, inhibition, summed keypoint map
// ---------------------------------------------------------------------------
constexpr int kStX = 32, kStY = 32, kHalo = 8;
constexpr int kStW = kStX + 2 * kHalo, kStH = kStY + 2 * kHalo;

__device__ __forceinline__ unsigned int float_key(float f) {
  const unsigned int b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float key_float(unsigned int k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

__device__ __forceinline__ bool stencil_ok(int x, int y, int o1, int o2, int W, int H) {
  // cuda_bimp.cuh:446-449 (inclusive upper bounds)
  return x - o2 >= 0 && x - o2 <= W && x + o2 >= 0 && x + o2 <= W &&
         y - o1 >= 0 && y - o1 <= H && y + o1 >= 0 && y + o1 <= H &&
         x - 2 * o2 >= 0 && x - 2 * o2 <= W && x + 2 * o2 >= 0 && x + 2 * o2 <= W &&
         y - 2 * o1 >= 0 && y - 2 * o1 <= H && y + 2 * o1 >= 0 && y + 2 * o1 <= H;
}

__global__ void __launch_bounds__(256)
k_stencil(const ScaleDev* __restrict__ sds, const int2* __restrict__ work) {
  extern __shared__ float s_c[];   // kNumOri x kStH x kStW
  const int2 item = work[blockIdx.x];
  const ScaleDev* sd = sds + item.x;
  const int W = sd->dataW, H = sd->dataH;
  const int nbx = (W + kStX - 1) / kStX;
  const int by = item.y / nbx, bx = item.y - by * nbx;
  const int x0 = bx * kStX, y0 = by * kStY;
  const int t = threadIdx.x;

  // stage C (rows y0-8 .. y0+39, cols x0-8 .. x0+39) of all orientations
  const float* __restrict__ C = sd->C;
  const int cPitch = sd->cPitch;
  const long long cStride = sd->cStride;
  const int wrapW = sd->wrapW;
  for (int idx = t; idx < kNumOri * kStH * kStW; idx += 256) {
    const int o = idx / (kStH * kStW);
    const int rem = idx - o * (kStH * kStW);
    const int ly = rem / kStW, lx = rem - ly * kStW;
    const int gy = y0 - kHalo + ly, gx = x0 - kHalo + lx;
    float v = 0.f;
    if (gy >= 0 && gy <= H && gx >= 0 && gx <= W) {
      int ry = gy, rx = gx;
      if (wrapW && gx == W) { rx = 0; ry = gy + 1; }   // flat y*fftW + fftW
      v = C[(size_t)o * cStride + (size_t)ry * cPitch + rx];
    }
    s_c[idx] = v;
  }
  __syncthreads();

  const int lx = t & 31, ly0 = t >> 5;
  const int x = x0 + lx;
  float dmax = -INFINITY;
  const float gain = sd->radialGain, wT = sd->wTan, wR = sd->wRad;
#pragma unroll 1
  for (int i = 0; i < 4; ++i) {
    const int ly = ly0 + 8 * i;
    const int y = y0 + ly;
    if (x >= W || y >= H) continue;
    const int cy = ly + kHalo, cx = lx + kHalo;
    float S = 0.f, D = 0.f, T = 0.f, R = 0.f;
#pragma unroll
    for (int o = 0; o < kNumOri; ++o) {
      const int o1 = sd->es1[o], o2 = sd->es2[o];
      if (!stencil_ok(x, y, o1, o2, W, H)) continue;
      const float* c = s_c + o * (kStH * kStW);
      float s = c[(cy - o1) * kStW + cx + o2] - c[(cy + o1) * kStW + cx - o2];
      s = s > 0.f ? s : 0.f;
      if (s > 0.f) S += s;
      // the reference evaluates this line in double (0.5 is a double literal)
      const double dd = (double)c[cy * kStW + cx] - 0.5 * (double)c[(cy - 2 * o1) * kStW + cx + 2 * o2]
                        - 0.5 * (double)c[(cy + 2 * o1) * kStW + cx - 2 * o2];
      float d = (float)dd;
      d = d > 0.f ? d : 0.f;
      if (d > 0.f) D += d;
    }
#pragma unroll
    for (int o = 0; o < kNumOri; ++o) {
      const int o1 = sd->in1[o], o2 = sd->in2[o];
      if (!stencil_ok(x, y, o1, o2, W, H)) continue;
      const float* c = s_c + o * (kStH * kStW);
      const float* cp = s_c + ((o + kNumOri / 2) % kNumOri) * (kStH * kStW);
      const float centre = c[cy * kStW + cx];
      float v = c[(cy - o1) * kStW + cx - o2] - centre;
      v = v < 0.f ? 0.f : v;
      T += v;
      const int h1 = sd->ih1[o], h2 = sd->ih2[o];
      float r = centre - gain * cp[(cy + h1) * kStW + cx + h2];
      r = r < 0.f ? 0.f : r;
      r += centre - gain * cp[(cy - h1) * kStW + cx - h2];
      r = r < 0.f ? 0.f : r;
      R += r;
    }
    const float inhib = wT * T + wR * R;
    D = D + (-inhib);
    S = S + (-inhib);
    sd->D[(size_t)y * sd->dPitch + x] = D;
    sd->S[(size_t)y * sd->dPitch + x] = S;
    dmax = fmaxf(dmax, D);
  }
  // block max -> one atomic per block
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) dmax = fmaxf(dmax, __shfl_xor_sync(0xffffffffu, dmax, m));
  __shared__ float s_max[8];
  __syncthreads();
  if ((t & 31) == 0) s_max[t >> 5] = dmax;
  __syncthreads();
  if (t == 0) {
    float m = s_max[0];
    for (int k = 1; k < 8; ++k) m = fmaxf(m, s_max[k]);
    if (m > -INFINITY) atomicMax(sd->maxKey, float_key(m));
  }
}

// ---------------------------------------------------------------------------
// NMS, threshold, compaction
// ---------------------------------------------------------------------------
__device__ __forceinline__ float scale_thresh(const ScaleDev* sd) {
  // cuda_bimp.cu:720-721: float max, double thresh, passed as float
  const float mx = key_float(*sd->maxKey);
  return (float)((double)mx * (double)sd->threshRatio);
}

__device__ __forceinline__ bool is_keypoint(const float* __restrict__ D, int dp, int x, int y, float thr) {
  const float* r0 = D + (size_t)(y - 1) * dp;
  const float* r1 = r0 + dp;
  const float* r2 = r1 + dp;
  const float v = r1[x];
  float dil = fmaxf(fmaxf(r0[x - 1], r0[x]), r0[x + 1]);
  dil = fmaxf(dil, fmaxf(r1[x - 1], r1[x + 1]));
  dil = fmaxf(dil, fmaxf(fmaxf(r2[x - 1], r2[x]), r2[x + 1]));
  return (v - dil > 0.f) && (v > thr);
}

__global__ void __launch_bounds__(256)
k_nms_count(const ScaleDev* __restrict__ sds, const int2* __restrict__ rows, int* __restrict__ counts) {
  const int2 item = rows[blockIdx.x];
  const ScaleDev* sd = sds + item.x;
  const int off = sd->off;
  const int y = off + 1 + item.y;
  const float thr = scale_thresh(sd);
  const int xEnd = min(sd->dataW - off, sd->dataW - 1);
  int n = 0;
  for (int x = off + 1 + threadIdx.x; x < xEnd; x += blockDim.x)
    n += is_keypoint(sd->D, sd->dPitch, x, y, thr) ? 1 : 0;
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) n += __shfl_xor_sync(0xffffffffu, n, m);
  __shared__ int s_n[8];
  if ((threadIdx.x & 31) == 0) s_n[threadIdx.x >> 5] = n;
  __syncthreads();
  if (threadIdx.x == 0) {
    int tot = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) tot += s_n[k];
    counts[blockIdx.x] = tot;
  }
}

// Exclusive scan of counts[0..n) into offsets; per-image totals from the
// image boundaries.  One block of 1024 threads, 4 elements per thread per
// chunk, carried across chunks.
__global__ void __launch_bounds__(1024)
k_scan(const int* __restrict__ counts, int* __restrict__ offsets, int n,
       const int* __restrict__ imageRowStart, int nImages, int* __restrict__ imageTotals) {
  __shared__ int s_w[32];
  __shared__ int s_carry;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int base = 0; base < n; base += 4096) {
    int v[4];
    int sum = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int i = base + threadIdx.x * 4 + k;
      v[k] = i < n ? counts[i] : 0;
      sum += v[k];
    }
    int incl = sum;
#pragma unroll
    for (int m = 1; m < 32; m <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, incl, m);
      if (lane >= m) incl += u;
    }
    if (lane == 31) s_w[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      int wv = s_w[lane];
      int wi = wv;
#pragma unroll
      for (int m = 1; m < 32; m <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, wi, m);
        if (lane >= m) wi += u;
      }
      s_w[lane] = wi - wv;   // exclusive warp offsets
    }
    __syncthreads();
    int run = s_carry + s_w[wid] + incl - sum;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int i = base + threadIdx.x * 4 + k;
      if (i < n) offsets[i] = run;
      run += v[k];
    }
    __syncthreads();
    if (threadIdx.x == 1023) s_carry = run;
    __syncthreads();
  }
  for (int im = threadIdx.x; im < nImages; im += blockDim.x) {
    const int a = imageRowStart[im], b = imageRowStart[im + 1];
    int tot = 0;
    if (b > a) tot = offsets[b - 1] + counts[b - 1] - offsets[a];
    imageTotals[im] = tot;
  }
}

__global__ void __launch_bounds__(256)
k_nms_write(const ScaleDev* __restrict__ sds, const int2* __restrict__ rows,
            const int* __restrict__ offsets, const int* __restrict__ imageRowStart,
            const KpOut* __restrict__ outs) {
  const int2 item = rows[blockIdx.x];
  const ScaleDev* sd = sds + item.x;
  const KpOut out = outs[sd->image];
  const int off = sd->off;
  const int y = off + 1 + item.y;
  const float thr = scale_thresh(sd);
  int base = offsets[blockIdx.x] - offsets[imageRowStart[sd->image]];
  if (base >= out.capacity) return;
  const float* D = sd->D;
  const int dp = sd->dPitch;
  __shared__ int s_w[8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int xEnd = min(sd->dataW - off, sd->dataW - 1);
  for (int xs = off + 1; xs < xEnd; xs += blockDim.x) {
    const int x = xs + threadIdx.x;
    const bool kp = x < xEnd && is_keypoint(D, dp, x, y, thr);
    const unsigned int bal = __ballot_sync(0xffffffffu, kp);
    if (lane == 0) s_w[wid] = __popc(bal);
    __syncthreads();
    int before = 0, total = 0;
    for (int k = 0; k < 8; ++k) {
      before += k < wid ? s_w[k] : 0;
      total += s_w[k];
    }
    if (kp) {
      const int idx = base + before + __popc(bal & ((1u << lane) - 1u));
      if (idx < out.capacity) {
        const float* r1 = D + (size_t)y * dp;
        const float xv1 = r1[x - 1], xv2 = r1[x], xv3 = r1[x + 1];
        const float yv1 = r1[x - dp], yv3 = r1[x + dp];
        float xpos = (float)x, ypos = (float)y;
        // cuda_bimp.cuh:114-132 (parabola through the 3 samples per axis)
        const float denx = xv1 + xv3 - 2.f * xv2;
        const float deny = yv1 + yv3 - 2.f * xv2;
        const float numx = 0.5f * (xv1 - xv3);
        const float numy = 0.5f * (yv1 - yv3);
        if (denx != 0.f) xpos += __fdiv_rn(numx, denx);
        if (deny != 0.f) ypos += __fdiv_rn(numy, deny);
        float* kpm = out.kp;
        const size_t ld = out.ld;
        kpm[0 * ld + idx] = xpos * sd->pyrstep;
        kpm[1 * ld + idx] = ypos * sd->pyrstep;
        reinterpret_cast<int*>(kpm)[2 * ld + idx] = 1;
        reinterpret_cast<int*>(kpm)[3 * ld + idx] = sd->kpOctave;
        kpm[4 * ld + idx] = sd->kpSize;
        kpm[5 * ld + idx] = -1.f;
        kpm[6 * ld + idx] = xv2;
      }
    }
    base += total;
    __syncthreads();
    if (base >= out.capacity) break;
  }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
cudaError_t upload_twiddles() {
  float2 h[kTile];
  for (int k = 0; k < kTile; ++k) {
    const double a = -2.0 * M_PI * k / kTile;
    h[k] = make_float2((float)cos(a), (float)sin(a));
  }
  return cudaMemcpyToSymbol(c_w128, h, sizeof(h));
}

size_t gabor_smem_bytes() {
  return sizeof(float2) * (kTile * kTileLD + kTile * kXhCols + 8 * 17) + sizeof(int) * 2 * kTile;
}
size_t stencil_smem_bytes() { return sizeof(float) * kNumOri * kStH * kStW; }

cudaError_t configure_kernels() {
  cudaError_t e = cudaFuncSetAttribute(k_gabor_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)gabor_smem_bytes());
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_stencil, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)stencil_smem_bytes());
  if (e != cudaSuccess) return e;
  return upload_twiddles();
}

void launch_pyr(const PyrJob* d_jobs, int njobs, int maxW, int maxH, cudaStream_t s) {
  dim3 b(32, 8), g((maxW + 31) / 32, (maxH + 7) / 8, njobs);
  k_pyr_down<<<g, b, 0, s>>>(d_jobs);
}
void launch_gabor(const ScaleDev* d_sd, const TileWork* d_work, int nwork, int grid, cudaStream_t s) {
  k_gabor_tiles<<<grid, kTileThreads, gabor_smem_bytes(), s>>>(d_sd, d_work, nwork);
}
void launch_stencil(const ScaleDev* d_sd, const int2* d_work, int nwork, cudaStream_t s) {
  k_stencil<<<nwork, 256, stencil_smem_bytes(), s>>>(d_sd, d_work);
}
void launch_nms(const ScaleDev* d_sd, const int2* d_rows, int nrows, int* d_counts, int* d_offsets,
                const int* d_imageRowStart, int nImages, int* d_totals, const KpOut* d_outs,
                cudaStream_t s) {
  if (nrows > 0) k_nms_count<<<nrows, 256, 0, s>>>(d_sd, d_rows, d_counts);
  k_scan<<<1, 1024, 0, s>>>(d_counts, d_offsets, nrows, d_imageRowStart, nImages, d_totals);
  if (nrows > 0) k_nms_write<<<nrows, 256, 0, s>>>(d_sd, d_rows, d_offsets, d_imageRowStart, d_outs);
}

}  // namespace bimp_b200

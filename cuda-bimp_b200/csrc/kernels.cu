// BIMP device kernels for sm_100a.
//
//   k_pyr_down      uint8 Gaussian pyramid, up to three levels per launch
//                   (cv::cuda::pyrDown semantics)
//   k_gabor_tiles   overlap-save 128x128 tile FFT: image spectrum once per
//                   work item, then per orientation spectrum multiply +
//                   inverse FFT + complex magnitude; writes only the
//                   magnitude maps (k_gabor_tiles_ws: warp-specialised form)
//   k_stencil       end-stopped cells, tangential/radial inhibition and the
//                   summed keypoint map D (and S), all 8 orientations staged
//                   in shared memory; per-scale max(D)
//   k_nms_decide    strict 8-neighbour maxima above 0.104*max: decision
//                   words and per-group counts
//   k_nms_emit      keypoint records in (scale, y, x) order
//   k_nms_count, k_scan, k_nms_write: the same NMS in three launches over
//                   whole rows (the allocation-free extraction entry point)
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "bimp_internal.h"
#include "fft128.cuh"
#include "kernels.h"

namespace bimp_b200 {

// Programmatic dependent launch.  A kernel launched with programmatic stream
// serialisation may start before its predecessor in the stream has finished:
// griddep_wait() blocks until the predecessor grid has completed and its
// memory is visible (a no-op after an ordinary launch), and
// griddep_launch_dependents() lets the successor's CTAs be scheduled once
// every CTA of this grid has started (they then wait in griddep_wait, on SMs
// this grid's last wave leaves free).
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

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
//
// K levels in one launch: a CTA owns a T x T tile of the deepest level
// (T = 8, 16, 32 for K = 3, 2, 1) and the 2x, 4x larger tiles above it; it
// loads the source region the tile depends on (5-tap support, reflect-101
// at the level edges) into shared memory and computes each level's region
// from the one above, writing the part it owns.
constexpr int pyr_tile(int K) { return 32 >> (K - 1); }

constexpr int pyr_side(int K, int m) { return m == K ? pyr_tile(K) : 2 * pyr_side(K, m + 1) + 3; }
// Shared memory of the computed levels 1..K (square regions).
constexpr int pyr_smem(int K) {
  return K == 3 ? pyr_side(3, 1) * pyr_side(3, 1) + pyr_side(3, 2) * pyr_side(3, 2) + pyr_side(3, 3) * pyr_side(3, 3)
       : K == 2 ? pyr_side(2, 1) * pyr_side(2, 1) + pyr_side(2, 2) * pyr_side(2, 2)
                : pyr_side(1, 1) * pyr_side(1, 1);
}
// The source region is staged as 16-byte chunks: the chunks of a region row
// cover its S0 bytes after a lead of up to 15 bytes (the region's first
// column rounded down to a 16-byte boundary).
constexpr int pyr_chunks(int K) { return (pyr_side(K, 0) + 15 + 15) / 16; }
constexpr int kPyrThreads = 256;

// Largest horizontal-pass buffer of a K-level launch (rows of the level
// above x columns of the level computed).
constexpr int pyr_hbuf(int K) {
  return K == 3 ? pyr_side(3, 0) * pyr_side(3, 1) : K == 2 ? pyr_side(2, 0) * pyr_side(2, 1) : pyr_side(1, 0) * pyr_side(1, 1);
}

// Level M of a K-level launch from level M - 1: regions of side
// pyr_side(K, M - 1) (in) and pyr_side(K, M) (out) in shared memory.  A
// region partly outside level M - 1 first gets its reflect-101 border: each
// position outside the level takes the value of its reflection inside it,
// where that lies in the region (the other positions feed no output inside
// level M).  Sources lie inside the level and targets outside it, so the
// copies do not overlap.  Then every region runs the same two passes:
// output column c takes input columns 2 c .. 2 c + 4, output row r rows
// 2 r .. 2 r + 4 (exact integer sums: the same values as reflecting each
// tap), two outputs per item.
template <int K, int M>
__device__ __forceinline__ void pyr_level(const PyrJob& j, const int (&loY)[K + 1], const int (&loX)[K + 1],
                                          const int (&off)[K + 1], int oy, int ox, int lead, uint8_t* s_raw,
                                          uint8_t* s_lvl, uint16_t* s_h, int t) {
  constexpr int Si = pyr_side(K, M - 1), So = pyr_side(K, M), Sp = (So + 1) / 2;
  constexpr int ip = M == 1 ? 16 * pyr_chunks(K) : Si;   // row pitch of the level above in shared memory
  constexpr int own = pyr_tile(K) << (K - M);
  const int Wi = M == 1 ? j.sw : j.dw[M - 2], Hi = M == 1 ? j.sh : j.dh[M - 2];
  const int Wo = j.dw[M - 1], Ho = j.dh[M - 1];
  const int ownY = oy << (K - M), ownX = ox << (K - M);
  uint8_t* in = M == 1 ? s_raw + lead : s_lvl + off[M - 1];
  uint8_t* outS = s_lvl + off[M];
  uint8_t* dst = j.dst[M - 1];
  const int dp = j.dp[M - 1];
  const int ly = loY[M - 1], lx = loX[M - 1];
  if (!(lx >= 0 && ly >= 0 && lx + Si <= Wi && ly + Si <= Hi)) {
    // the region's rows [r0, r1) and columns [c0, c1) lie inside the level;
    // items: every column of the rows outside, then the columns outside of
    // the rows inside
    const int r0 = min(Si, max(0, -ly)), r1 = max(r0, min(Si, Hi - ly));
    const int c0 = min(Si, max(0, -lx)), c1 = max(c0, min(Si, Wi - lx));
    const int nOutC = Si - (c1 - c0);
    const int nA = (Si - (r1 - r0)) * Si, nB = (r1 - r0) * nOutC;
    for (int idx = t; idx < nA + nB; idx += kPyrThreads) {
      int r, c;
      if (idx < nA) {
        const int rr = idx / Si;
        c = idx - rr * Si;
        r = rr < r0 ? rr : r1 + (rr - r0);
      } else {
        const int k = idx - nA, ir = k / nOutC, cc = k - ir * nOutC;
        r = r0 + ir;
        c = cc < c0 ? cc : c1 + (cc - c0);
      }
      const int sr = reflect101(ly + r, Hi) - ly, sc = reflect101(lx + c, Wi) - lx;
      if (sr >= 0 && sr < Si && sc >= 0 && sc < Si) in[r * ip + c] = in[sr * ip + sc];
    }
    __syncthreads();
  }
  // horizontal pass: columns c, c + 1 share input columns 2 c + 2 .. 2 c + 4
  // (for an odd So the last item's second output is not stored; its two
  // extra input bytes lie inside the buffers)
  for (int idx = t; idx < Si * Sp; idx += kPyrThreads) {
    const int r = idx / Sp, c = 2 * (idx - r * Sp);
    const uint8_t* a = in + r * ip + 2 * c;
    const int a0 = a[0], a1 = a[1], a2 = a[2], a3 = a[3], a4 = a[4], a5 = a[5], a6 = a[6];
    s_h[r * So + c] = (uint16_t)(a0 + 4 * a1 + 6 * a2 + 4 * a3 + a4);
    if (c + 1 < So) s_h[r * So + c + 1] = (uint16_t)(a2 + 4 * a3 + 6 * a4 + 4 * a5 + a6);
  }
  __syncthreads();
  // vertical pass: rows r, r + 1 share h-pass rows 2 r + 2 .. 2 r + 4;
  // rounding to nearest with ties to even; the owned outputs inside the
  // level go to the level buffer
  for (int idx = t; idx < Sp * So; idx += kPyrThreads) {
    const int rp = idx / So, c = idx - rp * So, r = 2 * rp;
    const uint16_t* a = s_h + 2 * r * So + c;
    const int b0 = a[0], b1 = a[So], b2 = a[2 * So], b3 = a[3 * So], b4 = a[4 * So], b5 = a[5 * So],
              b6 = a[6 * So];
    const int x = loX[M] + c;
    const bool xin = x >= ownX && x < ownX + own && x < Wo;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (h == 1 && r + 1 >= So) break;
      const int acc = h ? b2 + 4 * b3 + 6 * b4 + 4 * b5 + b6 : b0 + 4 * b1 + 6 * b2 + 4 * b3 + b4;
      const int q = acc >> 8;
      int v = (acc + 127 + (q & 1)) >> 8;
      v = v > 255 ? 255 : v;
      outS[(r + h) * So + c] = (uint8_t)v;
      const int y = loY[M] + r + h;
      if (xin && y >= ownY && y < ownY + own && y < Ho) dst[(size_t)y * dp + x] = (uint8_t)v;
    }
  }
  __syncthreads();
}

template <int K>
__global__ void __launch_bounds__(kPyrThreads) k_pyr_down(const PyrJob* __restrict__ jobs,
                                                           unsigned int* __restrict__ reset, int resetWords) {
  constexpr int S0 = pyr_side(K, 0), CPR = pyr_chunks(K), SP = 16 * CPR;
  __shared__ __align__(16) uint8_t s_raw[S0 * SP];   // source region, row pitch SP
  __shared__ uint8_t s_lvl[pyr_smem(K)];             // levels 1..K
  __shared__ uint16_t s_h[pyr_hbuf(K) + 2 * pyr_side(K, 1)];   // + 2 rows read by the last row pair
  griddep_launch_dependents();
  // the detection's reset (the map maxima and the fault word), done here
  // instead of by a memset of its own: every later kernel waits for this grid
  if (reset && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0)
    for (int i = threadIdx.x; i < resetWords; i += kPyrThreads) reset[i] = 0u;
  // the job by value: read once (the level stores could alias it for the compiler)
  const PyrJob j = jobs[blockIdx.z];
  constexpr int T = pyr_tile(K);
  const int oy = blockIdx.y * T, ox = blockIdx.x * T;
  if (oy >= j.dh[K - 1] || ox >= j.dw[K - 1]) return;
  int loY[K + 1], loX[K + 1], off[K + 1];
  loY[K] = oy;
  loX[K] = ox;
#pragma unroll
  for (int m = K; m >= 1; --m) {
    loY[m - 1] = 2 * loY[m] - 2;
    loX[m - 1] = 2 * loX[m] - 2;
  }
  off[0] = 0;
  off[1] = 0;
#pragma unroll
  for (int m = 2; m <= K; ++m) off[m] = off[m - 1] + pyr_side(K, m - 1) * pyr_side(K, m - 1);
  const int t = threadIdx.x;
  // Source region as 16-byte chunks (level rows start 16-byte aligned and
  // their pitch is a multiple of 16, so a chunk that starts inside the pitch
  // lies inside the row).  All of a thread's loads are issued before the
  // first store.  Chunks outside the level leave their bytes unset until the
  // reflect-101 fill of the first level step.
  const int a16 = loX[0] & ~15;
  const int lead = loX[0] - a16;
  {
    constexpr int NCH = S0 * CPR, PER = (NCH + kPyrThreads - 1) / kPyrThreads;
    uint4 v[PER];
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int idx = t + kPyrThreads * i;
      const int r = idx / CPR, w = a16 + 16 * (idx - r * CPR);
      const int gy = loY[0] + r;
      v[i] = make_uint4(0u, 0u, 0u, 0u);
      if (idx < NCH && gy >= 0 && gy < j.sh && w >= 0 && w < j.sp)
        v[i] = *reinterpret_cast<const uint4*>(j.src + (size_t)gy * j.sp + w);
    }
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int idx = t + kPyrThreads * i;
      if (idx < NCH) reinterpret_cast<uint4*>(s_raw)[idx] = v[i];
    }
  }
  __syncthreads();
  pyr_level<K, 1>(j, loY, loX, off, oy, ox, lead, s_raw, s_lvl, s_h, t);
  if constexpr (K >= 2) pyr_level<K, 2>(j, loY, loX, off, oy, ox, lead, s_raw, s_lvl, s_h, t);
  if constexpr (K >= 3) pyr_level<K, 3>(j, loY, loX, off, oy, ox, lead, s_raw, s_lvl, s_h, t);
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

#include "gabor_tiles.cuh"

// ---------------------------------------------------------------------------
// stencil: end-stopping, inhibition, summed keypoint map
// ---------------------------------------------------------------------------
constexpr int kStX = 32, kStY = 32, kHalo = 8;   // kStY: the adjoint's stencil blocks
constexpr int kFwY = kStencilBlockH;               // forward stencil block rows
constexpr int kStW = kStX + 2 * kHalo, kStH = kFwY + 2 * kHalo;

__device__ __forceinline__ unsigned int float_key(float f) {
  const unsigned int b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float key_float(unsigned int k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// Per-scale stencil constants, staged once per block in shared memory.
struct StencilPar {
  int e1[kNumOri], e2[kNumOri];      // end-stop offsets (row, col)
  int i1[kNumOri], i2[kNumOri];      // inhibition offsets
  int h1[kNumOri], h2[kNumOri];      // radial half offsets
  int exlo[kNumOri], exhi[kNumOri], eylo[kNumOri], eyhi[kNumOri];  // end-stop bounds
  int ixlo[kNumOri], ixhi[kNumOri], iylo[kNumOri], iyhi[kNumOri];  // inhibition bounds
};

// Offset k (0..5: es1, es2, in1, in2, ih1, ih2) of orientation o: a
// compile-time constant for PAT > 0, else the staged runtime value.
template <int PAT>
__device__ __forceinline__ int soff(const StencilPar& P, int k, int o) {
  if constexpr (PAT > 0) {
    constexpr int sets[kNumOffsetSets][6][8] = BIMP_OFFSET_SETS;
    return sets[PAT - 1][k][o];
  } else {
    const int* base = k == 0 ? P.e1 : k == 1 ? P.e2 : k == 2 ? P.i1 : k == 3 ? P.i2 : k == 4 ? P.h1 : P.h2;
    return base[o];
  }
}

// One pixel of end-stopping and inhibition (cuda_bimp.cuh:436-517).  The
// bounds test of the reference (x -+ o2, x -+ 2 o2 in [0, W], likewise y)
// reduces to 2|o2| <= x <= W - 2|o2| and 2|o1| <= y <= H - 2|o1|.
// The double-stopped term c - 0.5 a - 0.5 b, which the reference evaluates
// in double and rounds once, is two fused float multiply-adds here (at most
// one float rounding apart).
// Stencil modes: detection writes D only (the single-stopped map S is not on
// the keypoint path); responses write D and S; the differentiable forward
// writes D, the tangential and radial sums T, R and the ReLU states the
// adjoint needs: per orientation o, bit 4o double-stopped d > 0, 4o+1
// tangential t > 0, 4o+2 radial r > 0, 4o+3 the first radial term r1 > 0
// (all 0 where the bounds test fails).
// Whether orientation o's taps at offsets k, k + 1 (0: end-stopping,
// 2: inhibition) pass the reference's bounds test at (x, y) of a W x H map.
// With compile-time offsets the bounds are immediates against W and H in
// registers; the staged per-orientation bounds would cost four shared loads
// per orientation and pixel in every edge block, whose pixels then ran at
// about half the rate of the inner blocks' pixels.
template <int PAT>
__device__ __forceinline__ bool stencil_in(const StencilPar& P, int k, int o, int x, int y, int W, int H) {
  if constexpr (PAT > 0) {
    const int a1 = 2 * abs(soff<PAT>(P, k, o)), a2 = 2 * abs(soff<PAT>(P, k + 1, o));
    return x >= a2 && x <= W - a2 && y >= a1 && y <= H - a1;
  } else if (k == 0) {
    return x >= P.exlo[o] && x <= P.exhi[o] && y >= P.eylo[o] && y <= P.eyhi[o];
  } else {
    return x >= P.ixlo[o] && x <= P.ixhi[o] && y >= P.iylo[o] && y <= P.iyhi[o];
  }
}

template <bool CHECK, int PAT, int MODE>
__device__ __forceinline__ void stencil_pixel(const float* __restrict__ s_c, const StencilPar& P, int x, int y,
                                              int cy, int cx, float gain, float wT, float wR, float& Dout,
                                              float& Sout, float& Tout, float& Rout, unsigned int& bits,
                                              int W, int H) {
  float S = 0.f, D = 0.f, T = 0.f, R = 0.f;
  unsigned int b = 0;
  const float* c0 = s_c + cy * kStW + cx;
#pragma unroll
  for (int o = 0; o < kNumOri; ++o) {
    if (CHECK && !stencil_in<PAT>(P, 0, o, x, y, W, H)) continue;
    const int o1 = soff<PAT>(P, 0, o), o2 = soff<PAT>(P, 1, o);
    const float* c = c0 + o * (kStH * kStW);
    if constexpr (MODE == kStencilDS) S += fmaxf(c[-o1 * kStW + o2] - c[o1 * kStW - o2], 0.f);
    const float d = fmaf(-0.5f, c[2 * o1 * kStW - 2 * o2], fmaf(-0.5f, c[-2 * o1 * kStW + 2 * o2], c[0]));
    if constexpr (MODE == kStencilAdj) b |= (d > 0.f ? 1u : 0u) << (4 * o);
    D += fmaxf(d, 0.f);
  }
#pragma unroll
  for (int o = 0; o < kNumOri; ++o) {
    if (CHECK && !stencil_in<PAT>(P, 2, o, x, y, W, H)) continue;
    const int o1 = soff<PAT>(P, 2, o), o2 = soff<PAT>(P, 3, o);
    const float* c = c0 + o * (kStH * kStW);
    const float* cp = c0 + ((o + kNumOri / 2) % kNumOri) * (kStH * kStW);
    const float centre = c[0];
    const float v = c[-o1 * kStW - o2] - centre;
    if constexpr (MODE == kStencilAdj) b |= (v > 0.f ? 2u : 0u) << (4 * o);
    T += fmaxf(v, 0.f);
    const int h1 = soff<PAT>(P, 4, o), h2 = soff<PAT>(P, 5, o);
    float r = centre - gain * cp[h1 * kStW + h2];
    if constexpr (MODE == kStencilAdj) b |= (r > 0.f ? 8u : 0u) << (4 * o);
    r = fmaxf(r, 0.f);
    r += centre - gain * cp[-h1 * kStW - h2];
    if constexpr (MODE == kStencilAdj) b |= (r > 0.f ? 4u : 0u) << (4 * o);
    R += fmaxf(r, 0.f);
  }
  const float inhib = wT * T + wR * R;
  Dout = D + (-inhib);
  Sout = S + (-inhib);
  if constexpr (MODE == kStencilAdj) {
    Tout = T;
    Rout = R;
    bits = b;
  }
}

// Packed pairs of floats (lane 0: the upper pixel, lane 1: the pixel 16
// rows below) for the f32x2 arithmetic of sm_100.
typedef unsigned long long f2p;
__device__ __forceinline__ f2p pk2(float a, float b) {
  f2p r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void upk2(f2p v, float& a, float& b) { asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v)); }
__device__ __forceinline__ f2p add2(f2p a, f2p b) {
  f2p d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2p sub2(f2p a, f2p b) {
  f2p d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2p fma2(f2p a, f2p b, f2p c) {
  f2p d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ f2p relu2(f2p v) {
  float a, b;
  upk2(v, a, b);
  return pk2(fmaxf(a, 0.f), fmaxf(b, 0.f));
}

// D of two pixels 16 rows apart, every tap inside its bounds (an inner
// block), compile-time offsets: the arithmetic of stencil_pixel in the same
// order and roundings, two pixels per instruction.
template <int PAT>
__device__ __forceinline__ void stencil_pair_d(const float* __restrict__ s_c, int cy, int cx, float gain, float wT,
                                               float wR, float& Da, float& Db) {
  constexpr int dR = 16 * kStW;
  const float* c0 = s_c + cy * kStW + cx;
  const f2p mh = pk2(-0.5f, -0.5f), mg = pk2(-gain, -gain);
  f2p D = pk2(0.f, 0.f), T = D, R = D;
  f2p cen[kNumOri];
#pragma unroll
  for (int o = 0; o < kNumOri; ++o) {
    const int o1 = soff<PAT>(StencilPar{}, 0, o), o2 = soff<PAT>(StencilPar{}, 1, o);
    const float* c = c0 + o * (kStH * kStW);
    cen[o] = pk2(c[0], c[dR]);
    const int ka = 2 * o1 * kStW - 2 * o2, kb = -2 * o1 * kStW + 2 * o2;
    const f2p d = fma2(mh, pk2(c[ka], c[dR + ka]), fma2(mh, pk2(c[kb], c[dR + kb]), cen[o]));
    D = add2(D, relu2(d));
  }
#pragma unroll
  for (int o = 0; o < kNumOri; ++o) {
    const int o1 = soff<PAT>(StencilPar{}, 2, o), o2 = soff<PAT>(StencilPar{}, 3, o);
    const float* c = c0 + o * (kStH * kStW);
    const float* cp = c0 + ((o + kNumOri / 2) % kNumOri) * (kStH * kStW);
    const int kt = -o1 * kStW - o2;
    T = add2(T, relu2(sub2(pk2(c[kt], c[dR + kt]), cen[o])));
    const int h1 = soff<PAT>(StencilPar{}, 4, o), h2 = soff<PAT>(StencilPar{}, 5, o);
    const int k1 = h1 * kStW + h2;
    f2p r = relu2(fma2(mg, pk2(cp[k1], cp[dR + k1]), cen[o]));
    r = add2(r, fma2(mg, pk2(cp[-k1], cp[dR - k1]), cen[o]));
    R = add2(R, relu2(r));
  }
  float d0, d1, t0, t1, r0, r1;
  upk2(D, d0, d1);
  upk2(T, t0, t1);
  upk2(R, r0, r1);
  const float inhA = wT * t0 + wR * r0;
  const float inhB = wT * t1 + wR * r1;
  Da = d0 + (-inhA);
  Db = d1 + (-inhB);
}

// Output maps of one stencil block.
struct StencilOut {
  float* D;
  float* S;
  float* T;
  float* R;
  unsigned int* bits;
  int pitch;
};

// The rows of one thread (ly0, ly0 + NT/32, ...).  CHECK = false: every
// pixel of the block is inside the map and at least 8 from its edges, so
// the rows run as straight-line code whose loads and sums interleave.
template <bool CHECK, int PAT, int MODE, int NT>
__device__ __forceinline__ float stencil_rows(const float* __restrict__ s_c, const StencilPar& P, int x0, int y0,
                                              int W, int H, float gain, float wT, float wR, const StencilOut& out) {
  const int t = threadIdx.x;
  const int lx = t & 31, ly0 = t >> 5;
  const int x = x0 + lx;
  constexpr int kRows = kFwY / (NT / 32);
  float D[kRows], S[kRows], T[kRows], R[kRows];
  unsigned int b[kRows];
  if constexpr (!CHECK && PAT > 0 && MODE == kStencilD && NT / 32 == 16) {
#pragma unroll
    for (int i = 0; i < kRows; i += 2)
      stencil_pair_d<PAT>(s_c, ly0 + 16 * i + kHalo, lx + kHalo, gain, wT, wR, D[i], D[i + 1]);
  } else {
#pragma unroll
    for (int i = 0; i < kRows; ++i) {
      const int ly = ly0 + (NT / 32) * i;
      stencil_pixel<CHECK, PAT, MODE>(s_c, P, x, y0 + ly, ly + kHalo, lx + kHalo, gain, wT, wR, D[i], S[i], T[i],
                                      R[i], b[i], W, H);
    }
  }
  float dmax = -INFINITY;
#pragma unroll
  for (int i = 0; i < kRows; ++i) {
    const int y = y0 + ly0 + (NT / 32) * i;
    if (CHECK && (x >= W || y >= H)) continue;
    const size_t k = (size_t)y * out.pitch + x;
    out.D[k] = D[i];
    if constexpr (MODE == kStencilDS) out.S[k] = S[i];
    if constexpr (MODE == kStencilAdj) {
      out.T[k] = T[i];
      out.R[k] = R[i];
      out.bits[k] = b[i];
    }
    dmax = fmaxf(dmax, D[i]);
  }
  return dmax;
}

template <int PAT, int MODE, int NT>
__device__ __forceinline__ float stencil_block(const float* __restrict__ s_c, const StencilPar& P, int x0, int y0,
                                               int W, int H, float gain, float wT, float wR, const StencilOut& out) {
  // no bounds test needed when every pixel of the block is >= 8 from the edges
  const bool inner = x0 >= kHalo && x0 + kStX <= W - kHalo && y0 >= kHalo && y0 + kFwY <= H - kHalo;
  return inner ? stencil_rows<false, PAT, MODE, NT>(s_c, P, x0, y0, W, H, gain, wT, wR, out)
               : stencil_rows<true, PAT, MODE, NT>(s_c, P, x0, y0, W, H, gain, wT, wR, out);
}

// Persistent, warp-specialised stencil kernel: one CTA per SM walks the block
// list.  A producer warp stages the complex-cell windows (8 orientations x 48
// rows x 48 floats: a 32 x 32 block plus an 8-pixel halo) as one TMA tensor
// box each, with the block's parameters, into a ring of kStBufs buffers, so
// that up to kStBufs - 1 windows are in flight while 16 consumer warps
// compute the oldest.  Full barriers (TMA bytes) and empty barriers (one
// arrival per consumer warp) order the two sides; there is no CTA-wide
// barrier in the loop.  Every wait is bounded; on expiry the kernel sets
// *fault and stops.
constexpr int kStConsumers = 512;                    // 16 compute warps
constexpr int kStThreads = kStConsumers + 32;        // + the producer warp
constexpr int kStCtasPerSm = 1;                      // resident CTAs per SM (2 with 16-row blocks: no faster)
constexpr int kStBuf = kNumOri * kStH * kStW;        // floats per staging buffer
constexpr int kStBufs = 3;                           // staging ring depth

// Everything a consumer needs about its block, written by the producer.
struct StencilBlk {
  StencilPar P;
  int x0, y0, W, H, pattern;
  float gain, wT, wR;
  StencilOut out;
  unsigned int* maxKey;
};

// One block's record as the producer lanes hold it in registers between
// fetching it from global memory and writing it to shared memory: lanes
// 0..7 the offsets of orientation `lane`, lane 8 the block's scalars, lane 0
// also the tensor map.  Fetching the next block's record one block ahead
// hides the dependent global loads (work item -> descriptor -> fields).
struct StencilPre {
  int x0, y0, W, H;
  int e1, e2, i1, i2, h1, h2;
  int pattern, pitch;
  float gain, wT, wR;
  float *D, *S, *T, *R;
  unsigned int *bits, *maxKey;
  const void* cMap;
};

__device__ __forceinline__ StencilPre stencil_fetch(const ScaleDev* __restrict__ sds, const int2* __restrict__ work,
                                                    int idx, int lane) {
  StencilPre r;
  const int2 item = work[idx];
  const ScaleDev* sd = sds + item.x;
  r.W = sd->dataW;
  r.H = sd->dataH;
  const int nbx = (r.W + kStX - 1) / kStX;
  const int by = item.y / nbx;
  r.x0 = (item.y - by * nbx) * kStX;
  r.y0 = by * kFwY;
  if (lane < kNumOri) {
    r.e1 = sd->es1[lane]; r.e2 = sd->es2[lane]; r.i1 = sd->in1[lane]; r.i2 = sd->in2[lane];
    r.h1 = sd->ih1[lane]; r.h2 = sd->ih2[lane];
  }
  if (lane == kNumOri) {
    r.pattern = sd->pattern; r.pitch = sd->dPitch;
    r.gain = sd->radialGain; r.wT = sd->wTan; r.wR = sd->wRad;
    r.D = sd->D; r.S = sd->S; r.T = sd->T; r.R = sd->R; r.bits = sd->bits; r.maxKey = sd->maxKey;
  }
  if (lane == 0) r.cMap = sd->cMap;
  return r;
}

// Lane `lane` (< 8: orientation lane) of the producer writes the block record.
__device__ __forceinline__ void stencil_put(const StencilPre& r, StencilBlk& B, int lane) {
  const int W = r.W, H = r.H;
  if (lane < kNumOri) {
    const int o = lane;
    StencilPar& P = B.P;
    P.e1[o] = r.e1; P.e2[o] = r.e2; P.i1[o] = r.i1; P.i2[o] = r.i2;
    P.h1[o] = r.h1; P.h2[o] = r.h2;
    P.exlo[o] = 2 * abs(r.e2); P.exhi[o] = W - 2 * abs(r.e2);
    P.eylo[o] = 2 * abs(r.e1); P.eyhi[o] = H - 2 * abs(r.e1);
    P.ixlo[o] = 2 * abs(r.i2); P.ixhi[o] = W - 2 * abs(r.i2);
    P.iylo[o] = 2 * abs(r.i1); P.iyhi[o] = H - 2 * abs(r.i1);
  } else if (lane == kNumOri) {
    B.x0 = r.x0; B.y0 = r.y0; B.W = W; B.H = H; B.pattern = r.pattern;
    B.gain = r.gain; B.wT = r.wT; B.wR = r.wR;
    B.out.D = r.D; B.out.S = r.S; B.out.T = r.T; B.out.R = r.R; B.out.bits = r.bits;
    B.out.pitch = r.pitch;
    B.maxKey = r.maxKey;
  }
}

// One thread: the block's window as one TMA box (48 x 48 x 8 floats at
// x0 - 8, y0 - 8) through the entry's tensor map.  x0 - 8 is a multiple of 4
// floats (16 bytes); parts of the box outside the maps read as zero.  The
// arrive releases the block record written before it.
__device__ __forceinline__ void stencil_stage_tma(const void* cMap, int x0, int y0, float* buf, uint32_t bar) {
  fence_proxy_async();   // the buffer was last read through the generic proxy
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"((uint32_t)(kStBuf * 4))
               : "memory");
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
          "r"(smem_u32(buf)),
      "l"(cMap), "r"(x0 - kHalo), "r"(y0 - kHalo), "r"(0), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void mbar_init_count(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

template <int MODE>
__global__ void __launch_bounds__(kStThreads, kStCtasPerSm)
k_stencil(const ScaleDev* __restrict__ sds, const int2* __restrict__ work, int nwork,
          unsigned int* __restrict__ fault_word) {
  extern __shared__ float4 s_c4[];   // kStBufs buffers of kNumOri x kStH x kStW floats (+128 B for alignment)
  // TMA box destinations are 128-byte aligned.  The offset is added to the
  // shared-memory pointer itself (not through an integer round trip), so
  // that the compiler keeps every access to the window a shared-memory load.
  float* s_buf = reinterpret_cast<float*>(s_c4) + ((128u - (smem_u32(s_c4) & 127u)) & 127u) / 4u;
  __shared__ StencilBlk blk[kStBufs];
  __shared__ __align__(8) uint64_t s_full[kStBufs], s_empty[kStBufs];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  griddep_launch_dependents();
  if ((int)blockIdx.x >= nwork) return;
  const uint32_t full0 = smem_u32(&s_full[0]), empty0 = smem_u32(&s_empty[0]);
  if (t == 0) {
    for (int i = 0; i < kStBufs; ++i) {
      mbar_init_count(full0 + 8 * i, 1);
      mbar_init_count(empty0 + 8 * i, kStConsumers / 32);
    }
    fence_mbar_init();
  }
  __syncthreads();
  griddep_wait();   // the complex cells come from the previous kernel
  const int nk = (nwork - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;   // blocks of this CTA
  if (warp == kStConsumers / 32) {
    // producer warp: block k goes to buffer k mod kStBufs, its use k / kStBufs
    int issued = 0;
    bool expired = false;
    StencilPre cur = stencil_fetch(sds, work, blockIdx.x, lane);
    for (int k = 0; k < nk; ++k) {
      const int b = k % kStBufs, u = k / kStBufs;
      if (u >= 1 && !mbar_wait(empty0 + 8 * b, (u - 1) & 1)) {   // consumers released use u - 1
        expired = true;
        break;
      }
      stencil_put(cur, blk[b], lane);
      __syncwarp();
      if (lane == 0) stencil_stage_tma(cur.cMap, cur.x0, cur.y0, s_buf + b * kStBuf, full0 + 8 * b);
      __syncwarp();
      issued = k + 1;
      if (k + 1 < nk) cur = stencil_fetch(sds, work, blockIdx.x + (k + 1) * gridDim.x, lane);
    }
    if (expired && lane == 0) atomicOr(fault_word, 2u);
    // before the CTA can end, the last copy into each buffer must land
    if (lane == 0) {
      for (int k = issued - 1; k >= 0 && k >= issued - kStBufs; --k)
        mbar_wait(full0 + 8 * (k % kStBufs), (k / kStBufs) & 1);
    }
    return;
  }
  // consumer warps.  The map max is kept per lane across the blocks of one
  // scale and goes out as one atomic per warp when the scale changes (not
  // one per block: consecutive blocks share their scale's max word).
  unsigned int* runKey = nullptr;
  float runMax = -INFINITY;
  auto flush = [&]() {
    float m = runMax;
#pragma unroll
    for (int sh = 16; sh > 0; sh >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, sh));
    if (lane == 0 && runKey && m > -INFINITY) atomicMax(runKey, float_key(m));
  };
  for (int k = 0; k < nk; ++k) {
    const int b = k % kStBufs, u = k / kStBufs;
    if (!mbar_wait(full0 + 8 * b, u & 1)) {
      if (lane == 0) atomicOr(fault_word, 2u);
      break;
    }
    const StencilBlk& B = blk[b];
    const float* s_c = s_buf + b * kStBuf;
    if (B.maxKey != runKey) {
      flush();
      runKey = B.maxKey;
      runMax = -INFINITY;
    }
    float dmax;
    if (B.pattern == 1)
      dmax = stencil_block<1, MODE, kStConsumers>(s_c, B.P, B.x0, B.y0, B.W, B.H, B.gain, B.wT, B.wR, B.out);
    else if (B.pattern == 2)
      dmax = stencil_block<2, MODE, kStConsumers>(s_c, B.P, B.x0, B.y0, B.W, B.H, B.gain, B.wT, B.wR, B.out);
    else
      dmax = stencil_block<0, MODE, kStConsumers>(s_c, B.P, B.x0, B.y0, B.W, B.H, B.gain, B.wT, B.wR, B.out);
    runMax = fmaxf(runMax, dmax);
    __syncwarp();
    if (lane == 0) mbar_arrive(empty0 + 8 * b);   // this warp is done with buffer b and blk[b]
  }
  flush();
}

// ---------------------------------------------------------------------------
// NMS, threshold, compaction
// ---------------------------------------------------------------------------
__device__ __forceinline__ float scale_thresh(const ScaleDev* sd) {
  // cuda_bimp.cu:720-721: float max, double thresh, passed as float
  const float mx = key_float(*sd->maxKey);
  return (float)((double)mx * sd->threshRatio);
}

__device__ __forceinline__ bool is_keypoint(const float* __restrict__ D, int dp, int x, int y, float thr) {
  const float* r0 = D + (size_t)(y - 1) * dp;
  const float* r1 = r0 + dp;
  const float* r2 = r1 + dp;
  const float v = r1[x];
  if (!(v > thr)) return false;   // most pixels: one load
  float dil = fmaxf(fmaxf(r0[x - 1], r0[x]), r0[x + 1]);
  dil = fmaxf(dil, fmaxf(r1[x - 1], r1[x + 1]));
  dil = fmaxf(dil, fmaxf(fmaxf(r2[x - 1], r2[x]), r2[x + 1]));
  return v - dil > 0.f;
}

// Candidate rows are counted by 4 warps each (2 rows per 256-thread block):
// warp q of a row tests the 32-pixel chunks q, q + 4, ... -- strict
// 8-neighbour maximum above the threshold -- and, when the map has decision
// words, stores the chunk's ballot for the write pass.
constexpr int kNmsWarpsPerRow = 4;
constexpr int kNmsRowsPerBlock = 2;
constexpr int kNmsThreads = 32 * kNmsWarpsPerRow * kNmsRowsPerBlock;

__global__ void __launch_bounds__(kNmsThreads)
k_nms_count(const ScaleDev* __restrict__ sds, const int2* __restrict__ rows, int nrows, int* __restrict__ counts) {
  __shared__ int s_cnt[kNmsRowsPerBlock];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int q = warp % kNmsWarpsPerRow, rl = warp / kNmsWarpsPerRow;
  const int r = blockIdx.x * kNmsRowsPerBlock + rl;
  if (threadIdx.x < kNmsRowsPerBlock) s_cnt[threadIdx.x] = 0;
  __syncthreads();
  if (r < nrows) {
    const int2 item = rows[r];
    const ScaleDev* sd = sds + item.x;
    const int off = sd->off;
    const int y = off + 1 + item.y;
    const float thr = scale_thresh(sd);
    const int xEnd = min(sd->dataW - off, sd->dataW - 1);
    const float* __restrict__ D = sd->D;
    const int dp = sd->dPitch;
    unsigned int* __restrict__ mask = sd->nmsMask ? sd->nmsMask + (size_t)item.y * sd->nmsChunks : nullptr;
    const int nch = (xEnd - off - 1 + 31) / 32;
    int n = 0;
#pragma unroll 4
    for (int c = q; c < nch; c += kNmsWarpsPerRow) {
      const int x = off + 1 + 32 * c + lane;
      const unsigned int bal = __ballot_sync(0xffffffffu, x < xEnd && is_keypoint(D, dp, x, y, thr));
      n += __popc(bal);
      if (mask && lane == 0) mask[c] = bal;   // the write pass reads the decisions back
    }
    if (lane == 0 && n) atomicAdd(&s_cnt[rl], n);
  }
  __syncthreads();
  if (threadIdx.x < kNmsRowsPerBlock && blockIdx.x * kNmsRowsPerBlock + threadIdx.x < nrows)
    counts[blockIdx.x * kNmsRowsPerBlock + threadIdx.x] = s_cnt[threadIdx.x];
}

// One warp per candidate row for the write pass.
constexpr int kNmsWriteRows = 8;

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

// One keypoint record of row y at column x, slot idx: subpixel position from
// the parabolas through the 3 samples per axis (cuda_bimp.cuh:114-132),
// cv::KeyPoint fields.
__device__ __forceinline__ void nms_emit(const ScaleDev* __restrict__ sd, const KpOut& out, int y, int x, int idx) {
  const float* __restrict__ D = sd->D;
  const int dp = sd->dPitch;
  const float pyr = sd->pyrstep, kpSize = sd->kpSize;
  const int kpOctave = sd->kpOctave;
  const float* r1 = D + (size_t)y * dp;
  const float xv1 = r1[x - 1], xv2 = r1[x], xv3 = r1[x + 1];
  const float yv1 = r1[x - dp], yv3 = r1[x + dp];
  float xpos = (float)x, ypos = (float)y;
  const float denx = xv1 + xv3 - 2.f * xv2;
  const float deny = yv1 + yv3 - 2.f * xv2;
  const float numx = 0.5f * (xv1 - xv3);
  const float numy = 0.5f * (yv1 - yv3);
  if (denx != 0.f) xpos += __fdiv_rn(numx, denx);
  if (deny != 0.f) ypos += __fdiv_rn(numy, deny);
  float* kpm = out.kp;
  if (out.aos) {   // pt.x, pt.y, size, angle, response, octave, class_id
    float* k = kpm + (size_t)7 * idx;
    k[0] = xpos * pyr;
    k[1] = ypos * pyr;
    k[2] = kpSize;
    k[3] = -1.f;
    k[4] = xv2;
    reinterpret_cast<int*>(k)[5] = kpOctave;
    reinterpret_cast<int*>(k)[6] = 1;
  } else {
    const size_t ld = out.ld;
    kpm[0 * ld + idx] = xpos * pyr;
    kpm[1 * ld + idx] = ypos * pyr;
    reinterpret_cast<int*>(kpm)[2 * ld + idx] = 1;
    reinterpret_cast<int*>(kpm)[3 * ld + idx] = kpOctave;
    kpm[4 * ld + idx] = kpSize;
    kpm[5 * ld + idx] = -1.f;
    kpm[6 * ld + idx] = xv2;
  }
}

// One warp: the records of candidate row `iy` from its stored decision words
// (bit i of word c is the pixel x0 + 32 c + i; nch words), at slots base,
// base + 1, ... (x order).  32 words per round, one per lane: each lane
// writes its word's keypoints at the word's place in the row (a warp prefix
// sum of the word popcounts keeps x order), so a dense row costs as many
// steps as its densest word has bits, not one step per chunk.
__device__ __forceinline__ void nms_write_words(const ScaleDev* __restrict__ sd, const KpOut& out, int y,
                                                const unsigned int* __restrict__ mask, int nch, int x0, int base,
                                                int lane) {
  for (int c0 = 0; c0 < nch && base < out.capacity; c0 += 32) {
    unsigned int word = c0 + lane < nch ? mask[c0 + lane] : 0u;
    const int pc = __popc(word);
    int incl = pc;
#pragma unroll
    for (int m = 1; m < 32; m <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, incl, m);
      if (lane >= m) incl += u;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    int idx = base + incl - pc;
    while (word) {
      const int bit = __ffs(word) - 1;
      word &= word - 1u;
      if (idx < out.capacity) nms_emit(sd, out, y, x0 + 32 * (c0 + lane) + bit, idx);
      ++idx;
    }
    base += total;
  }
}

// The three-kernel path's words: bit i of word c is the pixel off + 1 + 32 c + i.
__device__ __forceinline__ void nms_write_row(const ScaleDev* __restrict__ sd, const KpOut& out, int iy, int base,
                                              int lane) {
  const int off = sd->off;
  const int xEnd = min(sd->dataW - off, sd->dataW - 1);
  const int nch = (xEnd - off - 1 + 31) / 32;
  nms_write_words(sd, out, off + 1 + iy, sd->nmsMask + (size_t)iy * sd->nmsChunks, nch, off + 1, base, lane);
}

// Records of a row in x order at the row's offset (one warp per row).
__global__ void __launch_bounds__(32 * kNmsWriteRows)
k_nms_write(const ScaleDev* __restrict__ sds, const int2* __restrict__ rows, int nrows,
            const int* __restrict__ offsets, const int* __restrict__ imageRowStart,
            const KpOut* __restrict__ outs) {
  const int lane = threadIdx.x & 31;
  const int r = blockIdx.x * kNmsWriteRows + (threadIdx.x >> 5);
  if (r >= nrows) return;
  const int2 item = rows[r];
  const ScaleDev* sd = sds + item.x;
  const KpOut out = outs[sd->image];
  const int base = offsets[r] - offsets[imageRowStart[sd->image]];
  if (base >= out.capacity) return;
  if (sd->nmsMask) {
    nms_write_row(sd, out, item.y, base, lane);
    return;
  }
  // no stored decisions: test each chunk's pixels (one ballot per chunk)
  const int off = sd->off;
  const int y = off + 1 + item.y;
  const float thr = scale_thresh(sd);
  const int xEnd = min(sd->dataW - off, sd->dataW - 1);
  const int nch = (xEnd - off - 1 + 31) / 32;
  int b = base;
  for (int c = 0; c < nch; ++c) {
    const int x = off + 1 + 32 * c + lane;
    const unsigned int bal = __ballot_sync(0xffffffffu, x < xEnd && is_keypoint(sd->D, sd->dPitch, x, y, thr));
    if (!bal) continue;
    if ((bal >> lane) & 1u) {
      const int idx = b + __popc(bal & ((1u << lane) - 1u));
      if (idx < out.capacity) nms_emit(sd, out, y, x, idx);
    }
    b += __popc(bal);
    if (b >= out.capacity) return;
  }
}

// ---------------------------------------------------------------------------
// NMS in two launches: decisions and counts, then the records
// ---------------------------------------------------------------------------
// The candidate rows of an image are cut into pieces of up to 512 pixels,
// in (scale, row, x) order, and grouped kNmsRowsPerCta to a CTA (one warp per
// piece), the same grouping in both kernels.  k_nms_decide stores each
// piece's decision words and the CTA's keypoint count; k_nms_emit gives each
// CTA its image-relative offset as the sum of the counts of the image's
// earlier CTAs (one parallel read of at most a few thousand ints), the pieces
// their offsets within the CTA from the popcounts of their words, and writes
// the records.  No CTA waits for another.
// Aligned decision words of a candidate row: word c covers the pixels
// 32 (first + c) .. 32 (first + c) + 31, first = (off + 1) / 32; pixels outside
// the candidate range (off, xEnd) are 0.
__device__ __forceinline__ void nms_row_words(const ScaleDev* __restrict__ sd, int& first, int& nch) {
  const int off = sd->off;
  const int xEnd = min(sd->dataW - off, sd->dataW - 1);
  first = (off + 1) >> 5;
  nch = xEnd > off + 1 ? ((xEnd - 1) >> 5) - first + 1 : 0;
}

// One warp: the aligned decision words of one piece of candidate row iy
// (stored to the row's mask words) and its keypoint count.  A segment is 128 pixels, four per
// lane: the lane reads them and the rows above and below as 16-byte vectors
// (the row pitch is a multiple of 32 floats), two segments per round, so a
// row costs about one memory latency per 256 pixels; the neighbours across
// lanes come by shuffles, across segments by two scalar loads.  Two segments
// per round keep the kernel within 64 registers (four CTAs per SM).  Each
// lane's four decisions form a nibble; the words are OR-reductions of eight
// lanes' shifted nibbles.
constexpr int kNmsSegBatch = 2;
// A piece is the part of a candidate row inside one 512-pixel-aligned span
// (four segments, sixteen decision words), so that a long row is decided by
// several warps at once.
constexpr int kNmsPieceShift = 9;
__device__ __forceinline__ int nms_decide_piece(const ScaleDev* __restrict__ sd, int iy, int piece, int lane) {
  const int off = sd->off;
  const int y = off + 1 + iy;
  const int W = sd->dataW;
  const int xEnd = min(W - off, W - 1);
  const float thr = scale_thresh(sd);
  const float* __restrict__ D = sd->D;
  const int dp = sd->dPitch;
  const float* __restrict__ rc = D + (size_t)y * dp;
  const float* __restrict__ ru = rc - dp;
  const float* __restrict__ rd = rc + dp;
  int first, nch;
  nms_row_words(sd, first, nch);
  unsigned int* __restrict__ mask = sd->nmsMask + (size_t)iy * sd->nmsChunks;
  if (nch <= 0) return 0;
  const int seg0 = max((off + 1) >> 7, piece << (kNmsPieceShift - 7));
  const int seg1 = min((xEnd - 1) >> 7, ((piece + 1) << (kNmsPieceShift - 7)) - 1);
  int n = 0;
  for (int sb = seg0; sb <= seg1; sb += kNmsSegBatch) {
    float4 c[kNmsSegBatch], u[kNmsSegBatch], d[kNmsSegBatch];
    float cl[kNmsSegBatch], ul[kNmsSegBatch], dl[kNmsSegBatch], cr[kNmsSegBatch], ur[kNmsSegBatch], dr[kNmsSegBatch];
#pragma unroll
    for (int k = 0; k < kNmsSegBatch; ++k) {
      const int x4 = 128 * (sb + k) + 4 * lane;
      const bool in = sb + k <= seg1 && x4 < W;
      c[k] = in ? *reinterpret_cast<const float4*>(rc + x4) : make_float4(0.f, 0.f, 0.f, 0.f);
      u[k] = in ? *reinterpret_cast<const float4*>(ru + x4) : make_float4(0.f, 0.f, 0.f, 0.f);
      d[k] = in ? *reinterpret_cast<const float4*>(rd + x4) : make_float4(0.f, 0.f, 0.f, 0.f);
      // the pixels beyond the lane group: left of lane 0, right of lane 31
      const bool le = in && lane == 0 && x4 >= 1, ri = in && lane == 31 && x4 + 4 < W;
      cl[k] = le ? rc[x4 - 1] : 0.f;
      ul[k] = le ? ru[x4 - 1] : 0.f;
      dl[k] = le ? rd[x4 - 1] : 0.f;
      cr[k] = ri ? rc[x4 + 4] : 0.f;
      ur[k] = ri ? ru[x4 + 4] : 0.f;
      dr[k] = ri ? rd[x4 + 4] : 0.f;
    }
#pragma unroll
    for (int k = 0; k < kNmsSegBatch; ++k) {
      if (sb + k > seg1) break;
      const int x4 = 128 * (sb + k) + 4 * lane;
      // left neighbour column of x4 and right neighbour column of x4 + 3
      float lc = __shfl_up_sync(0xffffffffu, c[k].w, 1), lu = __shfl_up_sync(0xffffffffu, u[k].w, 1),
            ld = __shfl_up_sync(0xffffffffu, d[k].w, 1);
      float rcv = __shfl_down_sync(0xffffffffu, c[k].x, 1), ruv = __shfl_down_sync(0xffffffffu, u[k].x, 1),
            rdv = __shfl_down_sync(0xffffffffu, d[k].x, 1);
      if (lane == 0) { lc = cl[k]; lu = ul[k]; ld = dl[k]; }
      if (lane == 31) { rcv = cr[k]; ruv = ur[k]; rdv = dr[k]; }
      const float cv[6] = {lc, c[k].x, c[k].y, c[k].z, c[k].w, rcv};
      const float uv[6] = {lu, u[k].x, u[k].y, u[k].z, u[k].w, ruv};
      const float dv[6] = {ld, d[k].x, d[k].y, d[k].z, d[k].w, rdv};
      // the 8-neighbour maximum from the column maxima of the rows above and
      // below, shared by adjacent pixels (max is exact, so the order of the
      // comparisons does not matter)
      float vm[6];
#pragma unroll
      for (int q = 0; q < 6; ++q) vm[q] = fmaxf(uv[q], dv[q]);
      // this lane's four decisions as a nibble (bit i: pixel x4 + i)
      unsigned int nib = 0;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int x = x4 + i;
        const float v = cv[i + 1];
        bool keep = false;
        if (x > off && x < xEnd && v > thr) {
          const float dil = fmaxf(fmaxf(vm[i], vm[i + 1]), fmaxf(vm[i + 2], fmaxf(cv[i], cv[i + 2])));
          keep = v - dil > 0.f;
        }
        nib |= (keep ? 1u : 0u) << i;
      }
      n += __popc(nib);
      // word w of the segment (pixels 32 w .. 32 w + 31): the nibbles of
      // lanes 8 w .. 8 w + 7, lane 8 w + l at bits 4 l, OR-ed across the 8 lanes
      unsigned int word = nib << (4 * (lane & 7));
      word |= __shfl_xor_sync(0xffffffffu, word, 1);
      word |= __shfl_xor_sync(0xffffffffu, word, 2);
      word |= __shfl_xor_sync(0xffffffffu, word, 4);
      if ((lane & 7) == 0) {
        const int widx = 4 * (sb + k) + (lane >> 3) - first;
        if (widx >= 0 && widx < nch) mask[widx] = word;
      }
    }
  }
  // the piece's keypoint count (each lane counted its own pixels)
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) n += __shfl_xor_sync(0xffffffffu, n, m);
  return n;
}

__global__ void __launch_bounds__(32 * kNmsRowsPerCta, 4)
k_nms_decide(const ScaleDev* __restrict__ sds, const int2* __restrict__ rows, const NmsCta* __restrict__ ctas,
             int* __restrict__ ctaCount) {
  __shared__ int s_cnt[kNmsRowsPerCta];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const NmsCta cta = ctas[blockIdx.x];
  griddep_launch_dependents();
  griddep_wait();   // the summed maps and their maxima come from the previous kernel
  int cnt = 0;
  if (warp < cta.nRows) {
    const int2 item = rows[cta.rowStart + warp];   // {entry, row | piece << 16}
    cnt = nms_decide_piece(sds + item.x, item.y & 0xffff, item.y >> 16, lane);
  }
  if (lane == 0) s_cnt[warp] = cnt;
  __syncthreads();
  if (threadIdx.x == 0) {
    int total = 0;
    for (int w = 0; w < kNmsRowsPerCta; ++w) total += s_cnt[w];
    ctaCount[blockIdx.x] = total;
  }
}

__global__ void __launch_bounds__(32 * kNmsRowsPerCta)
k_nms_emit(const ScaleDev* __restrict__ sds, const int2* __restrict__ rows, const NmsCta* __restrict__ ctas,
           const int* __restrict__ ctaCount, int* __restrict__ imageTotals, const KpOut* __restrict__ outs) {
  __shared__ int s_cnt[kNmsRowsPerCta];
  __shared__ int s_part[kNmsRowsPerCta];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const NmsCta cta = ctas[blockIdx.x];
  int2 item = make_int2(0, 0);
  int first = 0, wlo = 0, whi = 0, iy = 0;
  griddep_wait();   // the decision words and counts come from k_nms_decide
  // this piece's keypoint count from its decision words
  int cnt = 0;
  if (warp < cta.nRows) {
    item = rows[cta.rowStart + warp];   // {entry, row | piece << 16}
    iy = item.y & 0xffff;
    const int piece = item.y >> 16;
    const ScaleDev* sd = sds + item.x;
    int nch;
    nms_row_words(sd, first, nch);
    wlo = max(0, (piece << (kNmsPieceShift - 5)) - first);
    whi = min(nch, ((piece + 1) << (kNmsPieceShift - 5)) - first);
    const unsigned int* mask = sd->nmsMask + (size_t)iy * sd->nmsChunks;
    for (int c = wlo + lane; c < whi; c += 32) cnt += __popc(mask[c]);
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, m);
  }
  // the counts of the image's earlier CTAs
  int before = 0;
  for (int i = cta.firstCta + t; i < (int)blockIdx.x; i += blockDim.x) before += ctaCount[i];
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) before += __shfl_xor_sync(0xffffffffu, before, m);
  if (lane == 0) {
    s_cnt[warp] = cnt;
    s_part[warp] = before;
  }
  __syncthreads();
  int base = 0, total = 0;
  for (int w = 0; w < kNmsRowsPerCta; ++w) {
    base += s_part[w];
    total += s_cnt[w];
  }
  if (cta.last && t == 0) {
    imageTotals[cta.image] = base + total;
    int* const cnt = outs[cta.image].count;
    if (cnt) *cnt = base + total;
  }
  if (warp < cta.nRows && cnt > 0) {
    for (int w = 0; w < warp; ++w) base += s_cnt[w];
    const ScaleDev* sd = sds + item.x;
    const KpOut out = outs[cta.image];
    if (base < out.capacity)
      nms_write_words(sd, out, sd->off + 1 + iy, sd->nmsMask + (size_t)iy * sd->nmsChunks + wlo, whi - wlo,
                      32 * (first + wlo), base, lane);
  }
}

// ---------------------------------------------------------------------------
// line and edge detection (detectLE_kernel, cuda_bimp.cuh:362-432)
// ---------------------------------------------------------------------------
// Per pixel of one scale: if the summed complex response Ch (the caller's
// map, or sum_o C_o when d_ch is null) is at least 0.1, take the dominant
// orientation (the first strict maximum of C_o > 0), step one pixel along
// (round(cos t), round(sin t)), t = o * 0.392699, and keep the pixel if its
// odd or even response is a strict extremum along that step, the other
// (or the same) response crosses zero across it, and C is a strict maximum
// along it.  Type: 1 positive / 2 negative line (odd zero crossing at an
// even maximum / minimum), 3 positive / 4 negative edge (even zero crossing
// at an odd maximum / minimum; edges override lines, as the reference's
// assignment order does).  Result = C at kept pixels, else 0; orientation t
// at kept pixels, else 0; type 0 where nothing is assigned.  The reference
// reads its neighbours by flat address, which leaves the data at the
// border; here a pixel whose step leaves the data is not kept.
__global__ void __launch_bounds__(256)
k_detect_le(const ScaleDev* __restrict__ sd, const float* __restrict__ ch, int chLd, float* __restrict__ result,
            float* __restrict__ ori, int8_t* __restrict__ type, int ld) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int W = sd->dataW, H = sd->dataH;
  if (x >= W || y >= H) return;
  const float* __restrict__ C = sd->C;
  const float2* __restrict__ Z = sd->Z;
  const long long cs = sd->cStride;
  const size_t at = (size_t)y * sd->cPitch + x;
  float chv;
  if (ch) {
    chv = ch[(size_t)y * chLd + x];
  } else {
    chv = 0.f;
#pragma unroll
    for (int o = 0; o < kNumOri; ++o) chv += C[o * cs + at];
  }
  float res = 0.f, th = 0.f;
  int ty = 0;
  if (!(chv < 0.1f)) {
    int maxori = -1;
    float maxresp = 0.f;
#pragma unroll
    for (int o = 0; o < kNumOri; ++o) {
      const float cur = C[o * cs + at];
      if (cur > maxresp) { maxresp = cur; maxori = o; }
    }
    if (maxori >= 0) {
      const float theta = (float)(maxori * 0.392699);   // cuda_bimp.cuh:400 (double literal)
      const int ox = (int)roundf(cosf(theta)), oy = (int)roundf(sinf(theta));
      const int xp = x + ox, yp = y + oy, xm = x - ox, ym = y - oy;
      if (xp >= 0 && xp < W && yp >= 0 && yp < H && xm >= 0 && xm < W && ym >= 0 && ym < H) {
        const size_t ap = (size_t)yp * sd->cPitch + xp, am = (size_t)ym * sd->cPitch + xm;
        const float2 z0 = Z[maxori * cs + at], zp = Z[maxori * cs + ap], zm = Z[maxori * cs + am];
        const float o0 = z0.y, op = zp.y, om = zm.y, e0 = z0.x, ep = zp.x, em = zm.x;
        const bool romax = o0 > op && o0 > om, romin = o0 < op && o0 < om, rozc = op * om < 0.f;
        const bool remax = e0 > ep && e0 > em, remin = e0 < ep && e0 < em, rezc = ep * em < 0.f;
        const float c0 = C[maxori * cs + at], cp = C[maxori * cs + ap], cm = C[maxori * cs + am];
        const bool keep = (romax || romin || remax || remin) && (rezc || rozc) && !(c0 <= cp || c0 <= cm);
        if (keep) {
          ty = (rezc && romin) ? 4 : (rezc && romax) ? 3 : (rozc && remin) ? 2 : (rozc && remax) ? 1 : 0;
          th = theta;
          res = c0;
        }
      }
    }
  }
  const size_t k = (size_t)y * ld + x;
  result[k] = res;
  ori[k] = th;
  type[k] = (int8_t)ty;
}

#include "adjoint_kernels.cuh"

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

size_t gabor_smem_bytes() { return kGaborSmem; }
int pipelined_tile_max_valid() { return kWsRows; }
size_t stencil_smem_bytes() { return sizeof(float) * kStBufs * kStBuf + 128; }

namespace {
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}
}  // namespace

bool encode_c_maps(const ScaleDev* sds, int n, void* maps, std::string& err) {
  static_assert(sizeof(CUtensorMap) == kTensorMapBytes, "tensor map size");
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) {
    err = "cuTensorMapEncodeTiled is not available from the driver";
    return false;
  }
  CUtensorMap* out = static_cast<CUtensorMap*>(maps);
  for (int e = 0; e < n; ++e) {
    const ScaleDev& d = sds[e];
    const cuuint64_t dims[3] = {(cuuint64_t)d.cPitch, (cuuint64_t)d.cRows, (cuuint64_t)kNumOri};
    const cuuint64_t strides[2] = {(cuuint64_t)d.cPitch * sizeof(float), (cuuint64_t)d.cStride * sizeof(float)};
    const cuuint32_t box[3] = {(cuuint32_t)kStW, (cuuint32_t)kStH, (cuuint32_t)kNumOri};
    const cuuint32_t elem[3] = {1, 1, 1};
    const CUresult r = enc(&out[e], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, d.C, dims, strides, box, elem,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
      err = "cuTensorMapEncodeTiled failed with code " + std::to_string((int)r);
      return false;
    }
  }
  return true;
}

// CTAs of the persistent stencil kernel: one per SM.
static int g_num_sms[64] = {0};
int num_sms() {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return 148;
  if (g_num_sms[dev] == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    g_num_sms[dev] = n;
  }
  return g_num_sms[dev];
}

cudaError_t configure_kernels() {
  const cudaFuncAttribute big = cudaFuncAttributeMaxDynamicSharedMemorySize;
  cudaError_t e = cudaFuncSetAttribute(k_gabor_tiles<false, false>, big, (int)gabor_smem_bytes());
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_gabor_tiles<true, false>, big, (int)gabor_smem_bytes());
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_gabor_tiles<false, true>, big, (int)gabor_smem_bytes());
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_stencil<kStencilD>, big, (int)stencil_smem_bytes());
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_stencil<kStencilDS>, big, (int)stencil_smem_bytes());
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_stencil<kStencilAdj>, big, (int)stencil_smem_bytes());
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_gabor_tiles_bwd, big, (int)kGaborBwdSmem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_gabor_tiles_ws<false>, big, (int)kWsSmem);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_gabor_tiles_ws<true>, big, (int)kWsSmem);
  if (e != cudaSuccess) return e;
  return upload_twiddles();
}

// Launches kernel k with programmatic stream serialisation when pdl is set
// (the kernel must call griddep_wait() before it reads its predecessor's
// output).
template <typename... Params, typename... Args>
static void launch_ex(void (*k)(Params...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, bool pdl,
                      Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, k, static_cast<Params>(args)...);
}

// The keypoint destination descriptor of a context, written in stream order
// from a kernel argument (no host memory involved, so the write is also
// valid inside a stream capture).
__global__ void k_set_out(KpOut* __restrict__ d, KpOut v) { *d = v; }
void launch_set_out(KpOut* d, const KpOut& v, cudaStream_t s) { k_set_out<<<1, 1, 0, s>>>(d, v); }

void launch_pyr(const PyrJob* d_jobs, int njobs, int levels, int maxW, int maxH, cudaStream_t s,
                unsigned int* reset, int resetWords) {
  if (njobs <= 0 || levels <= 0) return;
  const int T = 32 >> (levels - 1);
  dim3 g((maxW + T - 1) / T, (maxH + T - 1) / T, njobs);
  if (levels == 3) k_pyr_down<3><<<g, kPyrThreads, 0, s>>>(d_jobs, reset, resetWords);
  else if (levels == 2) k_pyr_down<2><<<g, kPyrThreads, 0, s>>>(d_jobs, reset, resetWords);
  else k_pyr_down<1><<<g, kPyrThreads, 0, s>>>(d_jobs, reset, resetWords);
}
void launch_gabor(const ScaleDev* d_sd, const TileWork* d_work, int nwork, int grid, unsigned int* d_fault,
                  cudaStream_t s, bool pipelined, bool pdl) {
  if (pipelined)
    launch_ex(k_gabor_tiles_ws<false>, grid, kTileThreads, kWsSmem, s, pdl, d_sd, d_work, nwork);
  else
    launch_ex(k_gabor_tiles<false, false>, grid, kTileThreads, gabor_smem_bytes(), s, pdl, d_sd, d_work, nwork,
              d_fault);
}
void launch_gabor_flt(const ScaleDev* d_sd, const TileWork* d_work, int nwork, unsigned int* d_fault,
                      cudaStream_t s, bool pipelined) {
  if (nwork <= 0) return;
  if (pipelined)
    k_gabor_tiles_ws<true><<<nwork, kTileThreads, kWsSmem, s>>>(d_sd, d_work, nwork);
  else
    k_gabor_tiles<true, false><<<nwork, kTileThreads, gabor_smem_bytes(), s>>>(d_sd, d_work, nwork, d_fault);
}
void launch_gabor_keep_z(const ScaleDev* d_sd, const TileWork* d_work, int nwork, unsigned int* d_fault,
                         cudaStream_t s) {
  if (nwork > 0)
    k_gabor_tiles<false, true><<<nwork, kTileThreads, gabor_smem_bytes(), s>>>(d_sd, d_work, nwork, d_fault);
}
void launch_detect_le(const ScaleDev* d_sd, int dataW, int dataH, const float* d_ch, int chLd, float* d_result,
                      float* d_ori, int8_t* d_type, int ld, cudaStream_t s) {
  dim3 b(32, 8), g((dataW + 31) / 32, (dataH + 7) / 8);
  k_detect_le<<<g, b, 0, s>>>(d_sd, d_ch, chLd, d_result, d_ori, d_type, ld);
}
void launch_pyr_f(const PyrJobF* d_jobs, int njobs, int maxW, int maxH, cudaStream_t s) {
  dim3 b(32, 8), g((maxW + 31) / 32, (maxH + 7) / 8, njobs);
  k_pyr_down_f<<<g, b, 0, s>>>(d_jobs);
}
void launch_pyr_f_adj(const PyrJobF* d_jobs, int njobs, int maxW, int maxH, cudaStream_t s) {
  dim3 b(32, 8), g((maxW + 31) / 32, (maxH + 7) / 8, njobs);
  k_pyr_down_f_adj<<<g, b, 0, s>>>(d_jobs);
}
void launch_masked_loss(const ScaleDev* d_sd, const int2* d_work, int nwork, double* d_loss, double* d_gparams,
                        cudaStream_t s) {
  if (nwork > 0) k_masked_loss<<<std::min(nwork, 4 * num_sms()), 256, 0, s>>>(d_sd, d_work, nwork, d_loss, d_gparams);
}
void launch_stencil_bwd(const ScaleDev* d_sd, const int2* d_work, int nwork, cudaStream_t s) {
  if (nwork > 0) k_stencil_bwd<<<nwork, kStBwThreads, 0, s>>>(d_sd, d_work);
}

void launch_gabor_bwd(const ScaleDev* d_sd, const TileWork* d_work, int nwork, int grid, float2* d_xscratch,
                      double* d_gparams, cudaStream_t s) {
  if (nwork > 0)
    k_gabor_tiles_bwd<<<std::min(grid, nwork), kTileThreads, kGaborBwdSmem, s>>>(d_sd, d_work, nwork, d_xscratch,
                                                                                 d_gparams);
}
void launch_stencil(const ScaleDev* d_sd, const int2* d_work, int nwork, unsigned int* d_fault, cudaStream_t s,
                    int mode, bool pdl) {
  if (nwork <= 0) return;
  const int grid = std::min(nwork, kStCtasPerSm * num_sms());
  if (mode == kStencilDS)
    launch_ex(k_stencil<kStencilDS>, grid, kStThreads, stencil_smem_bytes(), s, pdl, d_sd, d_work, nwork, d_fault);
  else if (mode == kStencilAdj)
    launch_ex(k_stencil<kStencilAdj>, grid, kStThreads, stencil_smem_bytes(), s, pdl, d_sd, d_work, nwork, d_fault);
  else
    launch_ex(k_stencil<kStencilD>, grid, kStThreads, stencil_smem_bytes(), s, pdl, d_sd, d_work, nwork, d_fault);
}
void launch_nms_two_pass(const ScaleDev* d_sd, const int2* d_rows, const NmsCta* d_ctas, int nctas, int* d_ctaCount,
                         int* d_totals, const KpOut* d_outs, cudaStream_t s, bool pdl) {
  if (nctas <= 0) return;
  launch_ex(k_nms_decide, nctas, 32 * kNmsRowsPerCta, 0, s, pdl, d_sd, d_rows, d_ctas, d_ctaCount);
  launch_ex(k_nms_emit, nctas, 32 * kNmsRowsPerCta, 0, s, pdl, d_sd, d_rows, d_ctas, d_ctaCount, d_totals, d_outs);
}
void launch_nms(const ScaleDev* d_sd, const int2* d_rows, int nrows, int* d_counts, int* d_offsets,
                const int* d_imageRowStart, int nImages, int* d_totals, const KpOut* d_outs,
                cudaStream_t s) {
  if (nrows > 0)
    k_nms_count<<<(nrows + kNmsRowsPerBlock - 1) / kNmsRowsPerBlock, kNmsThreads, 0, s>>>(d_sd, d_rows, nrows,
                                                                                           d_counts);
  k_scan<<<1, 1024, 0, s>>>(d_counts, d_offsets, nrows, d_imageRowStart, nImages, d_totals);
  if (nrows > 0)
    k_nms_write<<<(nrows + kNmsWriteRows - 1) / kNmsWriteRows, 32 * kNmsWriteRows, 0, s>>>(
        d_sd, d_rows, nrows, d_offsets, d_imageRowStart, d_outs);
}

}  // namespace bimp_b200

// Register-level DFT building blocks and the shared-memory layout helpers of
// the 128x128 tile FFT.
//
// A 128-point transform is split as n = n1 + 8*n2, k = k2 + 16*k1:
//   forward  pass A: 16-point DFT over n2 (stride-8 elements), twiddle
//                    w128^(n1*k2), store at position n1 + 8*k2;
//            pass B: 8-point DFT over n1 (8 consecutive positions), output
//                    k1 stored at position 8*k2 + k1  (digit-permuted order);
//   inverse  pass B': 8-point inverse DFT over k1, twiddle w128^(-n1*k2);
//            pass A': 16-point inverse DFT over k2 -> natural order.
// Transforms are unnormalised; the 1/128^2 factor lives in the spectra.
#pragma once

#include <cuda_runtime.h>

namespace bimp_b200 {

#ifndef BIMP_HD
#define BIMP_HD __host__ __device__ __forceinline__
#endif

BIMP_HD float2 c_add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
BIMP_HD float2 c_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
BIMP_HD float2 c_mul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
BIMP_HD float2 c_mulc(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
BIMP_HD float2 c_scale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by -i (forward) or +i (inverse)
template <bool INV>
BIMP_HD float2 c_rot(float2 a) {
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

constexpr float kR2 = 0.70710678118654752440f;   // cos(pi/4)
constexpr float kC16 = 0.92387953251128675613f;  // cos(pi/8)
constexpr float kS16 = 0.38268343236508977173f;  // sin(pi/8)

// 4-point DFT in place (natural in, natural out).
template <bool INV>
BIMP_HD void dft4(float2& a0, float2& a1, float2& a2, float2& a3) {
  const float2 t0 = c_add(a0, a2), t1 = c_sub(a0, a2);
  const float2 t2 = c_add(a1, a3), t3 = c_rot<INV>(c_sub(a1, a3));
  a0 = c_add(t0, t2);
  a2 = c_sub(t0, t2);
  a1 = c_add(t1, t3);
  a3 = c_sub(t1, t3);
}

// w = exp(-+ 2 pi i j / 8) multiplications for j = 1, 2, 3.
template <bool INV> BIMP_HD float2 w8_1(float2 a) {
  // (1 -+ i)/sqrt2
  return INV ? make_float2(kR2 * (a.x - a.y), kR2 * (a.x + a.y))
             : make_float2(kR2 * (a.x + a.y), kR2 * (a.y - a.x));
}
template <bool INV> BIMP_HD float2 w8_3(float2 a) {
  // (-1 -+ i)/sqrt2
  return INV ? make_float2(-kR2 * (a.x + a.y), kR2 * (a.x - a.y))
             : make_float2(kR2 * (a.y - a.x), -kR2 * (a.x + a.y));
}

// 8-point DFT, natural in / natural out.
template <bool INV>
BIMP_HD void dft8(float2 (&v)[8]) {
  dft4<INV>(v[0], v[2], v[4], v[6]);
  dft4<INV>(v[1], v[3], v[5], v[7]);
  // odd branch outputs at v[1],v[3],v[5],v[7] correspond to k = 0..3
  const float2 o0 = v[1];
  const float2 o1 = w8_1<INV>(v[3]);
  const float2 o2 = c_rot<INV>(v[5]);
  const float2 o3 = w8_3<INV>(v[7]);
  const float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  v[0] = c_add(e0, o0); v[4] = c_sub(e0, o0);
  v[1] = c_add(e1, o1); v[5] = c_sub(e1, o1);
  v[2] = c_add(e2, o2); v[6] = c_sub(e2, o2);
  v[3] = c_add(e3, o3); v[7] = c_sub(e3, o3);
}

template <bool INV>
BIMP_HD float2 w16(float2 a, float c, float s) {
  // a * (c -+ i s)
  return INV ? make_float2(a.x * c - a.y * s, a.x * s + a.y * c)
             : make_float2(a.x * c + a.y * s, a.y * c - a.x * s);
}

// 16-point DFT, natural in / natural out (radix 4 x 4).
template <bool INV>
BIMP_HD void dft16(float2 (&v)[16]) {
  // step 1: 4-point DFTs over n_b for each n_a (elements n_a + 4 n_b)
  dft4<INV>(v[0], v[4], v[8], v[12]);
  dft4<INV>(v[1], v[5], v[9], v[13]);
  dft4<INV>(v[2], v[6], v[10], v[14]);
  dft4<INV>(v[3], v[7], v[11], v[15]);
  // slot n_a + 4 k_b now holds u[n_a][k_b]; twiddle by w16^(n_a k_b)
  v[5] = w16<INV>(v[5], kC16, kS16);     // 1*1
  v[9] = w16<INV>(v[9], kR2, kR2);       // 1*2
  v[13] = w16<INV>(v[13], kS16, kC16);   // 1*3
  v[6] = w16<INV>(v[6], kR2, kR2);       // 2*1
  v[10] = c_rot<INV>(v[10]);             // 2*2 = 4
  v[14] = w16<INV>(v[14], -kR2, kR2);    // 2*3 = 6
  v[7] = w16<INV>(v[7], kS16, kC16);     // 3*1
  v[11] = w16<INV>(v[11], -kR2, kR2);    // 3*2 = 6
  v[15] = w16<INV>(v[15], -kC16, -kS16); // 3*3 = 9
  // step 2: 4-point DFTs over n_a for each k_b (slots 4 k_b .. 4 k_b + 3)
  dft4<INV>(v[0], v[1], v[2], v[3]);
  dft4<INV>(v[4], v[5], v[6], v[7]);
  dft4<INV>(v[8], v[9], v[10], v[11]);
  dft4<INV>(v[12], v[13], v[14], v[15]);
  // slot 4 k_b + k_a holds X[k_b + 4 k_a]: transpose 4x4 into natural order
  float2 t;
  t = v[1]; v[1] = v[4]; v[4] = t;
  t = v[2]; v[2] = v[8]; v[8] = t;
  t = v[3]; v[3] = v[12]; v[12] = t;
  t = v[6]; v[6] = v[9]; v[9] = t;
  t = v[7]; v[7] = v[13]; v[13] = t;
  t = v[11]; v[11] = v[14]; v[14] = t;
}

// Bank swizzle of a position inside a 128-element row: rotates each group
// of 8 by (p >> 4) so that both the stride-8 and the contiguous-8 passes are
// conflict-free with a row stride of 136 complex.
BIMP_HD int phys(int p) { return (p & ~7) | ((p + (p >> 4)) & 7); }

}  // namespace bimp_b200

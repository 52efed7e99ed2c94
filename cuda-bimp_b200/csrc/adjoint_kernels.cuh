// Kernels of the adjoint of L = sum_s sum M_s * D_s (included by kernels.cu
// inside namespace bimp_b200, after the forward kernels).
//
//   k_pyr_down_f        float pyramid level (pyrDown without uint8 rounding)
//   k_pyr_down_f_adj    its transpose (scatter-add of the 5x5 taps)
//   k_masked_loss       sum M * D, T and R terms are handled in k_stencil_bwd
//   k_stencil_bwd       gather form of d L / d C over the stencil window
//   k_wrap_merge        column dataW of the window is torus (r+1, 0) when
//                       fftW == dataW: its gradient moves there
//   k_gabor_tiles_bwd   per tile: image spectrum X, then per orientation
//                       a = dL/dC * z/|z|, A = FFT(a), alpha/rho dot products
//                       sum dG * Re(conj(A) X), and Re IFFT(A G) into the
//                       window gradient; finally scattered to the level
#pragma once

__global__ void k_pyr_down_f(const PyrJobF* __restrict__ jobs) {
  const PyrJobF j = jobs[blockIdx.z];
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= j.dw || y >= j.dh) return;
  const float w5[5] = {1.f, 4.f, 6.f, 4.f, 1.f};
  int cols[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) cols[k] = reflect101(2 * x + k - 2, j.sw);
  float acc = 0.f;
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    const float* row = j.src + (size_t)reflect101(2 * y + i - 2, j.sh) * j.sp;
    float h = 0.f;
#pragma unroll
    for (int k = 0; k < 5; ++k) h += w5[k] * row[cols[k]];
    acc += w5[i] * h;
  }
  j.dst[(size_t)y * j.dp + x] = acc * (1.0f / 256.0f);
}

// g_src(r101(2y+i), r101(2x+j)) += w_i w_j / 256 * g_dst(y, x)
__global__ void k_pyr_down_f_adj(const PyrJobF* __restrict__ jobs) {
  const PyrJobF j = jobs[blockIdx.z];
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= j.dw || y >= j.dh) return;
  const float g = j.src[(size_t)y * j.sp + x] * (1.0f / 256.0f);   // here src = level l gradient
  if (g == 0.f) return;
  const float w5[5] = {1.f, 4.f, 6.f, 4.f, 1.f};
  int cols[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) cols[k] = reflect101(2 * x + k - 2, j.sw);
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    float* row = j.dst + (size_t)reflect101(2 * y + i - 2, j.sh) * j.dp;
#pragma unroll
    for (int k = 0; k < 5; ++k) atomicAdd(row + cols[k], w5[i] * w5[k] * g);
  }
}

__device__ __forceinline__ void block_add_double(double v, double* dst) {
#pragma unroll
  for (int m = 16; m > 0; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
  __shared__ double s_part[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) s_part[wid] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += s_part[k];
    atomicAdd(dst, s);
  }
}

// sum over the 32x32 block of M * D (work list of the forward stencil).
__global__ void __launch_bounds__(256) k_masked_loss(const ScaleDev* __restrict__ sds, const int2* __restrict__ work,
                                                     double* __restrict__ loss) {
  const int2 item = work[blockIdx.x];
  const ScaleDev* sd = sds + item.x;
  const int W = sd->dataW, H = sd->dataH;
  const int nbx = (W + kStX - 1) / kStX;
  const int by = item.y / nbx, bx = item.y - by * nbx;
  double acc = 0.0;
  const int x = bx * kStX + (threadIdx.x & 31);
  for (int i = threadIdx.x >> 5; i < kStY; i += 8) {
    const int y = by * kStY + i;
    if (x < W && y < H) acc += (double)sd->M[(size_t)y * W + x] * (double)sd->D[(size_t)y * sd->dPitch + x];
  }
  block_add_double(acc, loss);
}

// --- stencil backward ------------------------------------------------------
constexpr int kBwHalo = 16;                    // C staged +-16 around the block
constexpr int kBwCW = kStX + 2 * kBwHalo;      // 64
constexpr int kBwQW = kStX + 2 * kHalo;        // 48: source pixels +-8
constexpr size_t kStencilBwdSmem = sizeof(float) * (size_t)kNumOri * kBwCW * kBwCW;   // 128 KB

// Per source pixel q and orientation o, the ReLU states the forward took:
// bit 4o: double-stopped d > 0, 4o+1: tangential t > 0, 4o+2: radial r > 0,
// 4o+3: first radial term r1 > 0; each gated by the orientation's bounds test.
__global__ void __launch_bounds__(256, 1)
k_stencil_bwd(const ScaleDev* __restrict__ sds, const int2* __restrict__ work, double* __restrict__ gparams) {
  extern __shared__ float4 s_raw4[];
  float* sC = reinterpret_cast<float*>(s_raw4);                  // [8][64][64]
  __shared__ float sM[kBwQW * kBwQW];                            // loss weights +-8
  __shared__ unsigned int sBits[kBwQW * kBwQW];
  __shared__ StencilPar P;
  const int2 item = work[blockIdx.x];
  const ScaleDev* __restrict__ sd = sds + item.x;
  const int W = sd->dataW, H = sd->dataH;
  const int nbx = (W + 1 + kStX - 1) / kStX;
  const int by = item.y / nbx, bx = item.y - by * nbx;
  const int x0 = bx * kStX, y0 = by * kStY;
  const int t = threadIdx.x;
  const float gain = sd->radialGain, wT = sd->wTan, wR = sd->wRad;
  if (t < kNumOri) {
    const int o = t;
    const int e1 = sd->es1[o], e2 = sd->es2[o], i1 = sd->in1[o], i2 = sd->in2[o];
    P.e1[o] = e1; P.e2[o] = e2; P.i1[o] = i1; P.i2[o] = i2;
    P.h1[o] = sd->ih1[o]; P.h2[o] = sd->ih2[o];
    P.exlo[o] = 2 * abs(e2); P.exhi[o] = W - 2 * abs(e2);
    P.eylo[o] = 2 * abs(e1); P.eyhi[o] = H - 2 * abs(e1);
    P.ixlo[o] = 2 * abs(i2); P.ixhi[o] = W - 2 * abs(i2);
    P.iylo[o] = 2 * abs(i1); P.iyhi[o] = H - 2 * abs(i1);
  }
  // stage C over rows y0-16 .. y0+47 and cols x0-16 .. x0+47 (window reads)
  const float* __restrict__ C = sd->C;
  const int cPitch = sd->cPitch;
  const long long cStride = sd->cStride;
  for (int idx = t; idx < kNumOri * kBwCW * kBwCW; idx += 256) {
    const int row = idx / kBwCW, lx = idx - row * kBwCW;
    const int o = row / kBwCW, ly = row - o * kBwCW;
    const int gy = y0 - kBwHalo + ly, gx = x0 - kBwHalo + lx;
    float v = 0.f;
    if (gy >= 0 && gy <= H && gx >= 0 && gx <= W) {
      int ry = gy, rx = gx;
      if (sd->wrapW && gx == W) { rx = 0; ry = gy + 1; }
      v = C[(size_t)o * cStride + (size_t)ry * cPitch + rx];
    }
    sC[idx] = v;
  }
  for (int idx = t; idx < kBwQW * kBwQW; idx += 256) {
    const int ly = idx / kBwQW, lx = idx - ly * kBwQW;
    const int gy = y0 - kHalo + ly, gx = x0 - kHalo + lx;
    sM[idx] = (gy >= 0 && gy < H && gx >= 0 && gx < W) ? sd->M[(size_t)gy * W + gx] : 0.f;
  }
  __syncthreads();
  // phase 1: ReLU states of every source pixel q within +-8 of the block,
  // and sum M*T, M*R over the block's own pixels
  double accT = 0.0, accR = 0.0;
  for (int idx = t; idx < kBwQW * kBwQW; idx += 256) {
    const int qy = idx / kBwQW, qx = idx - qy * kBwQW;
    const int y = y0 - kHalo + qy, x = x0 - kHalo + qx;
    unsigned int bits = 0;
    if (y >= 0 && y < H && x >= 0 && x < W) {
      const int cy = qy + (kBwHalo - kHalo), cx = qx + (kBwHalo - kHalo);
      float T = 0.f, R = 0.f;
#pragma unroll
      for (int o = 0; o < kNumOri; ++o) {
        const float* c = sC + (o * kBwCW + cy) * kBwCW + cx;
        if (x >= P.exlo[o] && x <= P.exhi[o] && y >= P.eylo[o] && y <= P.eyhi[o]) {
          const int o1 = P.e1[o], o2 = P.e2[o];
          const float d = fmaf(-0.5f, c[2 * o1 * kBwCW - 2 * o2], fmaf(-0.5f, c[-2 * o1 * kBwCW + 2 * o2], c[0]));
          if (d > 0.f) bits |= 1u << (4 * o);
        }
        if (x >= P.ixlo[o] && x <= P.ixhi[o] && y >= P.iylo[o] && y <= P.iyhi[o]) {
          const int i1 = P.i1[o], i2 = P.i2[o], h1 = P.h1[o], h2 = P.h2[o];
          const float* cp = sC + (((o + 4) & 7) * kBwCW + cy) * kBwCW + cx;
          const float centre = c[0];
          const float tt = c[-i1 * kBwCW - i2] - centre;
          if (tt > 0.f) { bits |= 1u << (4 * o + 1); T += tt; }
          const float r1 = centre - gain * cp[h1 * kBwCW + h2];
          const float r = (r1 > 0.f ? r1 : 0.f) + centre - gain * cp[-h1 * kBwCW - h2];
          if (r > 0.f) { bits |= 1u << (4 * o + 2); R += r; }
          if (r1 > 0.f) bits |= 1u << (4 * o + 3);
        }
      }
      if (qy >= kHalo && qy < kHalo + kStY && qx >= kHalo && qx < kHalo + kStX) {
        accT += (double)sM[idx] * T;
        accR += (double)sM[idx] * R;
      }
    }
    sBits[idx] = bits;
  }
  __syncthreads();
  // phase 2: gather d L / d C_o(p) for the block's window positions p
  float* __restrict__ gC = sd->gC;
  const int lx = t & 31;
  for (int ly = t >> 5; ly < kStY; ly += 8) {
    const int py = y0 + ly, px = x0 + lx;
    if (py > H || px > W) continue;
    const int qy = ly + kHalo, qx = lx + kHalo;   // p in source-pixel coordinates
#pragma unroll
    for (int o = 0; o < kNumOri; ++o) {
      const int o1 = P.e1[o], o2 = P.e2[o], i1 = P.i1[o], i2 = P.i2[o];
      const int op = (o + 4) & 7;
      const int ph1 = P.h1[op], ph2 = P.h2[op];
      auto at = [&](int dy, int dx) { return (qy + dy) * kBwQW + (qx + dx); };
      float g = 0.f;
      // double-stopped: centre, and the two -1/2 taps
      {
        const int k0 = at(0, 0), ka = at(2 * o1, -2 * o2), kb = at(-2 * o1, 2 * o2);
        if (sBits[k0] & (1u << (4 * o))) g += sM[k0];
        if (sBits[ka] & (1u << (4 * o))) g -= 0.5f * sM[ka];
        if (sBits[kb] & (1u << (4 * o))) g -= 0.5f * sM[kb];
      }
      // tangential: p is read by q = p + i (as C(q - i)) and by q = p (centre)
      {
        const int kq = at(i1, i2), k0 = at(0, 0);
        if (sBits[kq] & (1u << (4 * o + 1))) g += -wT * sM[kq];
        if (sBits[k0] & (1u << (4 * o + 1))) g -= -wT * sM[k0];
      }
      // radial, o as the centre orientation
      {
        const int k0 = at(0, 0);
        const unsigned int b = sBits[k0];
        if (b & (1u << (4 * o + 2))) g += -wR * sM[k0] * ((b & (1u << (4 * o + 3))) ? 2.f : 1.f);
      }
      // radial, o as the perpendicular map of op: read at q + h (r1) and q - h (r)
      {
        const int k1 = at(-ph1, -ph2), k2 = at(ph1, ph2);
        const unsigned int b1 = sBits[k1], b2 = sBits[k2];
        if ((b1 & (1u << (4 * op + 2))) && (b1 & (1u << (4 * op + 3)))) g -= gain * (-wR * sM[k1]);
        if (b2 & (1u << (4 * op + 2))) g -= gain * (-wR * sM[k2]);
      }
      gC[(size_t)o * cStride + (size_t)py * cPitch + px] = g;
    }
  }
  block_add_double(-(double)wT * accT, gparams + 2);
  block_add_double(-(double)wR * accR, gparams + 3);
}

// fftW == dataW: the stencils read column dataW of row r from (r+1, 0).
__global__ void k_wrap_merge(const ScaleDev* __restrict__ sds, const int* __restrict__ entries, int n) {
  const int e = entries[blockIdx.y];
  const ScaleDev* sd = sds + e;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r > sd->dataH) return;
  for (int o = 0; o < kNumOri; ++o) {
    float* g = sd->gC + (size_t)o * sd->cStride;
    const float v = g[(size_t)r * sd->cPitch + sd->dataW];
    g[(size_t)r * sd->cPitch + sd->dataW] = 0.f;
    g[(size_t)(r + 1) * sd->cPitch] += v;
  }
}

// --- tile backward -----------------------------------------------------------
constexpr int kGaborBwdSmem = kSmemW + kSmemXh + kSmemTw + kSmemMaps;

__global__ void __launch_bounds__(kTileThreads, 1)
k_gabor_tiles_bwd(const ScaleDev* __restrict__ sds, const TileWork* __restrict__ work, int nwork,
                  float* __restrict__ gwin, double* __restrict__ gparams) {
  extern __shared__ float4 smem4b[];
  char* base = reinterpret_cast<char*>(smem4b);
  float2* W = reinterpret_cast<float2*>(base);
  float2* Xh = reinterpret_cast<float2*>(base + kSmemW);
  float2* tw = reinterpret_cast<float2*>(base + kSmemW + kSmemXh);
  short* rmap = reinterpret_cast<short*>(base + kSmemW + kSmemXh + kSmemTw);
  short* cmap = rmap + kTile;
  const int t = threadIdx.x;
  if (t < 8 * 17) {
    const int n1 = t / 17, k2 = t % 17;
    tw[t] = k2 < 16 ? c_w128[(n1 * k2) & 127] : make_float2(0.f, 0.f);
  }
  double accA = 0.0, accR = 0.0;
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const TileWork item = work[w];
    const ScaleDev* sd = sds + item.entry;
    const int kX = sd->kX, V = sd->V;
    const int ty = item.tile / sd->tilesX, tx = item.tile - ty * sd->tilesX;
    const int R0 = ty * V, C0 = tx * V;
    float* __restrict__ acc = gwin + (size_t)w * kTile * kTile;
    __syncthreads();
    tile_forward_spectrum<true>(sd, R0, C0, W, Xh, tw, rmap, cmap, t);
    const int cRows = sd->cRows, cCols = sd->cCols, cPitch = sd->cPitch;
    const long long cStride = sd->cStride;
    for (int o = 0; o < kNumOri; ++o) {
      // a = dL/dC * z / |z| on the valid outputs, zero elsewhere
      for (int j = t; j < kTile * kTile; j += kTileThreads) {
        const int y = j >> 7, x = j & 127;
        float2 a = make_float2(0.f, 0.f);
        const int gy = R0 + y - kX, gx = C0 + x - kX;
        if (y >= kX && y < kX + V && x >= kX && x < kX + V && gy < cRows && gx < cCols) {
          const size_t k = (size_t)o * cStride + (size_t)gy * cPitch + gx;
          const float2 z = sd->Z[k];
          const float m = sqrtf(z.x * z.x + z.y * z.y);
          if (m > 0.f) {
            const float s = sd->gC[k] / m;
            a = make_float2(s * z.x, s * z.y);
          }
        }
        W[widx(y, x)] = a;
      }
      __syncthreads();
      // forward FFT of a: x-dim on the valid rows (others are zero), then y-dim
      for (int j = t; j < V * 8; j += kTileThreads) {
        const int y = kX + (j >> 3), n1 = j & 7;
        float2 v[16];
#pragma unroll
        for (int m = 0; m < 16; ++m) v[m] = W[widx(y, n1 + 8 * m)];
        dft16<false>(v);
#pragma unroll
        for (int k2 = 0; k2 < 16; ++k2) W[widx(y, n1 + 8 * k2)] = c_mul(v[k2], tw[n1 * 17 + k2]);
      }
      __syncthreads();
      for (int j = t; j < V * 16; j += kTileThreads) {
        const int y = kX + (j >> 4), k2 = j & 15;
        float2 v[8];
#pragma unroll
        for (int n1 = 0; n1 < 8; ++n1) v[n1] = W[widx(y, 8 * k2 + n1)];
        dft8<false>(v);
#pragma unroll
        for (int k1 = 0; k1 < 8; ++k1) W[widx(y, 8 * k2 + k1)] = v[k1];
      }
      __syncthreads();
#pragma unroll
      for (int it = 0; it < 2; ++it) {
        const int j = t + it * kTileThreads;
        const int p = j & 127, n1 = j >> 7;
        float2 v[16];
#pragma unroll
        for (int m = 0; m < 16; ++m) v[m] = W[widx(n1 + 8 * m, p)];
        dft16<false>(v);
#pragma unroll
        for (int k2 = 0; k2 < 16; ++k2) W[widx(n1 + 8 * k2, p)] = c_mul(v[k2], tw[n1 * 17 + k2]);
      }
      __syncthreads();
#pragma unroll
      for (int it = 0; it < 4; ++it) {
        const int j = t + it * kTileThreads;
        const int p = j & 127, k2 = j >> 7;
        float2 v[8];
#pragma unroll
        for (int n1 = 0; n1 < 8; ++n1) v[n1] = W[widx(8 * k2 + n1, p)];
        dft8<false>(v);
#pragma unroll
        for (int k1 = 0; k1 < 8; ++k1) W[widx(8 * k2 + k1, p)] = v[k1];
      }
      __syncthreads();
      // parameter dot products and the product A * G, at permuted (py, p)
      {
        const float* G = sd->G + (size_t)o * kSpecFloats;
        const float* dA = sd->dGa + (size_t)o * kSpecFloats;
        const float* dR = sd->dGr + (size_t)o * kSpecFloats;
        float sa = 0.f, sr = 0.f;
        for (int j = t; j < kTile * kTile; j += kTileThreads) {
          const int py = j >> 7, p = j & 127;
          const int k = widx(py, p);
          const float2 A = W[k];
          const float2 X = spectrum_at(Xh, py, p);
          const float re = A.x * X.x + A.y * X.y;     // Re(conj(A) X)
          sa = fmaf(__ldg(dA + j), re, sa);
          sr = fmaf(__ldg(dR + j), re, sr);
          W[k] = c_scale(A, __ldg(G + j));
        }
        accA += sa;
        accR += sr;
      }
      __syncthreads();
      // inverse FFT of A * G over the whole window; Re -> window gradient
#pragma unroll
      for (int it = 0; it < 4; ++it) {
        const int j = t + it * kTileThreads;
        const int p = j & 127, k2 = j >> 7;
        float2 v[8];
#pragma unroll
        for (int k1 = 0; k1 < 8; ++k1) v[k1] = W[widx(8 * k2 + k1, p)];
        dft8<true>(v);
#pragma unroll
        for (int n1 = 0; n1 < 8; ++n1) W[widx(8 * k2 + n1, p)] = c_mulc(v[n1], tw[n1 * 17 + k2]);
      }
      __syncthreads();
#pragma unroll
      for (int it = 0; it < 2; ++it) {
        const int j = t + it * kTileThreads;
        const int p = j & 127, n1 = j >> 7;
        float2 v[16];
#pragma unroll
        for (int k2 = 0; k2 < 16; ++k2) v[k2] = W[widx(8 * k2 + n1, p)];
        dft16<true>(v);
#pragma unroll
        for (int n2 = 0; n2 < 16; ++n2) W[widx(n1 + 8 * n2, p)] = v[n2];
      }
      __syncthreads();
#pragma unroll
      for (int it = 0; it < 4; ++it) {
        const int j = t + it * kTileThreads;
        const int y = j >> 4, k2 = j & 15;
        float2 v[8];
#pragma unroll
        for (int k1 = 0; k1 < 8; ++k1) v[k1] = W[widx(y, 8 * k2 + k1)];
        dft8<true>(v);
#pragma unroll
        for (int n1 = 0; n1 < 8; ++n1) W[widx(y, 8 * k2 + n1)] = c_mulc(v[n1], tw[n1 * 17 + k2]);
      }
      __syncthreads();
#pragma unroll
      for (int it = 0; it < 2; ++it) {
        const int j = t + it * kTileThreads;
        const int y = j >> 3, n1 = j & 7;
        float2 v[16];
#pragma unroll
        for (int k2 = 0; k2 < 16; ++k2) v[k2] = W[widx(y, 8 * k2 + n1)];
        dft16<true>(v);
#pragma unroll
        for (int n2 = 0; n2 < 16; ++n2) {
          float* dst = acc + y * kTile + n1 + 8 * n2;
          *dst = o == 0 ? v[n2].x : *dst + v[n2].x;
        }
      }
      __syncthreads();
    }
    // window gradient -> float level, through the padded-torus index maps
    float* __restrict__ gl = sd->gLvl;
    const int gp = sd->lvlPitchF;
    for (int j = t; j < kTile * kTile; j += kTileThreads) {
      const int y = j >> 7, x = j & 127;
      const float g = acc[j];
      if (g != 0.f) atomicAdd(gl + (size_t)rmap[y] * gp + cmap[x], kFloatLevelScale * g);
    }
  }
  block_add_double(accA, gparams + 0);
  block_add_double(accR, gparams + 1);
}

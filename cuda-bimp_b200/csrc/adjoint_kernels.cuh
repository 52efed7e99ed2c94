// Kernels of the adjoint of L = sum_s sum M_s * D_s (included by kernels.cu
// inside namespace bimp_b200, after the forward kernels).
//
//   k_pyr_down_f        float pyramid level (pyrDown without uint8 rounding)
//   k_pyr_down_f_adj    its transpose (scatter-add of the 5x5 taps)
//   k_masked_loss       sum M * D (the loss) and the w_tan / w_rad gradients
//   k_stencil_bwd       gather form of d L / d C over the stencil window from
//                       the ReLU states the forward stencil recorded (when
//                       fftW == dataW, window column dataW is the torus
//                       element (r+1, 0): its gradient is kept aside and
//                       added there by the tile backward)
//   k_gabor_tiles_bwd   per tile: the image spectrum X and, per orientation,
//                       z = e + i o recomputed as the forward computes them
//                       (nothing of the forward's responses is stored);
//                       a = dL/dC * z/|z|, A = FFT(a), alpha/rho dot products
//                       sum dG Re(conj(A) X), and the sum of A G in the
//                       frequency domain; one inverse transform per tile
//                       gives the window gradient, scattered to the level
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

// Over the forward stencil blocks (32 x kStencilBlockH pixels, the forward
// stencil's block list), a persistent grid: sum M * D into loss[0], and
// -sum M * T, -sum M * R (dL/dw_tan and dL/dw_rad: D = D0 - w_tan T -
// w_rad R) into gparams[2..3].  Each CTA accumulates its blocks in registers
// and adds once per quantity (a per-block atomic on the same three words
// serialises).
__global__ void __launch_bounds__(256) k_masked_loss(const ScaleDev* __restrict__ sds, const int2* __restrict__ work,
                                                     int nwork, double* __restrict__ loss,
                                                     double* __restrict__ gparams) {
  double acc = 0.0, accT = 0.0, accR = 0.0;
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const int2 item = work[w];
    const ScaleDev* sd = sds + item.x;
    const int W = sd->dataW, H = sd->dataH;
    const int nbx = (W + kStX - 1) / kStX;
    const int by = item.y / nbx, bx = item.y - by * nbx;
    const int x = bx * kStX + (threadIdx.x & 31);
    for (int i = threadIdx.x >> 5; i < kStencilBlockH; i += 8) {
      const int y = by * kStencilBlockH + i;
      if (x < W && y < H) {
        const double m = sd->M[(size_t)y * W + x];
        const size_t k = (size_t)y * sd->dPitch + x;
        acc += m * (double)sd->D[k];
        accT += m * (double)sd->T[k];
        accR += m * (double)sd->R[k];
      }
    }
  }
  block_add_double(acc, loss);
  block_add_double(-accT, gparams + 2);
  block_add_double(-accR, gparams + 3);
}

// --- stencil backward ------------------------------------------------------
constexpr int kBwQW = kStX + 2 * kHalo;        // 48: source pixels +-8 around the block
constexpr int kStBwThreads = 256;

// Gather form of dL/dC_o(p) for a 32x32 block of window positions p
// (0 <= p <= (dataH, dataW)): every source pixel q whose stencils read p
// contributes its loss weight M(q) times the ReLU state the forward recorded
// at q (ScaleDev::bits).  Sources lie within +-8 of p.  The tangential and
// radial weights are constants here; their own gradients come from
// k_masked_loss.
__global__ void __launch_bounds__(kStBwThreads)
k_stencil_bwd(const ScaleDev* __restrict__ sds, const int2* __restrict__ work) {
  __shared__ float sM[kBwQW * kBwQW];
  __shared__ unsigned int sBits[kBwQW * kBwQW];
  __shared__ int sOff[kNumOri][6];
  const int2 item = work[blockIdx.x];
  const ScaleDev* __restrict__ sd = sds + item.x;
  const int W = sd->dataW, H = sd->dataH;
  const int nbx = (W + 1 + kStX - 1) / kStX;
  const int by = item.y / nbx, bx = item.y - by * nbx;
  const int x0 = bx * kStX, y0 = by * kStY;
  const int t = threadIdx.x;
  const float gain = sd->radialGain, wT = sd->wTan, wR = sd->wRad;
  const int wrapW = sd->wrapW;
  if (t < kNumOri) {
    sOff[t][0] = sd->es1[t]; sOff[t][1] = sd->es2[t];
    sOff[t][2] = sd->in1[t]; sOff[t][3] = sd->in2[t];
    sOff[t][4] = sd->ih1[t]; sOff[t][5] = sd->ih2[t];
  }
  const int dp = sd->dPitch;
  for (int idx = t; idx < kBwQW * kBwQW; idx += kStBwThreads) {
    const int ly = idx / kBwQW, lx = idx - ly * kBwQW;
    const int gy = y0 - kHalo + ly, gx = x0 - kHalo + lx;
    const bool in = gy >= 0 && gy < H && gx >= 0 && gx < W;
    sM[idx] = in ? sd->M[(size_t)gy * W + gx] : 0.f;
    sBits[idx] = in ? sd->bits[(size_t)gy * dp + gx] : 0u;
  }
  __syncthreads();
  float* __restrict__ gC = sd->gC;
  const int cPitch = sd->cPitch;
  const long long cStride = sd->cStride;
  const int lx = t & 31;
  for (int ly = t >> 5; ly < kStY; ly += kStBwThreads / 32) {
    const int py = y0 + ly, px = x0 + lx;
    if (py > H + 1 || px > W) continue;           // row H + 1: read by no stencil, gathers 0
    const int qy = ly + kHalo, qx = lx + kHalo;   // p in source-pixel coordinates
    auto at = [&](int dy, int dx) { return (qy + dy) * kBwQW + (qx + dx); };
    const unsigned int b0 = sBits[at(0, 0)];
    const float m0 = sM[at(0, 0)];
#pragma unroll
    for (int o = 0; o < kNumOri; ++o) {
      const int op = (o + kNumOri / 2) % kNumOri;
      const int o1 = sOff[o][0], o2 = sOff[o][1], i1 = sOff[o][2], i2 = sOff[o][3];
      const int ph1 = sOff[op][4], ph2 = sOff[op][5];
      const unsigned int bd = 1u << (4 * o), bt = 2u << (4 * o), br = 4u << (4 * o), br1 = 8u << (4 * o);
      const unsigned int pr = 4u << (4 * op), pr1 = 8u << (4 * op);
      float g = 0.f;
      // double-stopped: p is the centre of q = p, and a -1/2 tap of q = p +- 2 offset
      if (b0 & bd) g += m0;
      {
        const int ka = at(2 * o1, -2 * o2), kb = at(-2 * o1, 2 * o2);
        if (sBits[ka] & bd) g -= 0.5f * sM[ka];
        if (sBits[kb] & bd) g -= 0.5f * sM[kb];
      }
      // tangential: p is read by q = p + i (as C(q - i)) and by q = p (centre)
      {
        const int kq = at(i1, i2);
        if (sBits[kq] & bt) g -= wT * sM[kq];
        if (b0 & bt) g += wT * m0;
      }
      // radial, o as the centre orientation (both terms when r1 > 0)
      if (b0 & br) g -= wR * m0 * ((b0 & br1) ? 2.f : 1.f);
      // radial, o as the perpendicular map of op: read at q + h (r1) and q - h (r)
      {
        const int k1 = at(-ph1, -ph2), k2 = at(ph1, ph2);
        const unsigned int b1 = sBits[k1], b2 = sBits[k2];
        if ((b1 & pr) && (b1 & pr1)) g += gain * wR * sM[k1];
        if (b2 & pr) g += gain * wR * sM[k2];
      }
      // fftW == dataW: window column dataW of row r is the torus element
      // (r + 1, 0); its gradient goes to gWrap[o][r], which the tile
      // backward adds at (r + 1, 0)
      if (wrapW && px == W) {
        if (py <= H) sd->gWrap[o * (H + 1) + py] = g;
        g = 0.f;
      }
      gC[(size_t)o * cStride + (size_t)py * cPitch + px] = g;
    }
  }
}

// --- tile backward -----------------------------------------------------------
// |e + i o| at or below kMagFloor counts as zero: no gradient flows through
// the magnitude there (the minimal-norm subgradient of |z| at 0).  Exactly
// flat image regions give |e + i o| = 0 up to rounding (the float taps'
// residual DC in FP64, FFT rounding of about 1e-6 of the map peak in FP32),
// where z / |z| is the direction of rounding noise.  The floor is an
// absolute value for images on the [0, 1] scale.
constexpr float kMagFloor = 3.0e-5f;
constexpr int kSmemBh = kSmemXh;   // Hermitian half of the accumulated spectrum

// Position of natural frequency k in the digit-permuted order of the 8x16
// transforms (the order of G and of the saved spectra).
__device__ __forceinline__ int perm128d(int k) { return 8 * (k & 15) + (k >> 4); }

// Persistent CTAs walk the tiles (one CTA per SM: 196 KB of shared memory
// and all 512 TMEM columns).  The window gradient is linear in the
// per-orientation spectra, Re IFFT(sum_o A_o G_o), so the products are summed
// in the frequency domain (Hermitian half, Bh) and ONE inverse transform per
// tile replaces one per orientation.  Nothing of the forward's responses is
// stored: per tile the image spectrum X is recomputed from the float level
// (the forward's transform: full spectrum into TMEM, Hermitian half into this
// CTA's slot of `xscratch`), and per orientation e + i o is recomputed on the
// valid outputs by the forward's inverse passes (G read from L2 instead of
// staged); then a = dL/dC * z/|z| (0 where |z| <= kMagFloor or outside the
// valid outputs), A = FFT(a), the alpha/rho dot products
// sum dG Re(conj(A) X), and Bh += (A G + conj(A G)(-k))/2.  The
// per-orientation coefficients G(+-k), dGa, dGr come pre-gathered in the
// half layout (ScaleDev::bwA, bwB).
constexpr int kGaborBwdSmem = kSmemW + kSmemBh + kSmemTw + kSmemMaps + 16;

// Prefetch (into L2, or into this SM's L1) of the block of dL/dC that the
// magnitude pass of one orientation reads: rows [R0, R0 + rows), columns
// [x0, x1) of a map with row pitch `pitch` floats (rows start on 128-byte
// lines).  One 128-byte line per thread and step; addresses stay inside the
// map.  The loads come after three transform passes, so the lines are in
// place by then instead of each load waiting on device memory.
template <bool L1>
__device__ __forceinline__ void prefetch_block(const float* base, int pitch, int R0, int rows, int x0, int x1, int t) {
  if (rows <= 0 || x1 <= x0) return;
  const int l0 = x0 >> 5, nl = ((x1 - 1) >> 5) - l0 + 1;   // 32 floats per line
  for (int i = t; i < rows * nl; i += kTileThreads) {
    const int r = i / nl, l = l0 + (i - r * nl);
    const float* a = base + (size_t)(R0 + r) * pitch + 32 * l;
    if constexpr (L1) asm volatile("prefetch.global.L1 [%0];" ::"l"(a));
    else asm volatile("prefetch.global.L2 [%0];" ::"l"(a));
  }
}
static_assert(kGaborBwdSmem <= 232448, "tile backward exceeds the 227 KB shared-memory limit");

__global__ void __launch_bounds__(kTileThreads, 1)
k_gabor_tiles_bwd(const ScaleDev* __restrict__ sds, const TileWork* __restrict__ work, int nwork,
                  float2* __restrict__ xscratch, double* __restrict__ gparams) {
  extern __shared__ float4 smem4b[];
  char* base = reinterpret_cast<char*>(smem4b);
  float2* W = reinterpret_cast<float2*>(base);
  float2* Bh = reinterpret_cast<float2*>(base + kSmemW);
  float2* tw = reinterpret_cast<float2*>(base + kSmemW + kSmemBh);
  short* rmap = reinterpret_cast<short*>(base + kSmemW + kSmemBh + kSmemTw);
  short* cmap = rmap + kTile;
  uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(base + kSmemW + kSmemBh + kSmemTw + kSmemMaps);
  float2* Xh64 = W + 64 * kTile;   // forward transform only
  float2* Nyq = Bh;                // forward transform only (Bh is cleared after it)
  float2* __restrict__ Xs = xscratch + (size_t)blockIdx.x * kSpecHalf;
  const int t = threadIdx.x;
  if (t < 8 * 17) {
    const int n1 = t / 17, k2 = t % 17;
    tw[t] = k2 < 16 ? c_w128[(n1 * k2) & 127] : make_float2(0.f, 0.f);
  }
  if ((t >> 5) == 0) tmem_alloc_warp(smem_u32(tmemSlot));
  tmem_fence_before();
  __syncthreads();
  tmem_fence_after();
  const uint32_t tlane = *tmemSlot + ((uint32_t)((t >> 5) & 3) << 21);
  // column p of the full spectrum in the Hermitian half (as the forward)
  const int pI1 = t & 127, h = t >> 7;
  const int pa = pI1 >> 3, pb = pI1 & 7;
  const bool pNyq = pb == 4 && pa == 0;
  const bool pConj = pb >= 4 && !pNyq;
  const int pSlot = pb < 4 ? 4 * pa + pb : (pNyq ? 64 : (pa > 0 ? 4 * (16 - pa) + (7 - pb) : 8 - pb));
  const float pSign = pConj ? -1.f : 1.f;
  const float2* pSrc = pNyq ? Nyq : Xh64 + pSlot;
  const int pStride = pNyq ? 1 : 64;
  double accA = 0.0, accR = 0.0;
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const TileWork item = work[w];
    const ScaleDev* sd = sds + item.entry;
    const int kX = sd->kX, V = sd->V;
    const int ty = item.tile / sd->tilesX, tx = item.tile - ty * sd->tilesX;
    const int R0 = ty * V, C0 = tx * V;
    __syncthreads();   // previous tile finished with every buffer
    tile_forward_spectrum<true>(sd, R0, C0, W, Xh64, Nyq, tw, rmap, cmap, t);
#pragma unroll 1
    for (int q = 0; q < 4; ++q) {
      const int k2 = h + 4 * q;
      float2 x[8];
#pragma unroll
      for (int k1 = 0; k1 < 8; ++k1) {
        const int row = pConj ? (k2 > 0 ? 8 * (16 - k2) + (7 - k1) : (8 - k1) & 7) : 8 * k2 + k1;
        x[k1] = pSrc[row * pStride];
        x[k1].y *= pSign;
      }
      tmem_store8(tlane + 16 * k2, x);
    }
    for (int j = t; j < kSpecHalf; j += kTileThreads) {
      const int r = j / kXhCols, sl = j - r * kXhCols;
      Xs[j] = *xh_ptr(Xh64, Nyq, r, sl);
    }
    tmem_fence_before();
    __syncthreads();   // the Hermitian half in W / Bh is dead from here
    tmem_fence_after();
    for (int j = t; j < kTile * kXhCols; j += kTileThreads) Bh[j] = make_float2(0.f, 0.f);
    const int cRows = sd->cRows, cCols = sd->cCols, cPitch = sd->cPitch;
    const long long cStride = sd->cStride;
    const int wrapW = sd->wrapW;
    // this tile's block of every dL/dC map: rows and columns of its valid
    // outputs inside the map
    const int pfRows = min(V, cRows - R0), pfX1 = min(C0 + V, cCols);
    for (int o = 0; o < kNumOri; ++o) {
      const float* __restrict__ Go = sd->G + (size_t)o * kSpecFloats;
      prefetch_block<false>(sd->gC + (size_t)o * cStride, cPitch, R0, pfRows, C0, pfX1, t);
      // I1: y-dim pass B' with the spectrum product X * G_o (TMEM in, TMEM out)
#pragma unroll 1
      for (int q = 0; q < 4; ++q) {
        const int k2 = h + 4 * q;
        float2 v[8];
        tmem_load8(tlane + 16 * k2, v);
        const float* __restrict__ Gq = Go + (size_t)(8 * k2) * kTile + pI1;
        float2 twr[8];   // read before the TMEM stores (compiler barriers for shared loads)
#pragma unroll
        for (int n1 = 1; n1 < 8; ++n1) twr[n1] = tw[n1 * 17 + k2];
#pragma unroll
        for (int k1 = 0; k1 < 8; ++k1) v[k1] = c_scale(v[k1], __ldg(Gq + k1 * kTile));
        dft8<true>(v);
#pragma unroll
        for (int n1 = 0; n1 < 8; ++n1)
          tmem_store1(tlane + kTmemY + 2 * (16 * n1 + k2), n1 ? c_mulc(v[n1], twr[n1]) : v[0]);
      }
      tmem_wait_st();
      tmem_fence_before();
      __syncthreads();   // the y-pass output is complete; no thread still reads W
      tmem_fence_after();
      // (I2 and I3 use TMEM and shared memory only: L1 keeps the block)
      prefetch_block<true>(sd->gC + (size_t)o * cStride, cPitch, R0, pfRows, C0, pfX1, t);
      // I2: y-dim pass A' -> natural y; rows outside the valid band are zero
      // (a is zero there, and the transform of a below reads every row)
#pragma unroll
      for (int it = 0; it < 2; ++it) {
        const int j = t + it * kTileThreads;
        const int p = j & 127, n1 = j >> 7;
        float2 v[16];
        tmem_load16(tlane + kTmemY + 32 * n1, v);
        dft16<true>(v);
#pragma unroll
        for (int n2 = 0; n2 < 16; ++n2) {
          const int y = n1 + 8 * n2;
          W[widx(y, p)] = (y >= kX && y < kX + V) ? v[n2] : make_float2(0.f, 0.f);
        }
      }
      tmem_fence_before();
      __syncthreads();
      tmem_fence_after();
      // I3: x-dim pass B' on the valid rows (a thread's k2 is fixed: its
      // twiddles are read once, not behind each store)
      {
        const int k2 = t & 15;
        float2 twr[8];
#pragma unroll
        for (int n1 = 1; n1 < 8; ++n1) twr[n1] = tw[n1 * 17 + k2];
        for (int j = t; j < V * 16; j += kTileThreads) {
          const int y = kX + (j >> 4);
          float2 v[8];
#pragma unroll
          for (int k1 = 0; k1 < 8; ++k1) v[k1] = W[widx(y, 8 * k2 + k1)];
          dft8<true>(v);
#pragma unroll
          for (int n1 = 0; n1 < 8; ++n1) W[widx(y, 8 * k2 + n1)] = n1 ? c_mulc(v[n1], twr[n1]) : v[0];
        }
      }
      __syncthreads();
      // I4 + the first pass of FFT(a): x-dim pass A' gives z = e + i o at the
      // row's outputs x = n1 + 8 n2; a = dL/dC * z/|z| on the valid outputs
      // (|z| as the forward computed it); then the forward x-dim pass A of a
      // on the same 16 elements, in registers
      for (int j = t; j < V * 8; j += kTileThreads) {
        const int y = kX + (j >> 3), n1 = j & 7;
        const int gy = R0 + y - kX;
        // dL/dC of the item's valid outputs, loaded before the transform so
        // that their latency overlaps it
        float gcv[16];
        {
          const float* __restrict__ grow = sd->gC + (size_t)o * cStride + (size_t)gy * cPitch;
#pragma unroll
          for (int n2 = 0; n2 < 16; ++n2) {
            const int x = n1 + 8 * n2, gx = C0 + x - kX;
            gcv[n2] = (x >= kX && x < kX + V && gy < cRows && gx < cCols) ? __ldg(grow + gx) : 0.f;
            if (wrapW && gx == 0 && gy >= 1 && gy < cRows) gcv[n2] += __ldg(sd->gWrap + o * (sd->dataH + 1) + gy - 1);
          }
        }
        float2 v[16];
#pragma unroll
        for (int k2 = 0; k2 < 16; ++k2) v[k2] = W[widx(y, 8 * k2 + n1)];
        dft16<true>(v);
#pragma unroll
        for (int n2 = 0; n2 < 16; ++n2) {
          const int x = n1 + 8 * n2;
          const int gx = C0 + x - kX;
          float2 a = make_float2(0.f, 0.f);
          if (x >= kX && x < kX + V && gy < cRows && gx < cCols) {
            const float gc = gcv[n2];
            // |z| as the forward computes it (s * rsqrt(s)); 1/|z| is the
            // same reciprocal square root, so a = gc z / |z| takes no division
            const float sq = fmaf(v[n2].x, v[n2].x, v[n2].y * v[n2].y);
            float rs;
            asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(rs) : "f"(fmaxf(sq, 1e-30f)));
            const float m = sq * rs;
            if (m > kMagFloor) {
              const float sc = gc * rs;
              a = make_float2(sc * v[n2].x, sc * v[n2].y);
            }
          }
          v[n2] = a;
        }
        dft16<false>(v);
        float2 twr[16];
#pragma unroll
        for (int k2 = 0; k2 < 16; ++k2) twr[k2] = tw[n1 * 17 + k2];
#pragma unroll
        for (int k2 = 0; k2 < 16; ++k2) W[widx(y, n1 + 8 * k2)] = c_mul(v[k2], twr[k2]);
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
        float2 twr[16];
#pragma unroll
        for (int k2 = 0; k2 < 16; ++k2) twr[k2] = tw[n1 * 17 + k2];
#pragma unroll
        for (int k2 = 0; k2 < 16; ++k2) W[widx(n1 + 8 * k2, p)] = c_mul(v[k2], twr[k2]);
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
      // Hermitian accumulation and the parameter dot products.  Entry j of
      // the half layout holds k = (ky, kx), kx in [0, 64]; its partner -k
      // covers the columns 65..127, so every frequency enters the dot
      // products once (columns 0 and 64 pair with themselves: their -k
      // coefficients are 0).  X is Hermitian, X(-k) = conj(X(k)).
      {
        const float4* __restrict__ cA = sd->bwA + (size_t)o * kSpecHalf;
        const float2* __restrict__ cB = sd->bwB + (size_t)o * kSpecHalf;
        float sa = 0.f, sr = 0.f;
        // entry (py, sl) of the half layout, j = py * kXhCols + sl
        auto entry = [&](int py, int sl, int p, int np, int wp) {
          const int j = py * kXhCols + sl;
          const float4 c4 = __ldg(cA + j);   // G(k), G(-k), dGa(k), dGr(k)
          const float2 c2 = __ldg(cB + j);   // dGa(-k), dGr(-k)
          const float2 X = Xs[j];   // written by this CTA for this tile: a coherent load
          const int ky = 16 * (py & 7) + (py >> 3);
          const int npy = perm128d((kTile - ky) & 127);
          const float2 A1 = W[wp], A2 = W[widx(npy, np)];
          const float2 bb = Bh[j];
          Bh[j] = make_float2(fmaf(0.5f * c4.x, A1.x, fmaf(0.5f * c4.y, A2.x, bb.x)),
                              fmaf(0.5f * c4.x, A1.y, fmaf(-0.5f * c4.y, A2.y, bb.y)));
          const float re1 = A1.x * X.x + A1.y * X.y;   // Re(conj(A(k)) X(k))
          const float re2 = A2.x * X.x - A2.y * X.y;   // Re(conj(A(-k)) conj(X(k)))
          sa = fmaf(c4.z, re1, fmaf(c2.x, re2, sa));
          sr = fmaf(c4.w, re1, fmaf(c2.y, re2, sr));
        };
        // slots 0..63: thread t owns slot sl = t mod 64 and the rows
        // py = t / 64 + 8 r (r = 0..15), so its column terms are fixed and
        // widx(py, p) = 128 py + (phys(p) ^ 8 (py & 1)) with py & 1 fixed
        // Four entries at a time: all their loads first, then the updates
        // (the entries' Bh words are distinct, but a store would otherwise
        // hold back the next entry's shared-memory loads).
        {
          const int sl = t & 63, pr = t >> 6;
          const int kx = (sl >> 2) + 16 * (sl & 3);
          const int p = perm128d(kx), np = perm128d((kTile - kx) & 127);
          const int pp = phys(p) ^ ((pr & 1) << 3);
#pragma unroll 1
          for (int r0 = 0; r0 < 16; r0 += 4) {
            float4 c4[4];
            float2 c2[4], X[4], A1[4], A2[4], bb[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              const int py = pr + 8 * (r0 + u);
              const int j = py * kXhCols + sl;
              c4[u] = __ldg(cA + j);
              c2[u] = __ldg(cB + j);
              X[u] = Xs[j];
              const int ky = 16 * (py & 7) + (py >> 3);
              A1[u] = W[py * kTile + pp];
              A2[u] = W[widx(perm128d((kTile - ky) & 127), np)];
              bb[u] = Bh[j];
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              const int j = (pr + 8 * (r0 + u)) * kXhCols + sl;
              Bh[j] = make_float2(fmaf(0.5f * c4[u].x, A1[u].x, fmaf(0.5f * c4[u].y, A2[u].x, bb[u].x)),
                                  fmaf(0.5f * c4[u].x, A1[u].y, fmaf(-0.5f * c4[u].y, A2[u].y, bb[u].y)));
              const float re1 = A1[u].x * X[u].x + A1[u].y * X[u].y;
              const float re2 = A2[u].x * X[u].x - A2[u].y * X[u].y;
              sa = fmaf(c4[u].z, re1, fmaf(c2[u].x, re2, sa));
              sr = fmaf(c4[u].w, re1, fmaf(c2[u].y, re2, sr));
            }
          }
        }
        // the Nyquist slot 64 (kx = 64): one row per thread of the first 128
        if (t < kTile) {
          const int p = perm128d(64);
          entry(t, 64, p, p, widx(t, p));
        }
        accA += sa;
        accR += sr;
      }
      // no barrier: every Bh entry has one owner thread, and the next
      // orientation's I1 touches only TMEM until its barrier
    }
    __syncthreads();
    // one inverse transform of the Hermitian sum: Re -> window gradient,
    // scattered to the float level through the padded-torus index maps.
    // Column p = t & 127 of the full spectrum is read from the half Bh
    // without a branch (conj(Bh(-k)) for kx > 64).
    const int pa = (t & 127) >> 3, pb = t & 7;
    const bool pNyq = pb == 4 && pa == 0;
    const bool pConj = pb >= 4 && !pNyq;
    const int pSlot = pb < 4 ? 4 * pa + pb : (pNyq ? 64 : (pa > 0 ? 4 * (16 - pa) + (7 - pb) : 8 - pb));
    const float pSign = pConj ? -1.f : 1.f;
#pragma unroll
    for (int it = 0; it < 4; ++it) {
      const int j = t + it * kTileThreads;
      const int p = j & 127, k2 = j >> 7;
      float2 v[8];
#pragma unroll
      for (int k1 = 0; k1 < 8; ++k1) {
        const int row = pConj ? (k2 > 0 ? 8 * (16 - k2) + (7 - k1) : (8 - k1) & 7) : 8 * k2 + k1;
        v[k1] = Bh[row * kXhCols + pSlot];
        v[k1].y *= pSign;
      }
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
    float* __restrict__ gl = sd->gLvl;
    const int gp = sd->lvlPitchF;
#pragma unroll
    for (int it = 0; it < 2; ++it) {
      const int j = t + it * kTileThreads;
      const int y = j >> 3, n1 = j & 7;
      float2 v[16];
#pragma unroll
      for (int k2 = 0; k2 < 16; ++k2) v[k2] = W[widx(y, 8 * k2 + n1)];
      dft16<true>(v);
      float* row = gl + (size_t)rmap[y] * gp;
#pragma unroll
      for (int n2 = 0; n2 < 16; ++n2) {
        const float g = v[n2].x;
        if (g != 0.f) atomicAdd(row + cmap[n1 + 8 * n2], kFloatLevelScale * g);
      }
    }
  }
  tmem_fence_before();
  __syncthreads();
  tmem_fence_after();
  if ((t >> 5) == 0) tmem_dealloc_warp(*tmemSlot);
  block_add_double(accA, gparams + 0);
  block_add_double(accR, gparams + 1);
}

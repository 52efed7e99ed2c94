// k_gabor_tiles: overlap-save 128x128 tile FFT Gabor filtering (included by
// kernels.cu).
//
// One CTA (512 threads, 16 warps) per tile.  The tile's real input window is
// read from the pyramid level through the reference's padded-torus index map,
// transformed once (forward 2D FFT, Hermitian half), and the full spectrum is
// written to tensor memory (TMEM): lane p holds column p, 32-bit columns
// 2 py and 2 py + 1 the real and imaginary parts of row py.  Thread t reads
// only lane t mod 128, which is the lane its warp may access, so the spectrum
// product pass of every orientation fetches its 8 values with one tcgen05.ld
// and no Hermitian lookup.  For each orientation of the work item (all 8,
// or a run of them where the plan splits a tile between CTAs, each of which
// then transforms the tile forward) the spectrum is
// multiplied by that orientation's real Gabor spectrum G_o, inverse
// transformed as one complex FFT (e + i o) and reduced to |e + i o| on the
// valid outputs.  SAVE_Z also stores e + i o (the line/edge detector's even
// and odd responses).
//
// G_o (64 KB per orientation, L2-resident) is streamed in 16 KB chunks with
// TMA bulk copies (cp.async.bulk + mbarrier) into a ring of 6 chunk slots:
// the four chunks of orientation o + 1 are issued as soon as orientation o's
// spectrum product pass is complete and land during its three remaining
// passes, so that pass needs no barrier of its own.  The product pass writes
// its y-pass output to TMEM as well (lane p = column p), where the second
// y-pass reads it back; the product pass therefore uses no shared memory,
// and warps that finish an orientation's last pass start the next
// orientation's product pass without waiting at a barrier.  Every mbarrier wait is
// bounded; on expiry the kernel records a fault in *fault, waits once more
// (bounded) for its copies and carries on, and the host reports the fault.
//
// Included inside namespace bimp_b200 by kernels.cu, after the helpers it uses
// (pad_src, pmod, c_w128).
#pragma once

constexpr int kGChunkRows = 32;                          // rows of G per chunk
constexpr int kGChunkFloats = kGChunkRows * kTile;       // 4096 floats = 16 KB
constexpr int kGSlots = 6;                               // G ring: 1.5 orientations
constexpr int kSmemW = kTile * kTile * 8;                // work buffer 128 x 128 complex
constexpr int kSmemXh = kTile * kXhCols * 8;             // Hermitian half spectrum (adjoint kernel)
constexpr int kSmemG = kGSlots * kGChunkFloats * 4;      // G chunk ring
constexpr int kSmemTw = 8 * 17 * 8;                      // twiddles w128^(n1*k2) (1 for n1 k2 = 0: not applied)
constexpr int kSmemMaps = 2 * kTile * 2;                 // int16 row / column maps
constexpr int kSmemBars = kGSlots * 8 + 8;               // ring mbarriers + the TMEM base address
constexpr int kGaborSmem = kSmemW + kSmemG + kSmemTw + kSmemMaps + kSmemBars;
static_assert(kGaborSmem <= 232448, "tile kernel exceeds the 227 KB shared-memory limit");
// During the forward transform the Hermitian half lives in rows 64..127 of
// the work buffer (slots 0..63, 64 complex per row) and in ring slot 4 (the
// Nyquist slot 64): orientation 0's chunks occupy slots 0..3 at that time.
constexpr int kNyqSlot = 4;
static_assert(kNyqSlot >= 4 && kNyqSlot < kGSlots, "Nyquist scratch must not hold orientation 0's chunks");

// Tensor memory, 128 lanes x 512 32-bit columns: the tile's full spectrum
// (columns [0, 256): lane p, columns 2 py, 2 py + 1 = X[py][p]) and the
// output of the first inverse y-pass (columns [256, 512): lane p, columns
// 256 + 2 (16 n1 + k2) + {0, 1} = row 8 k2 + n1 of column p).
constexpr uint32_t kTmemCols = 4 * kTile;
constexpr uint32_t kTmemY = 2 * kTile;

__device__ __forceinline__ void tmem_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Whole warp: allocate kTmemCols columns, base address written to dst_smem.
__device__ __forceinline__ void tmem_alloc_warp(uint32_t dst_smem) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem),
               "n"(kTmemCols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc_warp(uint32_t taddr) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "n"(kTmemCols) : "memory");
}
// Whole warp: each thread stores 8 complex (16 columns from taddr's column)
// into its own lane and waits for the store to complete.
__device__ __forceinline__ void tmem_store8(uint32_t taddr, const float2 (&v)[8]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16};\n"
      "tcgen05.wait::st.sync.aligned;" ::"r"(taddr),
      "r"(__float_as_uint(v[0].x)), "r"(__float_as_uint(v[0].y)), "r"(__float_as_uint(v[1].x)),
      "r"(__float_as_uint(v[1].y)), "r"(__float_as_uint(v[2].x)), "r"(__float_as_uint(v[2].y)),
      "r"(__float_as_uint(v[3].x)), "r"(__float_as_uint(v[3].y)), "r"(__float_as_uint(v[4].x)),
      "r"(__float_as_uint(v[4].y)), "r"(__float_as_uint(v[5].x)), "r"(__float_as_uint(v[5].y)),
      "r"(__float_as_uint(v[6].x)), "r"(__float_as_uint(v[6].y)), "r"(__float_as_uint(v[7].x)),
      "r"(__float_as_uint(v[7].y))
      : "memory");
}
// Whole warp: each thread stores one complex (2 columns) into its own lane;
// completion is awaited with tmem_wait_st.
__device__ __forceinline__ void tmem_store1(uint32_t taddr, float2 v) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};" ::"r"(taddr), "r"(__float_as_uint(v.x)),
               "r"(__float_as_uint(v.y))
               : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
// Whole warp: each thread loads 16 complex (32 columns) from its own lane;
// the values are complete when the statement returns.
__device__ __forceinline__ void tmem_load16(uint32_t taddr, float2 (&v)[16]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = make_float2(__uint_as_float(r[2 * i]), __uint_as_float(r[2 * i + 1]));
}
// Whole warp: each thread loads 8 complex from its own lane; the values are
// complete when the statement returns.
__device__ __forceinline__ void tmem_load8(uint32_t taddr, float2 (&v)[8]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = make_float2(__uint_as_float(r[2 * i]), __uint_as_float(r[2 * i + 1]));
}

// |z| as s * rsqrt(max(s, 1e-30)), s = |z|^2 (hardware reciprocal square
// root, relative error a few 1e-7): exactly 0 for z = 0, and below 1e-15
// (where the max applies) the value stays below |z|.
__device__ __forceinline__ float cmag(float2 z) {
  const float s = fmaf(z.x, z.x, z.y * z.y);
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(fmaxf(s, 1e-30f)));
  return s * r;
}

// Float levels hold X (a float image, X = u8/255 for the uint8 content);
// the uint8 path's value 255*u8/65536 is then (255*255/65536) * X.
constexpr float kFloatLevelScale = 65025.0f / 65536.0f;

// Work-buffer index of row y, position p: the rotate-by-(p>>4) swizzle inside
// each group of 8 keeps the stride-8 and contiguous-8 passes conflict-free,
// and odd rows swap the two halves of every 16-group so that two rows served
// by one wavefront use disjoint banks.
__device__ __forceinline__ int widx(int y, int p) { return y * kTile + (phys(p) ^ ((y & 1) << 3)); }

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// 1-D TMA bulk copy global -> shared, completion counted on `bar`.
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
// Bounded wait for phase `parity` of `bar`; false if it did not complete.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (int i = 0; i < (1 << 22); ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Mean-removed pixel value of level row r, column c.  uint8: the
// reference's 255*u8/65536 (convertTo, cuda_bimp.cu:481) minus 0.5, exactly,
// as (255*u8 - 32768)/65536.  float: kFloatLevelScale * X - 0.5.
template <bool FLT>
__device__ __forceinline__ float level_value(const ScaleDev* sd, int r, int c) {
  if constexpr (FLT) {
    return kFloatLevelScale * sd->lvlF[(size_t)r * sd->lvlPitchF + c] - 0.5f;
  } else {
    // 12582912 + (255 u8 - 32768) as the bits of a float (1.5 * 2^23 plus an
    // integer of magnitude below 2^15 is exact), then x / 65536 exactly:
    // the same value as the integer converted and scaled, without the
    // conversion unit
    const int b = 0x4B400000 - 32768 + 255 * (int)sd->lvl[(size_t)r * sd->lvlPitch + c];
    return fmaf(__int_as_float(b), 1.0f / 65536.0f, -192.0f);
  }
}

// Element (row, slot) of the Hermitian half during the forward transform:
// slots 0..63 at Xh64[row * 64 + slot], the Nyquist slot 64 at Nyq[row].
__device__ __forceinline__ float2* xh_ptr(float2* Xh64, float2* Nyq, int row, int slot) {
  return slot < 64 ? Xh64 + row * 64 + slot : Nyq + row;
}

// Index maps of the tile's input window and its forward 2D FFT.
// rmap/cmap: window row/col -> level row/col through the padded torus.
// On return the Hermitian half X[py][slot] (py = permuted ky, slot = kx
// 0..64), including the DC of the removed 0.5 offset, is in Xh64 / Nyq
// (see xh_ptr).  Uses the first 64 rows of W as scratch.  Ends with a
// barrier.
template <bool FLT>
__device__ __forceinline__ void tile_forward_spectrum(const ScaleDev* sd, int R0, int C0, float2* W, float2* Xh64,
                                                      float2* Nyq, const float2* tw, short* rmap, short* cmap,
                                                      int t) {
  const int kX = sd->kX;
  if (t < kTile) {
    rmap[t] = (short)pad_src(pmod(R0 - kX + t, sd->fftH), sd->dataH, kX);
  } else if (t < 2 * kTile) {
    const int i = t - kTile;
    cmap[i] = (short)pad_src(pmod(C0 - kX + i, sd->fftW), sd->dataW, kX);
  }
  __syncthreads();
  // F1: x-dim pass A on packed rows z[r] = in[r] + i in[r+64], r < 64.
  // Removing the mean keeps the butterflies' intermediate magnitudes, and so
  // their float rounding, small; the 0.5 offset goes back into the DC bin.
  {
    const int r = t >> 3, n1 = t & 7;
    const int ra = rmap[r], rb = rmap[r + 64];
    float2 v[16];
#pragma unroll
    for (int m = 0; m < 16; ++m) {
      const int c = cmap[n1 + 8 * m];
      v[m] = make_float2(level_value<FLT>(sd, ra, c), level_value<FLT>(sd, rb, c));
    }
    dft16<false>(v);
    // twiddles into registers before the stores (loads of the table would
    // otherwise wait behind each store to the same shared memory)
    float2 twr[16];
#pragma unroll
    for (int k2 = 1; k2 < 16; ++k2) twr[k2] = tw[n1 * 17 + k2];
#pragma unroll
    for (int k2 = 0; k2 < 16; ++k2) W[widx(r, n1 + 8 * k2)] = k2 ? c_mul(v[k2], twr[k2]) : v[0];
  }
  __syncthreads();
  // F2: x-dim pass B
#pragma unroll
  for (int it = 0; it < 2; ++it) {
    const int j = t + it * kTileThreads;
    const int r = j >> 4, k2 = j & 15;
    float2 v[8];
#pragma unroll
    for (int n1 = 0; n1 < 8; ++n1) v[n1] = W[widx(r, 8 * k2 + n1)];
    dft8<false>(v);
#pragma unroll
    for (int k1 = 0; k1 < 8; ++k1) W[widx(r, 8 * k2 + k1)] = v[k1];
  }
  __syncthreads();
  // F3: y-dim pass A on the 65 half columns (kx = 0..64), reading the packed
  // rows and separating them on the way in: packed row r (< 64) holds
  // in[r] + i in[r + 64], so X[r][kx] = (Z[kx] + conj Z[-kx]) / 2 and
  // X[r + 64][kx] = (Z[kx] - conj Z[-kx]) / 2i.  The packed rows (rows 0..63
  // of W) and the half spectrum (rows 64..127 of W, and the Nyquist slot)
  // do not overlap.
  for (int j = t; j < 8 * kXhCols; j += kTileThreads) {
    const int n1 = j / kXhCols, s = j - n1 * kXhCols;
    const int kx = s < 64 ? (s >> 2) + 16 * (s & 3) : 64;
    const int nk = (128 - kx) & 127;
    const int pk = 8 * (kx & 15) + (kx >> 4), pn = 8 * (nk & 15) + (nk >> 4);
    float2 v[16];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int r = n1 + 8 * m;
      const float2 Z = W[widx(r, pk)], Zn = W[widx(r, pn)];
      v[m] = make_float2(0.5f * (Z.x + Zn.x), 0.5f * (Z.y - Zn.y));
      v[m + 8] = make_float2(0.5f * (Z.y + Zn.y), 0.5f * (Zn.x - Z.x));
    }
    dft16<false>(v);
    float2* col = xh_ptr(Xh64, Nyq, 0, s);
    const int st = s < 64 ? 64 : 1;
    float2 twr[16];
#pragma unroll
    for (int k2 = 1; k2 < 16; ++k2) twr[k2] = tw[n1 * 17 + k2];
#pragma unroll
    for (int k2 = 0; k2 < 16; ++k2) col[(n1 + 8 * k2) * st] = k2 ? c_mul(v[k2], twr[k2]) : v[0];
  }
  __syncthreads();
  // F4: y-dim pass B -> rows in permuted ky order
  for (int j = t; j < 16 * kXhCols; j += kTileThreads) {
    const int k2 = j / kXhCols, s = j - k2 * kXhCols;
    float2* col = xh_ptr(Xh64, Nyq, 0, s);
    const int st = s < 64 ? 64 : 1;
    float2 v[8];
#pragma unroll
    for (int n1 = 0; n1 < 8; ++n1) v[n1] = col[(8 * k2 + n1) * st];
    dft8<false>(v);
    if (j == 0) v[0].x += 0.5f * (float)(kTile * kTile);   // DC of the removed 0.5 offset
#pragma unroll
    for (int k1 = 0; k1 < 8; ++k1) col[(8 * k2 + k1) * st] = v[k1];
  }
  __syncthreads();
}

template <bool FLT, bool SAVE_Z>
__global__ void __launch_bounds__(kTileThreads, 1)
k_gabor_tiles(const ScaleDev* __restrict__ sds, const TileWork* __restrict__ work, int nwork,
              unsigned int* __restrict__ fault_word) {
  extern __shared__ float4 smem4[];
  char* base = reinterpret_cast<char*>(smem4);
  float2* W = reinterpret_cast<float2*>(base);
  float* Gbuf = reinterpret_cast<float*>(base + kSmemW);
  float2* tw = reinterpret_cast<float2*>(base + kSmemW + kSmemG);
  short* rmap = reinterpret_cast<short*>(base + kSmemW + kSmemG + kSmemTw);
  short* cmap = rmap + kTile;
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + kSmemW + kSmemG + kSmemTw + kSmemMaps);
  uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(bars + kGSlots);
  float2* Xh64 = W + 64 * kTile;                                             // forward transform only
  float2* Nyq = reinterpret_cast<float2*>(Gbuf + kNyqSlot * kGChunkFloats);  // forward transform only
  const uint32_t bar0 = smem_u32(&bars[0]), gdst0 = smem_u32(Gbuf);
  const int t = threadIdx.x;

  if (t < 8 * 17) {
    const int n1 = t / 17, k2 = t % 17;
    tw[t] = k2 < 16 ? c_w128[(n1 * k2) & 127] : make_float2(0.f, 0.f);
  }
  if (t == 0) {
    for (int i = 0; i < kGSlots; ++i) mbar_init(bar0 + 8 * i);
    fence_mbar_init();
  }
  if ((t >> 5) == 0) tmem_alloc_warp(smem_u32(tmemSlot));
  griddep_launch_dependents();
  tmem_fence_before();
  __syncthreads();
  tmem_fence_after();
  griddep_wait();   // the pyramid levels come from the previous kernel
  // this thread's lane (t mod 128) of the spectrum; (warp mod 4) * 32 is the
  // lane block the warp may access
  const uint32_t tlane = *tmemSlot + ((uint32_t)((t >> 5) & 3) << 21);

  uint32_t ph = 0;       // per ring slot: parity of its next fill (identical in every thread)
  bool fault = false;
  // Where this thread's column p of the full spectrum lives in the
  // Hermitian half (the same for every tile): the half holds kx = 0..64; the
  // other columns are conj(X(-k)), read from row -ky.
  const int pI1 = t & 127, h = t >> 7;
  const int pa = pI1 >> 3, pb = pI1 & 7;
  const bool pNyq = pb == 4 && pa == 0;
  const bool pConj = pb >= 4 && !pNyq;
  const int pSlot = pb < 4 ? 4 * pa + pb : (pNyq ? 64 : (pa > 0 ? 4 * (16 - pa) + (7 - pb) : 8 - pb));
  const float pSign = pConj ? -1.f : 1.f;
  const float2* pSrc = pNyq ? Nyq : Xh64 + pSlot;
  const int pStride = pNyq ? 1 : 64;

  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const TileWork item = work[w];
    const int oB = item.oBegin, oE = item.oEnd;
    if (oB >= oE) continue;   // empty slot of a padded plan (the same item in every thread)
    const ScaleDev* sd = sds + item.entry;
    const int kX = sd->kX, V = sd->V;
    const int ty = item.tile / sd->tilesX, tx = item.tile - ty * sd->tilesX;
    const int R0 = ty * V, C0 = tx * V;
    const float* __restrict__ G0 = sd->G;

    __syncthreads();   // previous tile finished with every buffer
    if (t == 0) {      // orientation oB's four chunks into slots 0..3
      fence_proxy_async();
      for (int c = 0; c < 4; ++c)
        bulk_load(gdst0 + c * kGChunkFloats * 4, G0 + (size_t)(4 * oB + c) * kGChunkFloats, kGChunkFloats * 4,
                  bar0 + 8 * c);
    }
    tile_forward_spectrum<FLT>(sd, R0, C0, W, Xh64, Nyq, tw, rmap, cmap, t);
    // full spectrum into TMEM: this thread writes the rows py = 8 k2 + k1,
    // k2 = h + 4 q, that it reads in every orientation's product pass
#pragma unroll 1
    for (int q = 0; q < 4; ++q) {
      const int k2 = h + 4 * q;
      float2 x[8];
#pragma unroll
      for (int k1 = 0; k1 < 8; ++k1) {
        // row of -ky in the permuted order (ky = 16 k1 + k2 for py = 8 k2 + k1)
        const int row = pConj ? (k2 > 0 ? 8 * (16 - k2) + (7 - k1) : (8 - k1) & 7) : 8 * k2 + k1;
        x[k1] = pSrc[row * pStride];
        x[k1].y *= pSign;
      }
      tmem_store8(tlane + 16 * k2, x);
    }
    tmem_fence_before();
    __syncthreads();   // the Hermitian half in W / slot 4 is dead from here
    tmem_fence_after();

    const int cRows = sd->cRows, cCols = sd->cCols, cPitch = sd->cPitch;
    // tiles holding window column 0 or column dataW of a map with fftW == dataW
    const bool wrapTile = sd->wrapW != 0 && (C0 == 0 || C0 + V >= cCols);
    // window positions x in [kX, xHi) are this tile's valid outputs; only
    // its first Vr valid rows lie inside the map, and the x-passes run on
    // those alone (a tile of the last tile row may hold only a few)
    const int xHi = min(kX + V, cCols - C0 + kX);
    const int Vr = min(V, cRows - R0);
    // I4's thread keeps column group n1 = t mod 8 for the whole tile: bit n2
    // of xMask says whether its output x = n1 + 8 n2 is in [kX, xHi)
    unsigned int xMask = 0;
#pragma unroll
    for (int n2 = 0; n2 < 16; ++n2) {
      const int x = (t & 7) + 8 * n2;
      xMask |= (x >= kX && x < xHi ? 1u : 0u) << n2;
    }
    float* __restrict__ C0p = sd->C;
    float2* __restrict__ Z0p = sd->Z;
    const long long cStride = sd->cStride;
    for (int o = oB; o < oE; ++o) {
      float* __restrict__ Cout = C0p + (size_t)o * cStride;
      const int r = o - oB;   // position in the item: chunk 4 r + q of the item sits in ring slot (4 r + q) mod 6
      // I1: y-dim pass B' with the spectrum product Z = X * G; quarter q
      // uses chunk 4 o + q of G (rows py in [32 q, 32 q + 32))
#pragma unroll 1
      for (int q = 0; q < 4; ++q) {
        const int k2 = h + 4 * q;
        const int slot = (4 * r + q) % kGSlots;
        float2 v[8];
        tmem_load8(tlane + 16 * k2, v);
        if (!mbar_wait(bar0 + 8 * slot, (ph >> slot) & 1)) fault = true;
        ph ^= 1u << slot;
        __syncwarp();   // the warp-collective TMEM stores below need a converged warp
        const float* Gq = Gbuf + slot * kGChunkFloats + 8 * h * kTile + pI1;
        // this quarter's twiddles, read before the TMEM stores (each store
        // is a compiler barrier for shared-memory loads)
        float2 twr[8];
#pragma unroll
        for (int n1 = 1; n1 < 8; ++n1) twr[n1] = tw[n1 * 17 + k2];
#pragma unroll
        for (int k1 = 0; k1 < 8; ++k1) v[k1] = c_scale(v[k1], Gq[k1 * kTile]);
        dft8<true>(v);
#pragma unroll
        for (int n1 = 0; n1 < 8; ++n1)
          tmem_store1(tlane + kTmemY + 2 * (16 * n1 + k2), n1 ? c_mulc(v[n1], twr[n1]) : v[0]);
      }
      tmem_wait_st();
      tmem_fence_before();
      // the y-pass output is complete, every slot of orientation o is
      // consumed, and (previous orientation) no thread still reads W
      __syncthreads();
      tmem_fence_after();
      if (t == 0 && o + 1 < oE) {   // orientation o + 1's chunks land during I2..I4
        fence_proxy_async();
        for (int j = 0; j < 4; ++j) {
          const int c = 4 * (o + 1) + j, sl = (4 * (r + 1) + j) % kGSlots;
          bulk_load(gdst0 + sl * kGChunkFloats * 4, G0 + (size_t)c * kGChunkFloats, kGChunkFloats * 4, bar0 + 8 * sl);
        }
      }
      // I2: y-dim pass A' -> natural y (all 128 rows: storing only the
      // valid rows, under a predicate per store, measured 11% slower)
#pragma unroll
      for (int it = 0; it < 2; ++it) {
        const int j = t + it * kTileThreads;
        const int p = j & 127, n1 = j >> 7;   // p = this thread's lane
        float2 v[16];
        tmem_load16(tlane + kTmemY + 32 * n1, v);
        dft16<true>(v);
#pragma unroll
        for (int n2 = 0; n2 < 16; ++n2) W[widx(n1 + 8 * n2, p)] = v[n2];
      }
      tmem_fence_before();
      __syncthreads();   // W holds the y-transformed tile; the TMEM y-pass area is free
      tmem_fence_after();
      // I3: x-dim pass B' on the rows holding valid outputs; a thread's k2
      // (= t mod 16) is the same in every item, so its twiddles are loaded once
      {
        const int k2 = t & 15;
        float2 twr[8];
#pragma unroll
        for (int n1 = 1; n1 < 8; ++n1) twr[n1] = tw[n1 * 17 + k2];
        for (int j = t; j < Vr * 16; j += kTileThreads) {
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
      // I4: x-dim pass A' -> natural x; complex magnitude of valid outputs
      for (int j = t; j < Vr * 8; j += kTileThreads) {
        const int y = kX + (j >> 3), n1 = j & 7;
        float2 v[16];
#pragma unroll
        for (int k2 = 0; k2 < 16; ++k2) v[k2] = W[widx(y, 8 * k2 + n1)];
        dft16<true>(v);
        const int gy = R0 + y - kX;
        if (gy < cRows) {
          float* dst = Cout + (size_t)gy * cPitch;
          if (!wrapTile) {
            float* dstx = dst + (C0 - kX);
#pragma unroll
            for (int n2 = 0; n2 < 16; ++n2) {
              const int x = n1 + 8 * n2;
              if ((xMask >> n2) & 1u) {
                dstx[x] = cmag(v[n2]);
                if constexpr (SAVE_Z) Z0p[(size_t)o * cStride + (size_t)gy * cPitch + (C0 - kX) + x] = v[n2];
              }
            }
          } else {
            // fftW == dataW: the stencils read window column dataW of row r
            // at the flat address r*fftW + fftW, the torus element (r + 1, 0),
            // so that element also goes to (r, dataW); the window's own
            // (r, dataW) output is kept only on the last row
#pragma unroll
            for (int n2 = 0; n2 < 16; ++n2) {
              const int x = n1 + 8 * n2;
              const int gx = C0 + x - kX;
              if (x >= kX && x < kX + V && gx < cCols) {
                const float m = cmag(v[n2]);
                if (!(gx == cCols - 1 && gy < cRows - 1)) {
                  dst[gx] = m;
                  if constexpr (SAVE_Z) Z0p[(size_t)o * cStride + (size_t)gy * cPitch + gx] = v[n2];
                }
                if (gx == 0 && gy >= 1) {
                  Cout[(size_t)(gy - 1) * cPitch + cCols - 1] = m;
                  if constexpr (SAVE_Z) Z0p[(size_t)o * cStride + (size_t)(gy - 1) * cPitch + cCols - 1] = v[n2];
                }
              }
            }
          }
        }
      }
      // no barrier here: the next orientation's I1 touches only TMEM and the
      // G ring, so warps done with I4 start it while the others finish
    }
  }
  if (fault) {
    // a wait expired: record it, then give the copies still in flight a
    // second bounded chance to land before the CTA releases its memory
    if (t == 0) atomicOr(fault_word, 1u);
    for (int i = 0; i < kGSlots; ++i) mbar_wait(bar0 + 8 * i, ((ph >> i) & 1) ^ 1);
  }
  tmem_fence_before();
  __syncthreads();
  tmem_fence_after();
  if ((t >> 5) == 0) tmem_dealloc_warp(*tmemSlot);
}

// ---------------------------------------------------------------------------
// k_gabor_tiles_ws: the same tile computation with warp-specialised,
// pipelined orientations
// ---------------------------------------------------------------------------
// After the tile's forward transform (all 16 warps, as above), warps 0-7
// (group Y) run the spectrum product and the two inverse y-passes of each
// orientation (TMEM in, TMEM y-area, then the valid rows into a shared-memory
// row buffer), while warps 8-15 (group X) run the two inverse x-passes and
// the complex magnitude of the previous orientation from the other buffer.
// Two row buffers of kWsRows x 128 complex alternate between orientations;
// named barriers hand them over (full: Y -> X, empty: X -> Y), and each group
// orders its own passes with a 256-thread named barrier, so no CTA-wide
// barrier stands inside the orientation loop.  G_o is read from L2 (the
// space of the TMA ring holds the second buffer).  Needs V <= kWsRows.
constexpr int kWsRows = 104;                                  // largest V this kernel takes
constexpr int kWsBuf = kWsRows * kTile;                       // complex per row buffer
constexpr int kWsSmemW = 2 * kWsBuf * 8;                      // both row buffers (also the forward scratch)
constexpr int kWsSmem = kWsSmemW + kSmemTw + kSmemMaps + 16;  // + twiddles, index maps, TMEM base slot
static_assert(kWsSmem <= 232448, "warp-specialised tile kernel exceeds the 227 KB shared-memory limit");
// forward transform scratch inside the two buffers: packed rows 0..63, the
// Hermitian half at rows 64..127, the Nyquist slot column at row 192
static_assert(2 * kWsRows >= 193, "forward-transform scratch does not fit the row buffers");
constexpr int kWsGroup = kTileThreads / 2;   // threads per group
enum : int { kBarY = 1, kBarX = 2, kBarFull0 = 3, kBarEmpty0 = 5 };   // named barrier ids (0 is __syncthreads)

__device__ __forceinline__ void nbar_sync(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }
__device__ __forceinline__ void nbar_arrive(int id, int n) {
  asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(n) : "memory");
}

template <bool FLT>
__global__ void __launch_bounds__(kTileThreads, 1)
k_gabor_tiles_ws(const ScaleDev* __restrict__ sds, const TileWork* __restrict__ work, int nwork) {
  extern __shared__ float4 smem4[];
  char* base = reinterpret_cast<char*>(smem4);
  float2* Wb = reinterpret_cast<float2*>(base);
  float2* tw = reinterpret_cast<float2*>(base + kWsSmemW);
  short* rmap = reinterpret_cast<short*>(base + kWsSmemW + kSmemTw);
  short* cmap = rmap + kTile;
  uint32_t* tmemSlot = reinterpret_cast<uint32_t*>(base + kWsSmemW + kSmemTw + kSmemMaps);
  float2* Xh64 = Wb + 64 * kTile;    // forward transform only
  float2* Nyq = Wb + 192 * kTile;    // forward transform only
  const int t = threadIdx.x;
  if (t < 8 * 17) {
    const int n1 = t / 17, k2 = t % 17;
    tw[t] = k2 < 16 ? c_w128[(n1 * k2) & 127] : make_float2(0.f, 0.f);
  }
  if ((t >> 5) == 0) tmem_alloc_warp(smem_u32(tmemSlot));
  griddep_launch_dependents();
  tmem_fence_before();
  __syncthreads();
  tmem_fence_after();
  griddep_wait();   // the pyramid levels come from the previous kernel
  const uint32_t tlane = *tmemSlot + ((uint32_t)((t >> 5) & 3) << 21);
  // spectrum store (all warps): column p of the full spectrum in the half
  const int pI1 = t & 127, h4 = t >> 7;
  const int pa = pI1 >> 3, pb = pI1 & 7;
  const bool pNyq = pb == 4 && pa == 0;
  const bool pConj = pb >= 4 && !pNyq;
  const int pSlot = pb < 4 ? 4 * pa + pb : (pNyq ? 64 : (pa > 0 ? 4 * (16 - pa) + (7 - pb) : 8 - pb));
  const float pSign = pConj ? -1.f : 1.f;
  const float2* pSrc = pNyq ? Nyq : Xh64 + pSlot;
  const int pStride = pNyq ? 1 : 64;
  const bool groupY = t < kWsGroup;
  const int tg = t & (kWsGroup - 1);   // index within the group
  const int hY = tg >> 7;              // group Y: spectrum rows k2 = hY + 2 q

  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const TileWork item = work[w];
    const int oB = item.oBegin, oE = item.oEnd, nO = oE - oB;
    if (nO <= 0) continue;   // empty slot of a padded plan
    const ScaleDev* sd = sds + item.entry;
    const int kX = sd->kX, V = sd->V;
    const int ty = item.tile / sd->tilesX, tx = item.tile - ty * sd->tilesX;
    const int R0 = ty * V, C0 = tx * V;
    __syncthreads();   // previous tile finished with every buffer
    tile_forward_spectrum<FLT>(sd, R0, C0, Wb, Xh64, Nyq, tw, rmap, cmap, t);
#pragma unroll 1
    for (int q = 0; q < 4; ++q) {
      const int k2 = h4 + 4 * q;
      float2 x[8];
#pragma unroll
      for (int k1 = 0; k1 < 8; ++k1) {
        const int row = pConj ? (k2 > 0 ? 8 * (16 - k2) + (7 - k1) : (8 - k1) & 7) : 8 * k2 + k1;
        x[k1] = pSrc[row * pStride];
        x[k1].y *= pSign;
      }
      tmem_store8(tlane + 16 * k2, x);
    }
    tmem_fence_before();
    __syncthreads();   // spectrum in TMEM; the forward scratch in the row buffers is dead
    tmem_fence_after();
    if (groupY) {
      for (int o = oB; o < oE; ++o) {
        const int b = (o - oB) & 1;
        float2* Wo = Wb + b * kWsBuf;
        const float* __restrict__ Go = sd->G + (size_t)o * kSpecFloats;
        // I1: y-dim pass B' with the spectrum product (TMEM in, TMEM y-area
        // out); each quarter's G values are loaded one quarter ahead
        float g[8];
#pragma unroll
        for (int k1 = 0; k1 < 8; ++k1) g[k1] = __ldg(Go + (size_t)(8 * hY + k1) * kTile + pI1);
#pragma unroll 1
        for (int q = 0; q < 8; ++q) {
          const int k2 = hY + 2 * q;
          float2 v[8];
          float gn[8];
          const int k2n = q < 7 ? k2 + 2 : k2;
#pragma unroll
          for (int k1 = 0; k1 < 8; ++k1) gn[k1] = __ldg(Go + (size_t)(8 * k2n + k1) * kTile + pI1);
          tmem_load8(tlane + 16 * k2, v);
          float2 twr[8];
#pragma unroll
          for (int n1 = 1; n1 < 8; ++n1) twr[n1] = tw[n1 * 17 + k2];
#pragma unroll
          for (int k1 = 0; k1 < 8; ++k1) v[k1] = c_scale(v[k1], g[k1]);
          dft8<true>(v);
#pragma unroll
          for (int n1 = 0; n1 < 8; ++n1)
            tmem_store1(tlane + kTmemY + 2 * (16 * n1 + k2), n1 ? c_mulc(v[n1], twr[n1]) : v[0]);
#pragma unroll
          for (int k1 = 0; k1 < 8; ++k1) g[k1] = gn[k1];
        }
        tmem_wait_st();
        tmem_fence_before();
        nbar_sync(kBarY, kWsGroup);   // the y-area holds orientation o's first y-pass
        tmem_fence_after();
        if (o - oB >= 2) nbar_sync(kBarEmpty0 + b, kTileThreads);   // group X is done with orientation o - 2
        // I2: y-dim pass A' -> natural y; the valid rows into buffer b
#pragma unroll
        for (int it = 0; it < 4; ++it) {
          const int j = tg + it * kWsGroup;
          const int p = j & 127, n1 = j >> 7;
          float2 v[16];
          tmem_load16(tlane + kTmemY + 32 * n1, v);
          dft16<true>(v);
#pragma unroll
          for (int n2 = 0; n2 < 16; ++n2) {
            const int y = n1 + 8 * n2 - kX;
            if (y >= 0 && y < V) Wo[widx(y, p)] = v[n2];
          }
        }
        tmem_fence_before();
        nbar_arrive(kBarFull0 + b, kTileThreads);   // buffer b holds orientation o
        nbar_sync(kBarY, kWsGroup);                 // every thread is done reading the y-area
        tmem_fence_after();
      }
    } else {
      const int cRows = sd->cRows, cCols = sd->cCols, cPitch = sd->cPitch;
      const bool wrapTile = sd->wrapW != 0 && (C0 == 0 || C0 + V >= cCols);
      const int xHi = min(kX + V, cCols - C0 + kX);
      const int Vr = min(V, cRows - R0);   // valid rows inside the map
      // I4 keeps column group n1 = tg mod 8 for the whole tile
      unsigned int xMask = 0;
#pragma unroll
      for (int n2 = 0; n2 < 16; ++n2) {
        const int x = (tg & 7) + 8 * n2;
        xMask |= (x >= kX && x < xHi ? 1u : 0u) << n2;
      }
      float* __restrict__ C0p = sd->C;
      const long long cStride = sd->cStride;
      for (int o = oB; o < oE; ++o) {
        const int b = (o - oB) & 1;
        float2* Wo = Wb + b * kWsBuf;
        float* __restrict__ Cout = C0p + (size_t)o * cStride;
        nbar_sync(kBarFull0 + b, kTileThreads);
        // I3: x-dim pass B' on the V rows of the buffer (a thread's k2 is
        // fixed: its twiddles are loaded once)
        {
          const int k2 = tg & 15;
          float2 twr[8];
#pragma unroll
          for (int n1 = 1; n1 < 8; ++n1) twr[n1] = tw[n1 * 17 + k2];
          for (int j = tg; j < Vr * 16; j += kWsGroup) {
            const int y = j >> 4;
            float2 v[8];
#pragma unroll
            for (int k1 = 0; k1 < 8; ++k1) v[k1] = Wo[widx(y, 8 * k2 + k1)];
            dft8<true>(v);
#pragma unroll
            for (int n1 = 0; n1 < 8; ++n1) Wo[widx(y, 8 * k2 + n1)] = n1 ? c_mulc(v[n1], twr[n1]) : v[0];
          }
        }
        nbar_sync(kBarX, kWsGroup);
        // I4: x-dim pass A' -> natural x; complex magnitude of valid outputs
        for (int j = tg; j < Vr * 8; j += kWsGroup) {
          const int y = j >> 3, n1 = j & 7;
          float2 v[16];
#pragma unroll
          for (int k2 = 0; k2 < 16; ++k2) v[k2] = Wo[widx(y, 8 * k2 + n1)];
          dft16<true>(v);
          const int gy = R0 + y;
          if (gy < cRows) {
            float* dst = Cout + (size_t)gy * cPitch;
            if (!wrapTile) {
              float* dstx = dst + (C0 - kX);
#pragma unroll
              for (int n2 = 0; n2 < 16; ++n2)
                if ((xMask >> n2) & 1u) dstx[n1 + 8 * n2] = cmag(v[n2]);
            } else {
              // fftW == dataW: window column dataW of row r is the torus
              // element (r + 1, 0) (see k_gabor_tiles)
#pragma unroll
              for (int n2 = 0; n2 < 16; ++n2) {
                const int x = n1 + 8 * n2;
                const int gx = C0 + x - kX;
                if (x >= kX && x < kX + V && gx < cCols) {
                  const float m = cmag(v[n2]);
                  if (!(gx == cCols - 1 && gy < cRows - 1)) dst[gx] = m;
                  if (gx == 0 && gy >= 1) Cout[(size_t)(gy - 1) * cPitch + cCols - 1] = m;
                }
              }
            }
          }
        }
        // buffer b may be refilled by orientation o + 2; the item's last two
        // orientations are ordered against the next tile by its barrier
        if (o - oB < nO - 2) nbar_arrive(kBarEmpty0 + b, kTileThreads);
      }
    }
  }
  tmem_fence_before();
  __syncthreads();
  tmem_fence_after();
  if ((t >> 5) == 0) tmem_dealloc_warp(*tmemSlot);
}

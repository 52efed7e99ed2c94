// Host side of the adjoint (include/bimp_b200_adjoint.h): one arena holding
// the float pyramid, maps, ReLU states and gradients of n equally sized
// images, and the launch sequences of the forward and backward.
//
// Nothing of the responses survives the forward: the backward recomputes each
// tile's spectrum and e + i o.  The per-cell scratch (complex cells C and
// their gradient, the inhibition maps T and R) exists for a chunk of images
// at a time; the forward and the backward walk the chunks in order, and the
// entries of images in different chunks share the same scratch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "bimp_b200.h"
#include "bimp_b200_adjoint.h"
#include "bimp_internal.h"
#include "kernels.h"

using namespace bimp_b200;

namespace {

int afail(int code, const std::string& m) {
  record_error(m);
  return code;
}

#define ADJ_CUDA(call)                                                                                  \
  do {                                                                                                  \
    cudaError_t e_ = (call);                                                                            \
    if (e_ != cudaSuccess)                                                                              \
      return afail(e_ == cudaErrorMemoryAllocation ? BIMP_ERR_NOMEM : BIMP_ERR_CUDA,                     \
                   std::string(#call) + ": " + cudaGetErrorString(e_));                                 \
  } while (0)

size_t up(size_t v, size_t a) { return (v + a - 1) / a * a; }

int rha(double v) { return static_cast<int>(v >= 0 ? std::floor(v + 0.5) : -std::floor(-v + 0.5)); }

}  // namespace

// Coefficients of the tile backward for one orientation, gathered into the
// Hermitian half layout of the tile spectra (entry j = py * kXhCols + slot,
// slot -> kx as in the forward transform's separation step):
//   A[j] = {G(k), G(-k), dGa(k), dGr(k)},  B[j] = {dGa(-k), dGr(-k)},
// with B = 0 where -k lies in k's own column (kx = 0 or 64), so that the
// backward's dot products visit every frequency once.
void gather_half(const float* G, const float* dA, const float* dR, float4* A, float2* B) {
  for (int j = 0; j < kSpecHalf; ++j) {
    const int py = j / kXhCols, sl = j - py * kXhCols;
    const int kx = sl < 64 ? (sl >> 2) + 16 * (sl & 3) : 64;
    const int ky = 16 * (py & 7) + (py >> 3);
    const int i1 = py * kTile + perm128(kx);
    const int i2 = perm128((kTile - ky) & 127) * kTile + perm128((kTile - kx) & 127);
    A[j] = make_float4(G[i1], G[i2], dA[i1], dR[i1]);
    const bool self = kx == 0 || kx == 64;
    B[j] = make_float2(self ? 0.f : dA[i2], self ? 0.f : dR[i2]);
  }
}

struct bimp_adjoint {
  int device = 0, W = 0, H = 0, n = 0, nScales = 0, maxLevel = 0;
  bimp_params params{};
  std::vector<ScaleHost> geo;
  char* mem = nullptr;
  size_t bytes = 0;
  std::vector<ScaleDev> h_sd;
  ScaleDev* d_sd = nullptr;
  TileWork* d_tiles = nullptr;
  int nTiles = 0;
  int2* d_sten = nullptr;                 // forward stencil blocks (data)
  int nSten = 0;
  int2* d_stenB = nullptr;                // backward gather blocks (window rows 0..dataH+1)
  int nStenB = 0;
  std::vector<float*> lvl, glvl;          // [level][image]
  std::vector<int> lw, lh, lp;            // per level (same for all images)
  float* d_lvl0 = nullptr;                // level 0 of every image, n * H rows of lp[0]
  float* d_glvl = nullptr;                // every level gradient, one block
  size_t glvlBytes = 0;
  PyrJobF* d_pyr = nullptr;               // [level-1][image] forward jobs
  PyrJobF* d_pyrAdj = nullptr;            // [level-1][image] transpose jobs
  float* d_M = nullptr;
  size_t maskStride = 0;
  std::vector<size_t> maskOff;
  float2* d_xscr = nullptr;               // per tile-backward CTA: the tile's image spectrum (Hermitian half)
  int bwdGrid = 0;                        // CTAs of the tile backward
  int chunk = 0;                          // images per chunk of the per-cell scratch
  bool pipelined = false;                 // the warp-specialised forward tile kernel fits every scale
  std::vector<int> tileStart, stenStart, stenBStart;   // per image (n + 1 entries)
  double* d_loss = nullptr;               // [0] loss, [1..4] parameter gradients
  double* d_gp = nullptr;
  unsigned int* d_max = nullptr;          // per entry + fault word

  int build(int dev, int w, int h, int ni, const float* lambdas, int nl, const bimp_params& p) {
    device = dev;
    W = w;
    H = h;
    n = ni;
    params = p;
    std::string err;
    if (!build_scales(w, h, std::vector<float>(lambdas, lambdas + nl), p, geo, err)) return afail(BIMP_ERR_INVALID, err);
    nScales = static_cast<int>(geo.size());
    for (auto& s : geo) maxLevel = std::max(maxLevel, s.level);
    // backward coefficients: G and the derivative spectra, gathered
    std::vector<float4> hA((size_t)nScales * kNumOri * kSpecHalf);
    std::vector<float2> hB((size_t)nScales * kNumOri * kSpecHalf);
    for (int s = 0; s < nScales; ++s) {
      std::vector<float> ea[kNumOri], oa[kNumOri], er[kNumOri], orr[kNumOri], dga, dgr;
      derivative_taps(geo[s], p, ea, oa, er, orr);
      tile_spectrum(ea, oa, geo[s].kW, geo[s].kX, dga);
      tile_spectrum(er, orr, geo[s].kW, geo[s].kX, dgr);
      for (int o = 0; o < kNumOri; ++o) {
        const size_t so = (size_t)o * kSpecFloats, ho = ((size_t)s * kNumOri + o) * kSpecHalf;
        gather_half(geo[s].spectrum.data() + so, dga.data() + so, dgr.data() + so, hA.data() + ho, hB.data() + ho);
      }
    }
    // ---- layout
    size_t at = 0;
    auto take = [&](size_t b) { const size_t o = up(at, 256); at = o + b; return o; };
    const size_t specB = sizeof(float) * (size_t)kNumOri * kSpecFloats;
    const size_t offG = take(specB * nScales);
    const size_t offBA = take(sizeof(float4) * hA.size()), offBB = take(sizeof(float2) * hB.size());
    int cw = w, ch = h;
    for (int l = 0; l <= maxLevel; ++l) {
      if (l > 0) { cw = (cw + 1) / 2; ch = (ch + 1) / 2; }
      lw.push_back(cw);
      lh.push_back(ch);
      lp.push_back(static_cast<int>(up(cw, 32)));
    }
    // levels grouped by level so that level 0 of all images is one block;
    // the level gradients form one block (cleared by one memset)
    std::vector<size_t> offL, offGL;   // one block of n images per level
    for (int l = 0; l <= maxLevel; ++l) offL.push_back(take(sizeof(float) * (size_t)n * lp[l] * lh[l]));
    at = up(at, 256);
    const size_t glBegin = at;
    for (int l = 0; l <= maxLevel; ++l) offGL.push_back(take(sizeof(float) * (size_t)n * lp[l] * lh[l]));
    glvlBytes = at - glBegin;
    maskStride = 0;
    for (auto& s : geo) {
      maskOff.push_back(maskStride);
      maskStride += (size_t)s.dataW * s.dataH;
    }
    const size_t offM = take(sizeof(float) * maskStride * n);
    std::vector<TileWork> tiles;
    std::vector<int2> sten, stenB;
    std::vector<ScaleDev> sds;
    std::vector<size_t> offD, offBits;                  // per entry
    std::vector<size_t> offC, offT, offR, offGC, offGW;  // per (chunk slot, scale)
    // images per chunk: all of them while their per-cell scratch stays under
    // kChunkBudget (BIMP_ADJOINT_CHUNK overrides it, for tests)
    {
      size_t per = 0;
      for (const ScaleHost& sc : geo) {
        const size_t cStride = (size_t)(sc.dataH + 2) * up(sc.dataW + 1, 32);
        per += 2 * sizeof(float) * kNumOri * cStride + sizeof(float) * kNumOri * (sc.dataH + 1) +
               2 * sizeof(float) * (size_t)sc.dataH * up(sc.dataW, 32);
      }
      constexpr size_t kChunkBudget = size_t(8) << 30;
      chunk = static_cast<int>(std::max<size_t>(1, std::min<size_t>(n, kChunkBudget / std::max<size_t>(per, 1))));
      if (const char* e = std::getenv("BIMP_ADJOINT_CHUNK")) {
        const int c = std::atoi(e);
        if (c > 0) chunk = std::min(c, n);
      }
    }
    for (int k = 0; k < chunk; ++k) {
      for (const ScaleHost& sc : geo) {
        const size_t cStride = (size_t)(sc.dataH + 2) * up(sc.dataW + 1, 32);
        const size_t mapB = sizeof(float) * (size_t)sc.dataH * up(sc.dataW, 32);
        offC.push_back(take(sizeof(float) * kNumOri * cStride));
        offGC.push_back(take(sizeof(float) * kNumOri * cStride));
        offGW.push_back(take(sizeof(float) * kNumOri * (sc.dataH + 1)));
        offT.push_back(take(mapB));
        offR.push_back(take(mapB));
      }
    }
    for (int i = 0; i < n; ++i) {
      tileStart.push_back(static_cast<int>(tiles.size()));
      stenStart.push_back(static_cast<int>(sten.size()));
      stenBStart.push_back(static_cast<int>(stenB.size()));
      for (int si = 0; si < nScales; ++si) {
        const ScaleHost& s = geo[si];
        ScaleDev d;
        std::memset(&d, 0, sizeof(d));
        d.dataW = s.dataW; d.dataH = s.dataH; d.fftW = s.fftW; d.fftH = s.fftH;
        d.kX = s.kX;
        d.V = kTile - 2 * s.kX;
        d.cRows = s.dataH + 2;
        d.cCols = s.dataW + 1;
        d.tilesX = (d.cCols + d.V - 1) / d.V;
        d.tilesY = (d.cRows + d.V - 1) / d.V;
        d.wrapW = s.fftW == s.dataW ? 1 : 0;
        d.lvlW = lw[s.level];
        d.lvlH = lh[s.level];
        d.lvlPitchF = lp[s.level];
        d.cPitch = static_cast<int>(up(s.dataW + 1, 32));
        d.cStride = (long long)(s.dataH + 2) * d.cPitch;
        for (int o = 0; o < kNumOri; ++o) {
          d.es1[o] = s.es1[o]; d.es2[o] = s.es2[o];
          d.in1[o] = s.in1[o]; d.in2[o] = s.in2[o];
          d.ih1[o] = rha(0.5 * s.in1[o]);
          d.ih2[o] = rha(0.5 * s.in2[o]);
        }
        d.pattern = 0;
        for (int set = 0; set < kNumOffsetSets && d.pattern == 0; ++set) {
          bool same = true;
          for (int o = 0; o < kNumOri; ++o)
            same = same && d.es1[o] == kOffsetSets[set][0][o] && d.es2[o] == kOffsetSets[set][1][o] &&
                   d.in1[o] == kOffsetSets[set][2][o] && d.in2[o] == kOffsetSets[set][3][o] &&
                   d.ih1[o] == kOffsetSets[set][4][o] && d.ih2[o] == kOffsetSets[set][5][o];
          if (same) d.pattern = set + 1;
        }
        d.radialGain = static_cast<float>(p.radial_gain);
        d.wTan = static_cast<float>(p.w_tan);
        d.wRad = static_cast<float>(p.w_rad);
        d.dPitch = static_cast<int>(up(s.dataW, 32));
        d.off = s.off;
        d.pyrstep = s.pyrstep;
        d.threshRatio = p.thresh_ratio;
        d.image = i;
        const int entry = static_cast<int>(sds.size());
        for (int tI = 0; tI < d.tilesX * d.tilesY; ++tI) tiles.push_back({entry, tI});
        const int nbx = (s.dataW + 31) / 32, nby = (s.dataH + kStencilBlockH - 1) / kStencilBlockH;
        for (int b = 0; b < nbx * nby; ++b) sten.push_back(make_int2(entry, b));
        const int nbx2 = (s.dataW + 1 + 31) / 32, nby2 = (s.dataH + 2 + 31) / 32;   // window + row dataH + 1
        for (int b = 0; b < nbx2 * nby2; ++b) stenB.push_back(make_int2(entry, b));
        const size_t mapB = sizeof(float) * (size_t)s.dataH * d.dPitch;
        offD.push_back(take(mapB));
        offBits.push_back(take(mapB));
        sds.push_back(d);
      }
    }
    tileStart.push_back(static_cast<int>(tiles.size()));
    stenStart.push_back(static_cast<int>(sten.size()));
    stenBStart.push_back(static_cast<int>(stenB.size()));
    nTiles = static_cast<int>(tiles.size());
    nSten = static_cast<int>(sten.size());
    nStenB = static_cast<int>(stenB.size());
    const size_t offSd = take(sizeof(ScaleDev) * sds.size());
    const size_t offT2 = take(sizeof(TileWork) * tiles.size());
    const size_t offSt = take(sizeof(int2) * sten.size());
    const size_t offStB = take(sizeof(int2) * stenB.size());
    const size_t offPyr = take(sizeof(PyrJobF) * std::max(1, maxLevel * n));
    const size_t offPyrA = take(sizeof(PyrJobF) * std::max(1, maxLevel * n));
    bwdGrid = std::max(1, std::min(nTiles, num_sms()));
    const size_t offXs = take(sizeof(float2) * (size_t)bwdGrid * kSpecHalf);
    const size_t offLoss = take(sizeof(double) * 8);
    const size_t offMax = take(sizeof(unsigned int) * (sds.size() + 1));
    const size_t offMaps = take(kTensorMapBytes * sds.size());
    bytes = at;
    cudaError_t e = cudaMalloc(&mem, bytes);
    if (e != cudaSuccess) {
      mem = nullptr;
      return afail(BIMP_ERR_NOMEM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed");
    }
    char* b = mem;
    float* dG = reinterpret_cast<float*>(b + offG);
    float4* dBA = reinterpret_cast<float4*>(b + offBA);
    float2* dBB = reinterpret_cast<float2*>(b + offBB);
    for (int l = 0; l <= maxLevel; ++l)
      for (int i = 0; i < n; ++i) {
        const size_t img = sizeof(float) * (size_t)i * lp[l] * lh[l];
        lvl.push_back(reinterpret_cast<float*>(b + offL[l] + img));
        glvl.push_back(reinterpret_cast<float*>(b + offGL[l] + img));
      }
    d_lvl0 = lvl[0];
    d_glvl = glvl[0];
    d_M = reinterpret_cast<float*>(b + offM);
    d_max = reinterpret_cast<unsigned int*>(b + offMax);
    for (size_t e2 = 0; e2 < sds.size(); ++e2) {
      ScaleDev& d = sds[e2];
      const int i = d.image, si = static_cast<int>(e2 % nScales);
      const ScaleHost& s = geo[si];
      d.lvlF = lvl[(size_t)s.level * n + i];
      d.gLvl = glvl[(size_t)s.level * n + i];
      d.G = dG + (size_t)si * kNumOri * kSpecFloats;
      d.bwA = dBA + (size_t)si * kNumOri * kSpecHalf;
      d.bwB = dBB + (size_t)si * kNumOri * kSpecHalf;
      const size_t slot = (size_t)(i % chunk) * nScales + si;   // chunk scratch shared across chunks
      d.C = reinterpret_cast<float*>(b + offC[slot]);
      d.Z = nullptr;
      d.gC = reinterpret_cast<float*>(b + offGC[slot]);
      d.gWrap = reinterpret_cast<float*>(b + offGW[slot]);
      d.T = reinterpret_cast<float*>(b + offT[slot]);
      d.R = reinterpret_cast<float*>(b + offR[slot]);
      d.D = reinterpret_cast<float*>(b + offD[e2]);
      d.bits = reinterpret_cast<unsigned int*>(b + offBits[e2]);
      d.M = d_M + (size_t)i * maskStride + maskOff[si];
      d.maxKey = d_max + e2;
    }
    std::vector<TensorMapBlob> maps(sds.size());
    {
      std::string err2;
      if (!encode_c_maps(sds.data(), static_cast<int>(sds.size()), maps.data(), err2))
        return afail(BIMP_ERR_CUDA, err2);
      for (size_t e2 = 0; e2 < sds.size(); ++e2) sds[e2].cMap = b + offMaps + e2 * kTensorMapBytes;
    }
    h_sd = sds;
    // the phased forward tile kernel unless BIMP_TILE_KERNEL=pipelined
    const char* kern = std::getenv("BIMP_TILE_KERNEL");
    pipelined = kern && std::strcmp(kern, "pipelined") == 0;
    for (const ScaleDev& d : sds) pipelined = pipelined && d.V <= pipelined_tile_max_valid();
    d_sd = reinterpret_cast<ScaleDev*>(b + offSd);
    d_tiles = reinterpret_cast<TileWork*>(b + offT2);
    d_sten = reinterpret_cast<int2*>(b + offSt);
    d_stenB = reinterpret_cast<int2*>(b + offStB);
    d_pyr = reinterpret_cast<PyrJobF*>(b + offPyr);
    d_pyrAdj = reinterpret_cast<PyrJobF*>(b + offPyrA);
    d_xscr = reinterpret_cast<float2*>(b + offXs);
    d_loss = reinterpret_cast<double*>(b + offLoss);
    d_gp = d_loss + 1;
    // uploads
    for (int si = 0; si < nScales; ++si)
      ADJ_CUDA(cudaMemcpy(dG + (size_t)si * kNumOri * kSpecFloats, geo[si].spectrum.data(), specB,
                          cudaMemcpyHostToDevice));
    ADJ_CUDA(cudaMemcpy(dBA, hA.data(), sizeof(float4) * hA.size(), cudaMemcpyHostToDevice));
    ADJ_CUDA(cudaMemcpy(dBB, hB.data(), sizeof(float2) * hB.size(), cudaMemcpyHostToDevice));
    ADJ_CUDA(cudaMemcpy(d_sd, sds.data(), sizeof(ScaleDev) * sds.size(), cudaMemcpyHostToDevice));
    ADJ_CUDA(cudaMemcpy(b + offMaps, maps.data(), kTensorMapBytes * sds.size(), cudaMemcpyHostToDevice));
    ADJ_CUDA(cudaMemcpy(d_tiles, tiles.data(), sizeof(TileWork) * tiles.size(), cudaMemcpyHostToDevice));
    ADJ_CUDA(cudaMemcpy(d_sten, sten.data(), sizeof(int2) * sten.size(), cudaMemcpyHostToDevice));
    ADJ_CUDA(cudaMemcpy(d_stenB, stenB.data(), sizeof(int2) * stenB.size(), cudaMemcpyHostToDevice));
    std::vector<PyrJobF> fj, aj;
    for (int l = 1; l <= maxLevel; ++l)
      for (int i = 0; i < n; ++i) {
        PyrJobF j;
        j.src = lvl[(size_t)(l - 1) * n + i];
        j.sw = lw[l - 1]; j.sh = lh[l - 1]; j.sp = lp[l - 1];
        j.dst = lvl[(size_t)l * n + i];
        j.dw = lw[l]; j.dh = lh[l]; j.dp = lp[l];
        fj.push_back(j);
        PyrJobF a = j;   // transpose: read level l gradient, scatter into level l-1
        a.src = glvl[(size_t)l * n + i];
        a.sp = lp[l];
        a.dst = glvl[(size_t)(l - 1) * n + i];
        a.dp = lp[l - 1];
        aj.push_back(a);
      }
    if (!fj.empty()) {
      ADJ_CUDA(cudaMemcpy(d_pyr, fj.data(), sizeof(PyrJobF) * fj.size(), cudaMemcpyHostToDevice));
      ADJ_CUDA(cudaMemcpy(d_pyrAdj, aj.data(), sizeof(PyrJobF) * aj.size(), cudaMemcpyHostToDevice));
    }
    return BIMP_OK;
  }

  int forward(const float* imgs, size_t pitch, const float* masks, double* loss, cudaStream_t s) {
    // the n images as one block of n * H rows
    ADJ_CUDA(cudaMemcpy2DAsync(d_lvl0, sizeof(float) * lp[0], imgs, sizeof(float) * pitch, sizeof(float) * W,
                               (size_t)n * H, cudaMemcpyDeviceToDevice, s));
    ADJ_CUDA(cudaMemcpyAsync(d_M, masks, sizeof(float) * maskStride * n, cudaMemcpyDeviceToDevice, s));
    for (int l = 1; l <= maxLevel; ++l) launch_pyr_f(d_pyr + (l - 1) * n, n, lw[l], lh[l], s);
    ADJ_CUDA(cudaMemsetAsync(d_max, 0, sizeof(unsigned int) * (h_sd.size() + 1), s));
    ADJ_CUDA(cudaMemsetAsync(d_loss, 0, sizeof(double) * 5, s));
    unsigned int* fault = d_max + h_sd.size();
    for (int i0 = 0; i0 < n; i0 += chunk) {
      const int i1 = std::min(n, i0 + chunk);
      launch_gabor_flt(d_sd, d_tiles + tileStart[i0], tileStart[i1] - tileStart[i0], fault, s, pipelined);
      launch_stencil(d_sd, d_sten + stenStart[i0], stenStart[i1] - stenStart[i0], fault, s, kStencilAdj);
      launch_masked_loss(d_sd, d_sten + stenStart[i0], stenStart[i1] - stenStart[i0], d_loss, d_gp, s);
    }
    if (loss) ADJ_CUDA(cudaMemcpyAsync(loss, d_loss, sizeof(double), cudaMemcpyDeviceToDevice, s));
    ADJ_CUDA(cudaGetLastError());
    return BIMP_OK;
  }

  // dL/dw_tan and dL/dw_rad (d_gp[2..3]) come from the forward's masked
  // sums; the backward accumulates alpha and rho and the image gradient.
  int backward(float* grad, size_t pitch, double* gparams, cudaStream_t s) {
    ADJ_CUDA(cudaMemsetAsync(d_glvl, 0, glvlBytes, s));
    ADJ_CUDA(cudaMemsetAsync(d_gp, 0, sizeof(double) * 2, s));
    for (int i0 = 0; i0 < n; i0 += chunk) {
      const int i1 = std::min(n, i0 + chunk);
      launch_stencil_bwd(d_sd, d_stenB + stenBStart[i0], stenBStart[i1] - stenBStart[i0], s);
      launch_gabor_bwd(d_sd, d_tiles + tileStart[i0], tileStart[i1] - tileStart[i0], bwdGrid, d_xscr, d_gp, s);
    }
    for (int l = maxLevel; l >= 1; --l) launch_pyr_f_adj(d_pyrAdj + (l - 1) * n, n, lw[l], lh[l], s);
    ADJ_CUDA(cudaMemcpy2DAsync(grad, sizeof(float) * pitch, d_glvl, sizeof(float) * lp[0], sizeof(float) * W,
                               (size_t)n * H, cudaMemcpyDeviceToDevice, s));
    if (gparams) ADJ_CUDA(cudaMemcpyAsync(gparams, d_gp, sizeof(double) * 4, cudaMemcpyDeviceToDevice, s));
    ADJ_CUDA(cudaGetLastError());
    return BIMP_OK;
  }
};

extern "C" {

int bimp_adjoint_create(bimp_adjoint** out, int width, int height, int n_images, const float* lambdas,
                        int n_lambdas, const bimp_params* params) {
  if (!out) return afail(BIMP_ERR_INVALID, "out is null");
  *out = nullptr;
  if (width < 16 || height < 16 || n_images <= 0 || !lambdas || n_lambdas <= 0)
    return afail(BIMP_ERR_INVALID, "bad adjoint arguments");
  if (width > 32767 || height > 32767) return afail(BIMP_ERR_UNSUPPORTED, "image sides above 32767");
  bimp_params p;
  bimp_default_params(&p);
  if (params) p = *params;
  int dev = 0;
  ADJ_CUDA(cudaGetDevice(&dev));
  int rc = configure_device(dev);
  if (rc != BIMP_OK) return rc;
  bimp_adjoint* a = new bimp_adjoint();
  rc = a->build(dev, width, height, n_images, lambdas, n_lambdas, p);
  if (rc != BIMP_OK) {
    if (a->mem) cudaFree(a->mem);
    delete a;
    return rc;
  }
  *out = a;
  return BIMP_OK;
}

int bimp_adjoint_destroy(bimp_adjoint* a) {
  if (!a) return BIMP_OK;
  cudaSetDevice(a->device);
  if (a->mem) cudaFree(a->mem);
  delete a;
  return BIMP_OK;
}

int bimp_adjoint_num_scales(const bimp_adjoint* a) { return a ? a->nScales : 0; }

size_t bimp_adjoint_device_bytes(const bimp_adjoint* a) { return a ? a->bytes : 0; }

int bimp_adjoint_mask_layout(const bimp_adjoint* a, int scale, int* data_w, int* data_h, size_t* offset,
                             size_t* mask_stride) {
  if (!a || scale < 0 || scale >= a->nScales) return afail(BIMP_ERR_INVALID, "bad scale");
  if (data_w) *data_w = a->geo[scale].dataW;
  if (data_h) *data_h = a->geo[scale].dataH;
  if (offset) *offset = a->maskOff[scale];
  if (mask_stride) *mask_stride = a->maskStride;
  return BIMP_OK;
}

int bimp_adjoint_forward(bimp_adjoint* a, const float* d_images, size_t pitch, const float* d_masks, double* d_loss,
                         void* stream) {
  if (!a || !d_images || !d_masks || pitch < (size_t)a->W) return afail(BIMP_ERR_INVALID, "bad forward arguments");
  ADJ_CUDA(cudaSetDevice(a->device));
  return a->forward(d_images, pitch, d_masks, d_loss, static_cast<cudaStream_t>(stream));
}

int bimp_adjoint_backward(bimp_adjoint* a, float* d_grad, size_t pitch, double* d_grad_params, void* stream) {
  if (!a || !d_grad || pitch < (size_t)a->W) return afail(BIMP_ERR_INVALID, "bad backward arguments");
  ADJ_CUDA(cudaSetDevice(a->device));
  return a->backward(d_grad, pitch, d_grad_params, static_cast<cudaStream_t>(stream));
}

int bimp_adjoint_dense_map(bimp_adjoint* a, int image, int scale, float* d_out, size_t ld, void* stream) {
  if (!a || !d_out || image < 0 || image >= a->n || scale < 0 || scale >= a->nScales)
    return afail(BIMP_ERR_INVALID, "bad dense-map arguments");
  const ScaleDev& d = a->h_sd[(size_t)image * a->nScales + scale];
  if (ld < (size_t)d.dataW) return afail(BIMP_ERR_INVALID, "ld too small");
  ADJ_CUDA(cudaMemcpy2DAsync(d_out, ld * sizeof(float), d.D, d.dPitch * sizeof(float), d.dataW * sizeof(float),
                             d.dataH, cudaMemcpyDeviceToDevice, static_cast<cudaStream_t>(stream)));
  return BIMP_OK;
}

int bimp_adjoint_complex_map(bimp_adjoint* a, int image, int scale, int orientation, float* d_out, size_t ld,
                             void* stream) {
  if (!a || !d_out || image < 0 || image >= a->n || scale < 0 || scale >= a->nScales || orientation < 0 ||
      orientation >= kNumOri)
    return afail(BIMP_ERR_INVALID, "bad complex-map arguments");
  const ScaleDev& d = a->h_sd[(size_t)image * a->nScales + scale];
  if (ld < (size_t)d.cCols) return afail(BIMP_ERR_INVALID, "ld smaller than data width + 1");
  // the complex cells survive the forward only for the images of its last chunk
  if (image < (a->n - 1) / a->chunk * a->chunk)
    return afail(BIMP_ERR_UNSUPPORTED, "complex cells of image " + std::to_string(image) +
                                           " were overwritten by a later chunk of the forward");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const float* src = d.C + (size_t)orientation * d.cStride;
  ADJ_CUDA(cudaMemcpy2DAsync(d_out, ld * sizeof(float), src, d.cPitch * sizeof(float), d.cCols * sizeof(float),
                             d.dataH + 1, cudaMemcpyDeviceToDevice, s));
  return BIMP_OK;
}

}  // extern "C"

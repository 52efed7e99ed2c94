// C ABI of the B200 BIMP detector: contexts (one image size), batches (many
// images of mixed sizes, one launch per kernel type, replayed as a CUDA
// graph), dense-map access and keypoint conversion.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "bimp_b200.h"
#include "bimp_b200_batch.h"
#include "bimp_internal.h"
#include "kernels.h"

using namespace bimp_b200;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define BIMP_CUDA(call)                                                              \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) {                                                         \
      return fail(e_ == cudaErrorMemoryAllocation ? BIMP_ERR_NOMEM : BIMP_ERR_CUDA,  \
                  std::string(#call) + ": " + cudaGetErrorString(e_));               \
    }                                                                                \
  } while (0)

std::mutex g_cfg_mutex;
bool g_cfg_done[128];

int ensure_device_configured(int dev) {
  std::lock_guard<std::mutex> lk(g_cfg_mutex);
  if (dev < 0 || dev >= 128) return fail(BIMP_ERR_NO_DEVICE, "device index out of range");
  if (g_cfg_done[dev]) return BIMP_OK;
  cudaDeviceProp prop;
  BIMP_CUDA(cudaGetDeviceProperties(&prop, dev));
  if (prop.major != 10) return fail(BIMP_ERR_NO_DEVICE, "this build targets sm_100a (B200)");
  BIMP_CUDA(configure_kernels());
  g_cfg_done[dev] = true;
  return BIMP_OK;
}

bimp_params default_params() {
  bimp_params p;
  p.gamma = 0.5;
  p.sigma_ratio = 0.56;
  p.size_ratio = 7.0;
  p.offset_ratio = 0.6;
  p.level_max = 7.5;
  p.radial_gain = 16.0;
  p.w_tan = 1.0;
  p.w_rad = 1.0;
  p.thresh_ratio = 0.104;
  return p;
}

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

int round_half_away(double v) {
  return static_cast<int>(v >= 0 ? std::floor(v + 0.5) : -std::floor(-v + 0.5));
}

// Programmatic dependent launch along the detection kernels: on unless
// BIMP_PDL=0 (kept switchable to measure both).
bool pdl_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("BIMP_PDL");
    return !(e && std::strcmp(e, "0") == 0);
  }();
  return on;
}

// Bump allocator over one device allocation.
struct Arena {
  size_t size = 0;
  char* base = nullptr;
  size_t reserve(size_t bytes) {
    const size_t at = align_up(size, 256);
    size = at + bytes;
    return at;
  }
};

}  // namespace

// Lets other translation units report through bimp_last_error().
void bimp_b200::record_error(const std::string& msg) { g_last_error = msg; }

// Kernel attributes and constants of `dev` (once per device), for other
// translation units that launch the kernels.
int bimp_b200::configure_device(int dev) { return ensure_device_configured(dev); }

// ---------------------------------------------------------------------------
// shared engine: N images with their own sizes, one wavelength bank
// ---------------------------------------------------------------------------
struct Engine {
  int device = 0;
  bimp_params params{};
  std::vector<ScaleHost> bank;          // geometry of the first image size + taps
  int nScales = 0;
  int nImages = 0;
  std::vector<int> widths, heights;         // geometry sizes (CudaStuff's width x height)
  std::vector<int> inWidths, inHeights;     // input image sizes (>= the geometry sizes)
  std::vector<std::vector<ScaleHost>> geo;   // per image per scale geometry
  // device memory
  char* d_mem = nullptr;
  size_t memBytes = 0;
  float* d_G = nullptr;
  std::vector<std::vector<uint8_t*>> lvl;    // per image per level
  std::vector<std::vector<int>> lvlW, lvlH, lvlP;
  std::vector<ScaleDev> h_sd;
  ScaleDev* d_sd = nullptr;
  TileWork* d_tiles = nullptr;   // the tile kernel's work list
  int nTiles = 0;                 // tiles of the current plan
  int nWork = 0;                  // entries of the work list
  int2* d_sten = nullptr;
  int nSten = 0;
  int2* d_rows = nullptr;
  int nRows = 0;
  NmsCta* d_nmsCtas = nullptr;          // the NMS kernels' row groups (one image each)
  int nNmsCtas = 0;
  int* d_nmsCount = nullptr;            // keypoints per NMS row group
  size_t resetBytes = 0;                // d_maxKeys and the fault word, zeroed per detection
  int* d_totals = nullptr;
  unsigned int* d_maxKeys = nullptr;
  unsigned int* d_fault = nullptr;      // set by the tile kernel, the stencil or the NMS if a bounded wait expired
  KpOut* d_outs = nullptr;
  std::vector<PyrJob> h_pyr;                 // grouped by level
  std::vector<int> pyrFirst, pyrCount, pyrLevels, pyrMaxW, pyrMaxH;   // per launch (up to 3 levels)
  PyrJob* d_pyr = nullptr;
  std::vector<size_t> imgKpOffset;           // internal keypoint buffers (batch)
  float* d_kpInternal = nullptr;
  int kpCapInternal = 0;
  int tileGrid = 0;    // CTAs of the tile kernel (each walks its items of the work list)
  int tileGridReq = 0; // the plan's grid: 0 one CTA per tile, > 0 the split plan's CTA bound
  bool tilePipelined = false;   // the warp-specialised tile kernel (every scale's V fits its row buffers)
  int tileCap = 0;     // capacity of d_tiles (the largest tile plan)
  int tilePolicy = 0, tileOrder = 0;

  // Tile plan (what the batch autotuner chooses between).
  // policy 0: V = 128 - 2 kX valid outputs per tile side (the largest);
  //        1: V rounded down to a multiple of 32 when that keeps at least
  //           3/4 of it, so that the valid-row passes split evenly over the
  //           16 warps of a tile (more tiles, fewer idle warps per tile).
  // order 0: tiles entry by entry; 1: the entries' tiles interleaved.
  // grid: CTAs of the tile kernel (<= 0: one per tile).
  static int plan_v(int kX, int policy) {
    const int vmax = kTile - 2 * kX;
    const int v32 = vmax / 32 * 32;
    return (policy == 1 && v32 * 4 >= vmax * 3) ? v32 : vmax;
  }
  // Balanced plan for a persistent grid of `grid` CTAs.  The (tile,
  // orientation) pairs, tile by tile in plan order, are cut into at most
  // `grid` contiguous runs of about equal cost; a run becomes one work item
  // per tile it touches (a tile cut between two CTAs is transformed forward by
  // both).  Costs come from the kernel's measured phase times (cycles between
  // its CTA barriers at 1080p, in units of one orientation of a V = 100
  // tile): per orientation, the product and inverse y-passes on all 128
  // columns 0.414, each round of the first inverse x-pass (16 items per valid
  // row inside the map over 512 threads) 0.0565, each round of the second
  // (8 items per row) 0.18, of which
  // the magnitudes and stores are 0.42 and scale with the share of the
  // tile's outputs inside the map; an item's forward transform and spectrum
  // store 1.35.  The smallest run bound that fits in `grid` runs is found by
  // bisection.  Item k of CTA b is
  // placed at index k * grid + b (the kernel strides its work list by the
  // grid); CTAs with fewer items get empty ones.  *usedGrid receives the
  // number of CTAs with work.
  static std::vector<TileWork> split_plan(const std::vector<TileWork>& tiles, const std::vector<ScaleDev>& sds,
                                          int grid, int* usedGrid) {
    const double kFwd = 1.35;
    std::vector<double> ori(tiles.size());
    double total = 0.0, worst = 0.0;
    for (size_t i = 0; i < tiles.size(); ++i) {
      const ScaleDev& d = sds[tiles[i].entry];
      const int ty = tiles[i].tile / d.tilesX, tx = tiles[i].tile - ty * d.tilesX;
      const int vr = std::min(d.V, d.cRows - ty * d.V);   // valid rows inside the map (the x-passes' rows)
      const double inside = (double)vr * std::min(d.V, d.cCols - tx * d.V) / ((double)d.V * d.V);
      const int r3 = (16 * vr + kTileThreads - 1) / kTileThreads, r4 = (8 * vr + kTileThreads - 1) / kTileThreads;
      ori[i] = 0.414 + 0.0565 * r3 + 0.18 * r4 * (0.58 + 0.42 * inside);
      total += kNumOri * ori[i] + kFwd;
      worst = std::max(worst, ori[i] + kFwd);
    }
    // greedy runs of the pair sequence under bound tau (a pair joins the
    // current run while the run stays within tau); returns the run count
    auto cut = [&](double tau, std::vector<std::vector<TileWork>>* runs) {
      int n = 0;
      double acc = 0.0;
      for (size_t i = 0; i < tiles.size(); ++i)
        for (int o = 0; o < kNumOri;) {
          if (n == 0 || (acc + kFwd + ori[i] > tau && acc > 0.0)) {
            ++n;
            acc = 0.0;
            if (runs) runs->emplace_back();
          }
          acc += kFwd + ori[i];   // the item's forward transform and first orientation
          int k = 1 + static_cast<int>(std::floor(std::max(0.0, tau - acc) / ori[i]));
          k = std::min(k, kNumOri - o);
          acc += (k - 1) * ori[i];
          if (runs) runs->back().push_back({tiles[i].entry, tiles[i].tile, o, o + k});
          o += k;
        }
      return n;
    };
    double lo = std::max(worst, total / std::max(1, grid)) * 0.999, hi = total + worst;
    for (int it = 0; it < 60 && hi - lo > 1e-6 * hi; ++it) {
      const double mid = 0.5 * (lo + hi);
      if (cut(mid, nullptr) <= grid) hi = mid;
      else lo = mid;
    }
    std::vector<std::vector<TileWork>> runs;
    cut(hi, &runs);
    const int g = static_cast<int>(runs.size());
    size_t depth = 0;
    for (auto& r : runs) depth = std::max(depth, r.size());
    std::vector<TileWork> out(depth * (size_t)g, TileWork{0, 0, 0, 0});
    for (int b = 0; b < g; ++b)
      for (size_t k = 0; k < runs[b].size(); ++k) out[k * (size_t)g + b] = runs[b][k];
    *usedGrid = g;
    return out;
  }
  static std::vector<TileWork> tile_plan(std::vector<ScaleDev>& sds, int policy, int order) {
    std::vector<std::vector<TileWork>> per(sds.size());
    for (size_t e = 0; e < sds.size(); ++e) {
      ScaleDev& d = sds[e];
      d.V = plan_v(d.kX, policy);
      d.tilesX = (d.cCols + d.V - 1) / d.V;
      d.tilesY = (d.cRows + d.V - 1) / d.V;
      for (int k = 0; k < d.tilesX * d.tilesY; ++k) per[e].push_back({static_cast<int>(e), k});
    }
    std::vector<TileWork> out;
    if (order == 0) {
      for (auto& v : per) out.insert(out.end(), v.begin(), v.end());
    } else {
      for (size_t k = 0;; ++k) {
        bool any = false;
        for (auto& v : per)
          if (k < v.size()) { out.push_back(v[k]); any = true; }
        if (!any) break;
      }
    }
    return out;
  }
  // The tile kernel's work list of a plan: one item per tile (grid <= 0, one
  // CTA each) or the balanced split plan for `grid` persistent CTAs.
  static std::vector<TileWork> work_list(std::vector<ScaleDev>& sds, int policy, int order, int grid, int* nTilesOut,
                                         int* gridOut) {
    std::vector<TileWork> tiles = tile_plan(sds, policy, order);
    *nTilesOut = static_cast<int>(tiles.size());
    *gridOut = static_cast<int>(tiles.size());
    if (grid > 0 && !tiles.empty()) return split_plan(tiles, sds, grid, gridOut);
    return tiles;
  }
  int retile(int policy, int order, int grid, int kernel = 0) {
    std::vector<ScaleDev> sds = h_sd;
    int nt = 0, g = 0;
    const std::vector<TileWork> work = work_list(sds, policy, order, grid, &nt, &g);
    if ((int)work.size() > tileCap) return fail(BIMP_ERR_INVALID, "tile plan larger than its buffer");
    BIMP_CUDA(cudaSetDevice(device));
    BIMP_CUDA(cudaMemcpy(d_sd, sds.data(), sizeof(ScaleDev) * sds.size(), cudaMemcpyHostToDevice));
    if (!work.empty())
      BIMP_CUDA(cudaMemcpy(d_tiles, work.data(), sizeof(TileWork) * work.size(), cudaMemcpyHostToDevice));
    h_sd = sds;
    nTiles = nt;
    nWork = static_cast<int>(work.size());
    tileGrid = g;
    tileGridReq = grid > 0 ? grid : 0;
    tilePolicy = policy;
    tileOrder = order;
    tilePipelined = kernel == 1 && pipelined_fits();
    return BIMP_OK;
  }
  // The warp-specialised tile kernel takes every scale with V up to its row
  // buffers' height.
  bool pipelined_fits() const {
    for (const ScaleDev& d : h_sd)
      if (d.V > pipelined_tile_max_valid()) return false;
    return true;
  }
  // Default kernel: the phased one (measured faster on the plain 1080p
  // detection); BIMP_TILE_KERNEL=pipelined selects the warp-specialised one,
  // and a batch's tile plan (or its autotuner) may choose either.
  bool pipelined_by_default() const {
    const char* k = std::getenv("BIMP_TILE_KERNEL");
    return k && std::strcmp(k, "pipelined") == 0 && pipelined_fits();
  }

  // inW/inH (null: the geometry sizes) are the sizes of the images a
  // detection takes: each pyramid level of the input is computed in full,
  // and each scale filters the top-left dataW x dataH window of its level.
  int build(int dev, const int* w, const int* h, int n, const float* lambdas, int nl,
            const bimp_params& p, int internalKpCap, const int* inW = nullptr, const int* inH = nullptr) {
    device = dev;
    params = p;
    nImages = n;
    widths.assign(w, w + n);
    heights.assign(h, h + n);
    inWidths.assign(inW ? inW : w, (inW ? inW : w) + n);
    inHeights.assign(inH ? inH : h, (inH ? inH : h) + n);
    std::vector<float> lam(lambdas, lambdas + nl);
    std::string err;
    geo.resize(n);
    for (int i = 0; i < n; ++i) {
      if (w[i] < 2 || h[i] < 2) return fail(BIMP_ERR_INVALID, "image size must be at least 2x2");
      if (w[i] > 32767 || h[i] > 32767 || inWidths[i] > 32767 || inHeights[i] > 32767)   // int16 tile index maps
        return fail(BIMP_ERR_UNSUPPORTED, "image sides above 32767 pixels are not supported");
      if (inWidths[i] < w[i] || inHeights[i] < h[i])
        return fail(BIMP_ERR_INVALID, "input image smaller than the context's size");
      if (!build_scales(w[i], h[i], lam, p, geo[i], err)) return fail(BIMP_ERR_INVALID, err);
      if (i == 0) bank = geo[0];
      for (auto& s : geo[i]) {        // taps and spectra are shared with image 0
        for (int o = 0; o < kNumOri; ++o) { s.even[o].clear(); s.odd[o].clear(); }
        if (i > 0) s.spectrum.clear();
      }
    }
    for (auto& s : geo[0]) s.spectrum.clear();
    nScales = static_cast<int>(bank.size());

    // ---- layout
    Arena a;
    const size_t offG = a.reserve(sizeof(float) * (size_t)nScales * kNumOri * kSpecFloats);
    lvl.assign(n, {});
    lvlW.assign(n, {});
    lvlH.assign(n, {});
    lvlP.assign(n, {});
    std::vector<std::vector<size_t>> offLvl(n);
    std::vector<std::vector<size_t>> offC(n), offD(n), offS(n);
    int maxLevel = 0;
    for (auto& s : bank) maxLevel = std::max(maxLevel, s.level);
    for (int i = 0; i < n; ++i) {
      int cw = inWidths[i], ch = inHeights[i];
      for (int l = 0; l <= maxLevel; ++l) {
        if (l > 0) { cw = (cw + 1) / 2; ch = (ch + 1) / 2; }
        const int pitch = static_cast<int>(align_up(cw, 16));
        lvlW[i].push_back(cw);
        lvlH[i].push_back(ch);
        lvlP[i].push_back(pitch);
        offLvl[i].push_back(a.reserve((size_t)pitch * ch));
      }
      for (auto& s : geo[i]) {
        const int cPitch = static_cast<int>(align_up(s.dataW + 1, 32));
        offC[i].push_back(a.reserve(sizeof(float) * (size_t)kNumOri * (s.dataH + 2) * cPitch));
        const int dPitch = static_cast<int>(align_up(s.dataW, 32));
        offD[i].push_back(a.reserve(sizeof(float) * (size_t)s.dataH * dPitch));
        offS[i].push_back(a.reserve(sizeof(float) * (size_t)s.dataH * dPitch));
      }
    }
    // work lists
    std::vector<TileWork> tiles;
    std::vector<int2> sten, rows;
    std::vector<size_t> maskWords;   // per entry
    std::vector<int> imgRowStart;
    std::vector<ScaleDev> sds;
    for (int i = 0; i < n; ++i) {
      imgRowStart.push_back(static_cast<int>(rows.size()));
      for (int si = 0; si < nScales; ++si) {
        const ScaleHost& s = geo[i][si];
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
        d.lvlW = lvlW[i][s.level];
        d.lvlH = lvlH[i][s.level];
        d.lvlPitch = lvlP[i][s.level];
        d.cPitch = static_cast<int>(align_up(s.dataW + 1, 32));
        d.cStride = (long long)(s.dataH + 2) * d.cPitch;
        for (int o = 0; o < kNumOri; ++o) {
          d.es1[o] = s.es1[o]; d.es2[o] = s.es2[o];
          d.in1[o] = s.in1[o]; d.in2[o] = s.in2[o];
          d.ih1[o] = round_half_away(0.5 * s.in1[o]);   // cuda_bimp.cuh:495-496
          d.ih2[o] = round_half_away(0.5 * s.in2[o]);
        }
        d.pattern = 0;
        for (int set = 0; set < kNumOffsetSets && d.pattern == 0; ++set) {
          bool same = true;
          for (int o = 0; o < kNumOri; ++o) {
            same = same && d.es1[o] == kOffsetSets[set][0][o] && d.es2[o] == kOffsetSets[set][1][o] &&
                   d.in1[o] == kOffsetSets[set][2][o] && d.in2[o] == kOffsetSets[set][3][o] &&
                   d.ih1[o] == kOffsetSets[set][4][o] && d.ih2[o] == kOffsetSets[set][5][o];
          }
          if (same) d.pattern = set + 1;
        }
        d.radialGain = static_cast<float>(p.radial_gain);
        d.wTan = static_cast<float>(p.w_tan);
        d.wRad = static_cast<float>(p.w_rad);
        d.dPitch = static_cast<int>(align_up(s.dataW, 32));
        d.off = s.off;
        d.pyrstep = s.pyrstep;
        d.kpSize = s.lambda * s.pyrstep;
        d.kpOctave = static_cast<int>(s.lambda * s.pyrstep);
        d.threshRatio = p.thresh_ratio;
        d.image = i;
        const int entry = static_cast<int>(sds.size());
        d.rowBase = static_cast<int>(rows.size());
        for (int tIdx = 0; tIdx < d.tilesX * d.tilesY; ++tIdx) tiles.push_back({entry, tIdx});
        const int nbx = (s.dataW + 31) / 32, nby = (s.dataH + kStencilBlockH - 1) / kStencilBlockH;
        for (int b = 0; b < nbx * nby; ++b) sten.push_back(make_int2(entry, b));
        const int yEnd = std::min(s.dataH - s.off - 1, s.dataH - 2);
        // keypoint-decision words: 32-pixel-aligned words covering a row's
        // candidate pixels (off, xEnd)
        const int xEnd = std::min(s.dataW - s.off, s.dataW - 1);
        d.nmsChunks = xEnd > s.off + 1 ? ((xEnd - 1) >> 5) - ((s.off + 1) >> 5) + 1 : 0;
        // the NMS work: each candidate row in 512-pixel-aligned pieces,
        // {entry, row | piece << 16}
        if (d.nmsChunks > 0)
          for (int y = s.off + 1; y <= yEnd; ++y)
            for (int pc = (s.off + 1) >> 9; pc <= (xEnd - 1) >> 9; ++pc)
              rows.push_back(make_int2(entry, (y - s.off - 1) | (pc << 16)));
        maskWords.push_back((size_t)std::max(0, yEnd - s.off) * d.nmsChunks);
        sds.push_back(d);
      }
    }
    imgRowStart.push_back(static_cast<int>(rows.size()));
    // NMS row groups: consecutive candidate rows of one image, kNmsRowsPerCta per CTA
    std::vector<NmsCta> nmsCtas;
    for (int i = 0; i < n; ++i) {
      const int first = static_cast<int>(nmsCtas.size());
      for (int r = imgRowStart[i]; r < imgRowStart[i + 1]; r += kNmsRowsPerCta)
        nmsCtas.push_back({r, std::min(kNmsRowsPerCta, imgRowStart[i + 1] - r), first, i, 0});
      if (static_cast<int>(nmsCtas.size()) > first) nmsCtas.back().last = 1;
    }
    nNmsCtas = static_cast<int>(nmsCtas.size());
    // pyramid jobs: up to 3 levels per launch (levels 1-3 from level 0,
    // 4-6 from level 3, ...)
    pyrFirst.clear(); pyrCount.clear(); pyrLevels.clear(); pyrMaxW.clear(); pyrMaxH.clear(); h_pyr.clear();
    for (int base = 0; base < maxLevel; base += 3) {
      const int K = std::min(3, maxLevel - base);
      pyrFirst.push_back(static_cast<int>(h_pyr.size()));
      int mw = 0, mh = 0;
      for (int i = 0; i < n; ++i) {
        PyrJob j{};
        j.sw = lvlW[i][base]; j.sh = lvlH[i][base]; j.sp = lvlP[i][base];
        for (int m = 0; m < K; ++m) {
          j.dw[m] = lvlW[i][base + m + 1]; j.dh[m] = lvlH[i][base + m + 1]; j.dp[m] = lvlP[i][base + m + 1];
        }
        h_pyr.push_back(j);
        mw = std::max(mw, j.dw[K - 1]); mh = std::max(mh, j.dh[K - 1]);
      }
      pyrCount.push_back(n);
      pyrLevels.push_back(K);
      pyrMaxW.push_back(mw);
      pyrMaxH.push_back(mh);
    }
    nTiles = static_cast<int>(tiles.size());
    // Default tile plan: the balanced split over one persistent CTA per SM.
    // BIMP_TILE_GRID=g uses g CTAs instead (g <= 0: one CTA per tile).
    BIMP_CUDA(cudaSetDevice(dev));
    const int sms = num_sms();
    int defGrid = sms;
    if (const char* g = std::getenv("BIMP_TILE_GRID")) defGrid = std::atoi(g);
    std::vector<TileWork> work = tiles;
    tileGrid = nTiles;
    if (defGrid > 0 && !tiles.empty()) work = split_plan(tiles, sds, defGrid, &tileGrid);
    nWork = static_cast<int>(work.size());
    tileGridReq = std::max(0, defGrid);
    nSten = static_cast<int>(sten.size());
    nRows = static_cast<int>(rows.size());
    const size_t offSd = a.reserve(sizeof(ScaleDev) * sds.size());
    {   // the tile buffer holds the largest plan the autotuner may choose
      // (and room for other grids a caller may ask for: a split plan's
      // padded list holds about nTiles + 3 grid entries when the tiles'
      // costs are within a factor of two; a plan beyond the buffer is
      // refused by retile)
      tileCap = nWork;
      int maxTiles = 0;
      const int grids[4] = {0, sms, 2 * sms, defGrid};
      for (int policy = 0; policy < 2; ++policy)
        for (int order = 0; order < 2; ++order)
          for (int g : grids) {
            std::vector<ScaleDev> tmp = sds;
            int nt = 0, ng = 0;
            tileCap = std::max(tileCap, static_cast<int>(work_list(tmp, policy, order, g, &nt, &ng).size()));
            maxTiles = std::max(maxTiles, nt);
          }
      tileCap = std::max(tileCap, 2 * maxTiles + 6 * sms);
    }
    const size_t offTiles = a.reserve(sizeof(TileWork) * std::max<size_t>(1, (size_t)tileCap));
    const size_t offSten = a.reserve(sizeof(int2) * std::max<size_t>(1, sten.size()));
    const size_t offRows = a.reserve(sizeof(int2) * std::max<size_t>(1, rows.size()));
    const size_t offNmsCtas = a.reserve(sizeof(NmsCta) * std::max<size_t>(1, nmsCtas.size()));
    const size_t offTotals = a.reserve(sizeof(int) * n);
    // per-detection reset region: the map maxima and the fault word
    resetBytes = sizeof(unsigned int) * (sds.size() + 1);
    const size_t offMax = a.reserve(resetBytes);
    const size_t offNmsCount = a.reserve(sizeof(int) * std::max<size_t>(1, nmsCtas.size()));
    const size_t offOuts = a.reserve(sizeof(KpOut) * n);
    const size_t offPyr = a.reserve(sizeof(PyrJob) * std::max<size_t>(1, h_pyr.size()));
    const size_t offMaps = a.reserve(kTensorMapBytes * sds.size());
    std::vector<size_t> offMask;
    for (size_t w : maskWords) offMask.push_back(a.reserve(sizeof(unsigned int) * std::max<size_t>(1, w)));
    size_t offKp = 0;
    kpCapInternal = internalKpCap;
    if (internalKpCap > 0)
      offKp = a.reserve(sizeof(float) * (size_t)n * BIMP_KP_VECTOR_LENGTH * internalKpCap);

    memBytes = a.size;
    cudaError_t e = cudaMalloc(&d_mem, memBytes);
    if (e != cudaSuccess) {
      d_mem = nullptr;
      return fail(BIMP_ERR_NOMEM, std::string("cudaMalloc of ") + std::to_string(memBytes) +
                                      " bytes: " + cudaGetErrorString(e));
    }
    char* base = d_mem;
    d_G = reinterpret_cast<float*>(base + offG);
    for (int i = 0; i < n; ++i) {
      for (size_t l = 0; l < offLvl[i].size(); ++l)
        lvl[i].push_back(reinterpret_cast<uint8_t*>(base + offLvl[i][l]));
    }
    for (int i = 0, e2 = 0; i < n; ++i) {
      for (int si = 0; si < nScales; ++si, ++e2) {
        ScaleDev& d = sds[e2];
        const ScaleHost& s = geo[i][si];
        d.lvl = lvl[i][s.level];
        d.G = d_G + (size_t)si * kNumOri * kSpecFloats;
        d.C = reinterpret_cast<float*>(base + offC[i][si]);
        d.D = reinterpret_cast<float*>(base + offD[i][si]);
        d.S = reinterpret_cast<float*>(base + offS[i][si]);
        d.maxKey = reinterpret_cast<unsigned int*>(base + offMax) + e2;
        d.nmsMask = reinterpret_cast<unsigned int*>(base + offMask[e2]);
      }
    }
    for (size_t g = 0, k = 0; g < pyrFirst.size(); ++g)
      for (int i = 0; i < n; ++i, ++k) {
        const int base = 3 * static_cast<int>(g);
        h_pyr[k].src = lvl[i][base];
        for (int m = 0; m < pyrLevels[g]; ++m) h_pyr[k].dst[m] = lvl[i][base + m + 1];
      }
    // TMA tensor maps of the complex-cell maps (the stencil's staging)
    std::vector<TensorMapBlob> maps(sds.size());
    {
      std::string err;
      if (!encode_c_maps(sds.data(), static_cast<int>(sds.size()), maps.data(), err)) return fail(BIMP_ERR_CUDA, err);
      for (size_t e2 = 0; e2 < sds.size(); ++e2) sds[e2].cMap = base + offMaps + e2 * kTensorMapBytes;
    }
    h_sd = sds;
    tilePipelined = pipelined_by_default();
    d_sd = reinterpret_cast<ScaleDev*>(base + offSd);
    d_tiles = reinterpret_cast<TileWork*>(base + offTiles);
    d_sten = reinterpret_cast<int2*>(base + offSten);
    d_rows = reinterpret_cast<int2*>(base + offRows);
    d_nmsCtas = reinterpret_cast<NmsCta*>(base + offNmsCtas);
    d_totals = reinterpret_cast<int*>(base + offTotals);
    d_maxKeys = reinterpret_cast<unsigned int*>(base + offMax);
    d_nmsCount = reinterpret_cast<int*>(base + offNmsCount);
    d_fault = d_maxKeys + sds.size();
    d_outs = reinterpret_cast<KpOut*>(base + offOuts);
    d_pyr = reinterpret_cast<PyrJob*>(base + offPyr);
    d_kpInternal = internalKpCap > 0 ? reinterpret_cast<float*>(base + offKp) : nullptr;

    // ---- uploads (setup only)
    for (int si = 0; si < nScales; ++si)
      BIMP_CUDA(cudaMemcpy(d_G + (size_t)si * kNumOri * kSpecFloats, bank[si].spectrum.data(),
                           sizeof(float) * kNumOri * kSpecFloats, cudaMemcpyHostToDevice));
    for (auto& s : bank) { s.spectrum.clear(); s.spectrum.shrink_to_fit(); }
    BIMP_CUDA(cudaMemcpy(d_sd, sds.data(), sizeof(ScaleDev) * sds.size(), cudaMemcpyHostToDevice));
    BIMP_CUDA(cudaMemcpy(base + offMaps, maps.data(), kTensorMapBytes * sds.size(), cudaMemcpyHostToDevice));
    if (!work.empty())
      BIMP_CUDA(cudaMemcpy(d_tiles, work.data(), sizeof(TileWork) * work.size(), cudaMemcpyHostToDevice));
    if (!sten.empty())
      BIMP_CUDA(cudaMemcpy(d_sten, sten.data(), sizeof(int2) * sten.size(), cudaMemcpyHostToDevice));
    if (!rows.empty())
      BIMP_CUDA(cudaMemcpy(d_rows, rows.data(), sizeof(int2) * rows.size(), cudaMemcpyHostToDevice));
    if (!nmsCtas.empty())
      BIMP_CUDA(cudaMemcpy(d_nmsCtas, nmsCtas.data(), sizeof(NmsCta) * nmsCtas.size(), cudaMemcpyHostToDevice));
    // images without candidate rows keep a total of zero
    BIMP_CUDA(cudaMemset(d_totals, 0, sizeof(int) * n));
    if (!h_pyr.empty())
      BIMP_CUDA(cudaMemcpy(d_pyr, h_pyr.data(), sizeof(PyrJob) * h_pyr.size(), cudaMemcpyHostToDevice));
    if (internalKpCap > 0) {
      std::vector<KpOut> outs(n);
      for (int i = 0; i < n; ++i) {
        outs[i].kp = d_kpInternal + (size_t)i * BIMP_KP_VECTOR_LENGTH * internalKpCap;
        outs[i].ld = internalKpCap;
        outs[i].capacity = internalKpCap;
        outs[i].aos = 0;
      }
      BIMP_CUDA(cudaMemcpy(d_outs, outs.data(), sizeof(KpOut) * n, cudaMemcpyHostToDevice));
    }
    BIMP_CUDA(cudaMemset(d_maxKeys, 0, resetBytes));
    return BIMP_OK;
  }

  int stage(int which, cudaStream_t s) {
    switch (which) {
      case 0:
        // the first launch also zeroes the per-detection reset words
        for (size_t l = 0; l < pyrFirst.size(); ++l)
          launch_pyr(d_pyr + pyrFirst[l], pyrCount[l], pyrLevels[l], pyrMaxW[l], pyrMaxH[l], s,
                     l == 0 ? d_maxKeys : nullptr, l == 0 ? static_cast<int>(resetBytes / sizeof(unsigned int)) : 0);
        break;
      // stages 1-3 follow the previous stage's kernel with programmatic
      // dependent launch (each waits in the kernel for its predecessor)
      case 1:
        if (nWork > 0) launch_gabor(d_sd, d_tiles, nWork, tileGrid, d_fault, s, tilePipelined, pdl_enabled());
        break;
      case 2:
        if (nSten > 0) launch_stencil(d_sd, d_sten, nSten, d_fault, s, kStencilD, pdl_enabled());
        break;
      case 3:
        launch_nms_two_pass(d_sd, d_rows, d_nmsCtas, nNmsCtas, d_nmsCount, d_totals, d_outs, s, pdl_enabled());
        break;
      default:
        return fail(BIMP_ERR_INVALID, "unknown stage");
    }
    BIMP_CUDA(cudaGetLastError());
    return BIMP_OK;
  }

  int kernel_launches() const {
    return static_cast<int>(pyrFirst.size()) + (nTiles > 0) + (nSten > 0) + 2 * (nNmsCtas > 0);
  }

  // Everything after the level-0 images are in place.
  int enqueue(cudaStream_t s) {
    // the reset of the map maxima and the fault word: done by the first
    // pyramid launch, or (a bank without pyramid levels) by a memset
    if (pyrFirst.empty()) BIMP_CUDA(cudaMemsetAsync(d_maxKeys, 0, resetBytes, s));
    int rc = stage(0, s);
    if (rc != BIMP_OK) return rc;
    for (int k = 1; k <= 3; ++k) {
      rc = stage(k, s);
      if (rc != BIMP_OK) return rc;
    }
    return BIMP_OK;
  }

  void release() {
    if (d_mem) cudaFree(d_mem);
    d_mem = nullptr;
  }
};

// ---------------------------------------------------------------------------
// context: one image size
// ---------------------------------------------------------------------------
struct bimp_context {
  Engine eng;
  int width = 0, height = 0;         // geometry (CudaStuff) size
  int inWidth = 0, inHeight = 0;     // size of the images a detection takes
  std::vector<ScaleHost> info;
  // host path: pinned count/fault words; device scratch the NMS writes
  // cv::KeyPoint records into before the single copy to the caller's array
  int* h_count = nullptr;   // pinned: [0] keypoint total, [1] device fault word
  float* d_kpScratch = nullptr;
  int d_kpScratchCap = 0;
  // pinned host staging of the records, and how many records go back with
  // the count before the first synchronisation (the last call's count plus
  // a margin), so that one synchronisation usually serves a whole call
  bimp_keypoint* h_stage = nullptr;
  int h_stageCap = 0;
  int specRecords = 1024;
  // line/edge detection, allocated on first use: e + i o of one scale, that
  // scale's descriptor and tile list
  float2* d_leZ = nullptr;
  ScaleDev* d_leSd = nullptr;
  TileWork* d_leTiles = nullptr;
  // the detection's fixed launch sequence (max reset, pyramid, tile kernel,
  // stencil, NMS), captured once at creation and launched into the caller's
  // stream after each call's input copies; null if the capture failed
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  // the output descriptor last written on the device (not rewritten when
  // unchanged, unless the context was ever used in a caller's stream
  // capture: a replay of that graph rewrites it behind this record)
  KpOut lastOut{};
  bool outSet = false;
  bool captured = false;
};

struct bimp_batch {
  Engine eng;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t capStream = nullptr;
  int* h_totals = nullptr;   // pinned: n_images totals, then the device fault word
  std::vector<bimp_keypoint> tmp;
};

// Host frames in flight: `depth` contexts of one image size, each with its
// own stream, used round robin, so that one frame's copies overlap another
// frame's kernels.
struct bimp_pipeline {
  std::vector<bimp_context*> ctx;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> done;
  std::vector<int> spec;
  int depth = 0, capacity = 0, head = 0, inFlight = 0, device = 0;
};

namespace {
// (Re)captures the batch's detection into its CUDA graph.
int capture_batch(bimp_batch* b) {
  if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
  if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
  cudaError_t e = cudaStreamBeginCapture(b->capStream, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    const int rc2 = b->eng.enqueue(b->capStream);
    const cudaError_t e2 = cudaStreamEndCapture(b->capStream, &b->graph);
    e = rc2 != BIMP_OK ? cudaErrorUnknown : e2;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
  if (e != cudaSuccess) return fail(BIMP_ERR_CUDA, std::string("batch graph setup: ") + cudaGetErrorString(e));
  return BIMP_OK;
}
// Captures a context's launch sequence into its graph.  On any failure the
// context keeps no graph and launches the same kernels directly.
void capture_ctx(bimp_context* c) {
  cudaStream_t cs = nullptr;
  if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  cudaGraph_t g = nullptr;
  if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
    const int rc = c->eng.enqueue(cs);
    const cudaError_t e = cudaStreamEndCapture(cs, &g);
    cudaGraphExec_t x = nullptr;
    if (rc == BIMP_OK && e == cudaSuccess && g && cudaGraphInstantiate(&x, g, 0) == cudaSuccess) {
      c->graph = g;
      c->exec = x;
      g = nullptr;
    }
  }
  if (g) cudaGraphDestroy(g);
  cudaGetLastError();
  cudaStreamDestroy(cs);
}
}  // namespace

extern "C" {

const char* bimp_version(void) { return "bimp_b200 0.1 (sm_100a)"; }
const char* bimp_last_error(void) { return g_last_error.c_str(); }
void bimp_default_params(bimp_params* p) {
  if (p) *p = default_params();
}

int bimp_make_lambdas_log(float start, float end, int spo, float* out, int cap, int* n) {
  if (!n || spo <= 0 || !(start > 0.f)) return fail(BIMP_ERR_INVALID, "bad makeLambdasLog arguments");
  const std::vector<float> v = make_lambdas_log(start, end, spo);
  *n = static_cast<int>(v.size());
  if (out)
    for (int i = 0; i < std::min(cap, *n); ++i) out[i] = v[i];
  return BIMP_OK;
}

int bimp_make_lambdas_lin(float start, float end, int num, float* out, int cap, int* n) {
  if (!n || num <= 0) return fail(BIMP_ERR_INVALID, "bad makeLambdasLin arguments");
  const std::vector<float> v = make_lambdas_lin(start, end, num);
  *n = static_cast<int>(v.size());
  if (out)
    for (int i = 0; i < std::min(cap, *n); ++i) out[i] = v[i];
  return BIMP_OK;
}

int bimp_snap_transform_size(int n) { return snap_transform_size(n); }

int bimp_ctx_create_for_input(bimp_context** ctx, int width, int height, int input_width, int input_height,
                              const float* lambdas, int n_lambdas, const bimp_params* params) {
  if (!ctx) return fail(BIMP_ERR_INVALID, "ctx is null");
  *ctx = nullptr;
  if (!lambdas || n_lambdas <= 0) return fail(BIMP_ERR_INVALID, "empty wavelength list");
  if (width < 2 || height < 2) return fail(BIMP_ERR_INVALID, "image size must be at least 2x2");
  if (input_width < width || input_height < height)
    return fail(BIMP_ERR_INVALID, "input image smaller than the context's size");
  int dev = 0;
  BIMP_CUDA(cudaGetDevice(&dev));
  int rc = ensure_device_configured(dev);
  if (rc != BIMP_OK) return rc;
  bimp_context* c = new bimp_context();
  c->width = width;
  c->height = height;
  c->inWidth = input_width;
  c->inHeight = input_height;
  const bimp_params p = params ? *params : default_params();
  rc = c->eng.build(dev, &width, &height, 1, lambdas, n_lambdas, p, 0, &input_width, &input_height);
  if (rc != BIMP_OK) {
    c->eng.release();
    delete c;
    return rc;
  }
  c->info = c->eng.geo[0];
  cudaError_t e = cudaMallocHost(&c->h_count, 2 * sizeof(int));
  if (e != cudaSuccess) {
    c->eng.release();
    delete c;
    return fail(BIMP_ERR_NOMEM, "cudaMallocHost failed");
  }
  capture_ctx(c);
  *ctx = c;
  return BIMP_OK;
}

int bimp_ctx_create(bimp_context** ctx, int width, int height, const float* lambdas, int n_lambdas,
                    const bimp_params* params) {
  return bimp_ctx_create_for_input(ctx, width, height, width, height, lambdas, n_lambdas, params);
}

int bimp_ctx_destroy(bimp_context* c) {
  if (!c) return BIMP_OK;
  cudaSetDevice(c->eng.device);
  if (c->exec) cudaGraphExecDestroy(c->exec);
  if (c->graph) cudaGraphDestroy(c->graph);
  c->eng.release();
  if (c->h_count) cudaFreeHost(c->h_count);
  if (c->d_kpScratch) cudaFree(c->d_kpScratch);
  if (c->h_stage) cudaFreeHost(c->h_stage);
  if (c->d_leZ) cudaFree(c->d_leZ);
  if (c->d_leSd) cudaFree(c->d_leSd);
  if (c->d_leTiles) cudaFree(c->d_leTiles);
  delete c;
  return BIMP_OK;
}

int bimp_ctx_num_scales(const bimp_context* c) { return c ? c->eng.nScales : 0; }

int bimp_ctx_scale_info(const bimp_context* c, int s, bimp_scale_info* out) {
  if (!c || !out || s < 0 || s >= c->eng.nScales) return fail(BIMP_ERR_INVALID, "bad scale index");
  const ScaleHost& h = c->info[s];
  out->lambda_full = h.lambda2;
  out->lambda_level = h.lambda;
  out->pyrstep = h.pyrstep;
  out->kernel_w = h.kW;
  out->kernel_x = h.kX;
  out->data_w = h.dataW;
  out->data_h = h.dataH;
  out->fft_w = h.fftW;
  out->fft_h = h.fftH;
  out->margin = h.off;
  return BIMP_OK;
}

static int ctx_run(bimp_context* c, const uint8_t* image, size_t pitch, int width, int height,
                   cudaMemcpyKind kind, float* d_kp, size_t ld, int capacity, int* d_count,
                   cudaStream_t s, int aos = 0) {
  if (!c || !image) return fail(BIMP_ERR_INVALID, "null argument");
  if (width != c->inWidth || height != c->inHeight)
    return fail(BIMP_ERR_INVALID, "image size differs from the context's");
  if (pitch < (size_t)width) return fail(BIMP_ERR_INVALID, "pitch smaller than width");
  if (capacity < 0) return fail(BIMP_ERR_INVALID, "negative capacity");
  if (capacity > 0 && (!d_kp || ld < (size_t)capacity)) return fail(BIMP_ERR_INVALID, "bad keypoint matrix");
  BIMP_CUDA(cudaSetDevice(c->eng.device));
  Engine& e = c->eng;
  BIMP_CUDA(cudaMemcpy2DAsync(e.lvl[0][0], e.lvlP[0][0], image, pitch, width, height, kind, s));
  KpOut o;
  o.kp = d_kp;
  o.ld = ld;
  o.capacity = capacity;
  o.aos = aos;
  // the NMS writes the keypoint total to d_count itself when the image has
  // candidate rows (otherwise the total stays 0 and is copied below)
  o.count = e.nNmsCtas > 0 ? d_count : nullptr;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  BIMP_CUDA(cudaStreamIsCapturing(s, &cap));
  // the destination descriptor: rewritten when it changes, and always when
  // the caller's stream is being captured (a replay must not depend on
  // what later calls leave in the device copy)
  if (cap != cudaStreamCaptureStatusNone) c->captured = true;
  if (c->captured || !c->outSet || std::memcmp(&o, &c->lastOut, sizeof(o)) != 0) {
    launch_set_out(e.d_outs, o, s);
    BIMP_CUDA(cudaGetLastError());
    c->lastOut = o;
    c->outSet = true;
  }
  // the captured sequence, unless the caller's stream is itself being
  // captured (then the kernels go straight into the caller's capture)
  if (c->exec && cap == cudaStreamCaptureStatusNone) {
    BIMP_CUDA(cudaGraphLaunch(c->exec, s));
  } else {
    const int rc = e.enqueue(s);
    if (rc != BIMP_OK) return rc;
  }
  if (d_count && !o.count)
    BIMP_CUDA(cudaMemcpyAsync(d_count, e.d_totals, sizeof(int), cudaMemcpyDeviceToDevice, s));
  return BIMP_OK;
}

int bimp_detect_device_async(bimp_context* c, const uint8_t* d_image, size_t pitch, int width,
                             int height, float* d_kp, size_t ld, int capacity, int* d_count,
                             void* stream) {
  return ctx_run(c, d_image, pitch, width, height, cudaMemcpyDeviceToDevice, d_kp, ld, capacity,
                 d_count, static_cast<cudaStream_t>(stream));
}

int bimp_detect_device(bimp_context* c, const uint8_t* d_image, size_t pitch, int width, int height,
                       float* d_kp, size_t ld, int capacity, int* n_found, void* stream) {
  if (!n_found) return fail(BIMP_ERR_INVALID, "n_found is null");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc = ctx_run(c, d_image, pitch, width, height, cudaMemcpyDeviceToDevice, d_kp, ld, capacity,
                   nullptr, s);
  if (rc != BIMP_OK) return rc;
  BIMP_CUDA(cudaMemcpyAsync(c->h_count, c->eng.d_totals, sizeof(int), cudaMemcpyDeviceToHost, s));
  BIMP_CUDA(cudaMemcpyAsync(c->h_count + 1, c->eng.d_fault, sizeof(int), cudaMemcpyDeviceToHost, s));
  BIMP_CUDA(cudaStreamSynchronize(s));
  *n_found = *c->h_count;
  if (c->h_count[1]) return fail(BIMP_ERR_CUDA, "a bounded device wait expired in the tile kernel");
  if (*n_found > capacity)
    return fail(BIMP_ERR_CAPACITY, "keypoints exceed capacity (" + std::to_string(*n_found) + ")");
  return BIMP_OK;
}

static int ensure_host_buffers(bimp_context* c, int capacity) {
  if (c->d_kpScratchCap < capacity) {
    if (c->d_kpScratch) cudaFree(c->d_kpScratch);
    c->d_kpScratch = nullptr;
    c->d_kpScratchCap = 0;
    BIMP_CUDA(cudaMalloc(&c->d_kpScratch, sizeof(float) * BIMP_KP_VECTOR_LENGTH * (size_t)capacity));
    c->d_kpScratchCap = capacity;
  }
  if (c->h_stageCap < capacity) {
    if (c->h_stage) cudaFreeHost(c->h_stage);
    c->h_stage = nullptr;
    c->h_stageCap = 0;
    BIMP_CUDA(cudaMallocHost(&c->h_stage, sizeof(bimp_keypoint) * (size_t)capacity));
    c->h_stageCap = capacity;
  }
  return BIMP_OK;
}

// Host path, first half: the image copy, the detection (records written as
// cv::KeyPoint-layout structs into the device scratch), and the copies back
// of the count, the fault word and the first *spec records into the pinned
// staging, all on stream s.  Nothing waits.
static int host_enqueue(bimp_context* c, const uint8_t* image, size_t pitch, int width, int height, int capacity,
                        cudaStream_t s, int* spec) {
  BIMP_CUDA(cudaSetDevice(c->eng.device));
  const int cap = std::max(capacity, 1);
  int rc = ensure_host_buffers(c, cap);
  if (rc != BIMP_OK) return rc;
  rc = ctx_run(c, image, pitch, width, height, cudaMemcpyHostToDevice, c->d_kpScratch, cap, capacity, nullptr, s, 1);
  if (rc != BIMP_OK) return rc;
  BIMP_CUDA(cudaMemcpyAsync(c->h_count, c->eng.d_totals, sizeof(int), cudaMemcpyDeviceToHost, s));
  BIMP_CUDA(cudaMemcpyAsync(c->h_count + 1, c->eng.d_fault, sizeof(int), cudaMemcpyDeviceToHost, s));
  *spec = std::min(capacity, c->specRecords);
  if (*spec > 0)
    BIMP_CUDA(cudaMemcpyAsync(c->h_stage, c->d_kpScratch, sizeof(bimp_keypoint) * (size_t)*spec,
                              cudaMemcpyDeviceToHost, s));
  return BIMP_OK;
}

// Host path, second half, once stream s has finished the first: the records
// beyond the speculative copy (rare: a count well above the previous call's)
// come back with one more copy and synchronisation, then everything is
// copied from the staging into the caller's array.
static int host_finish(bimp_context* c, int spec, bimp_keypoint* out, int capacity, int* n_found, cudaStream_t s) {
  const int total = c->h_count[0];
  *n_found = total;
  if (c->h_count[1]) return fail(BIMP_ERR_CUDA, "a bounded device wait expired");
  const int n = std::min(total, capacity);
  if (n > spec) {
    BIMP_CUDA(cudaMemcpyAsync(c->h_stage + spec, reinterpret_cast<const bimp_keypoint*>(c->d_kpScratch) + spec,
                              sizeof(bimp_keypoint) * (size_t)(n - spec), cudaMemcpyDeviceToHost, s));
    BIMP_CUDA(cudaStreamSynchronize(s));
  }
  static_assert(sizeof(bimp_keypoint) == 7 * sizeof(float), "record layout");
  if (n > 0) std::memcpy(out, c->h_stage, sizeof(bimp_keypoint) * (size_t)n);
  c->specRecords = std::max(256, std::min(std::max(capacity, 1), n + n / 8 + 256));
  if (total > capacity)
    return fail(BIMP_ERR_CAPACITY, "keypoints exceed capacity (" + std::to_string(total) + ")");
  return BIMP_OK;
}

int bimp_detect_host(bimp_context* c, const uint8_t* image, size_t pitch, int width, int height,
                     bimp_keypoint* out, int capacity, int* n_found, void* stream) {
  if (!c || !n_found || capacity < 0 || (capacity > 0 && !out))
    return fail(BIMP_ERR_INVALID, "null argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int spec = 0;
  const int rc = host_enqueue(c, image, pitch, width, height, capacity, s, &spec);
  if (rc != BIMP_OK) return rc;
  BIMP_CUDA(cudaStreamSynchronize(s));
  return host_finish(c, spec, out, capacity, n_found, s);
}

int bimp_dense_map(bimp_context* c, int scale, int which, float* d_out, size_t ld, void* stream) {
  if (!c || !d_out || scale < 0 || scale >= c->eng.nScales || which < 0 || which > 1)
    return fail(BIMP_ERR_INVALID, "bad dense-map arguments");
  const ScaleDev& d = c->eng.h_sd[scale];
  if (ld < (size_t)d.dataW) return fail(BIMP_ERR_INVALID, "ld smaller than data width");
  BIMP_CUDA(cudaSetDevice(c->eng.device));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (which == 1) {
    // S is not on the keypoint path: detection writes D only, and the
    // single-stopped map is computed here from the last detection's complex
    // cells (the same stencil pass, which rewrites D with identical values)
    if (c->eng.nSten > 0)
      launch_stencil(c->eng.d_sd, c->eng.d_sten, c->eng.nSten, c->eng.d_fault, s, kStencilDS);
    BIMP_CUDA(cudaGetLastError());
  }
  const float* src = which == 0 ? d.D : d.S;
  BIMP_CUDA(cudaMemcpy2DAsync(d_out, ld * sizeof(float), src, d.dPitch * sizeof(float),
                              d.dataW * sizeof(float), d.dataH, cudaMemcpyDeviceToDevice, s));
  return BIMP_OK;
}

int bimp_detect_lines_edges(bimp_context* c, int scale, const float* d_ch, size_t ch_ld, float* d_result,
                            float* d_ori, int8_t* d_type, size_t ld, void* stream) {
  if (!c || scale < 0 || scale >= c->eng.nScales || !d_result || !d_ori || !d_type)
    return fail(BIMP_ERR_INVALID, "bad line/edge arguments");
  const Engine& e = c->eng;
  ScaleDev d = e.h_sd[scale];
  if (ld < (size_t)d.dataW || (d_ch && ch_ld < (size_t)d.dataW))
    return fail(BIMP_ERR_INVALID, "ld smaller than data width");
  BIMP_CUDA(cudaSetDevice(e.device));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (!c->d_leZ) {   // sized for the largest scale
    long long maxStride = 0;
    int maxTiles = 0;
    for (const ScaleDev& q : e.h_sd) {
      maxStride = std::max(maxStride, q.cStride);
      maxTiles = std::max(maxTiles, q.tilesX * q.tilesY);
    }
    BIMP_CUDA(cudaMalloc(&c->d_leZ, sizeof(float2) * kNumOri * (size_t)maxStride));
    BIMP_CUDA(cudaMalloc(&c->d_leSd, sizeof(ScaleDev)));
    BIMP_CUDA(cudaMalloc(&c->d_leTiles, sizeof(TileWork) * (size_t)std::max(1, maxTiles)));
  }
  // rerun this scale's tile FFT keeping e + i o (the magnitudes it rewrites
  // are the same numbers)
  d.Z = c->d_leZ;
  std::vector<TileWork> tiles;
  for (int k = 0; k < d.tilesX * d.tilesY; ++k) tiles.push_back({0, k});
  BIMP_CUDA(cudaMemcpyAsync(c->d_leSd, &d, sizeof(ScaleDev), cudaMemcpyHostToDevice, s));
  BIMP_CUDA(cudaMemcpyAsync(c->d_leTiles, tiles.data(), sizeof(TileWork) * tiles.size(), cudaMemcpyHostToDevice, s));
  launch_gabor_keep_z(c->d_leSd, c->d_leTiles, static_cast<int>(tiles.size()), e.d_fault, s);
  launch_detect_le(c->d_leSd, d.dataW, d.dataH, d_ch, static_cast<int>(ch_ld), d_result, d_ori, d_type,
                   static_cast<int>(ld), s);
  BIMP_CUDA(cudaGetLastError());
  // the host copies above read stack memory: finish before returning
  BIMP_CUDA(cudaStreamSynchronize(s));
  return BIMP_OK;
}

int bimp_complex_map(bimp_context* c, int scale, int o, float* d_out, size_t ld, void* stream) {
  if (!c || !d_out || scale < 0 || scale >= c->eng.nScales || o < 0 || o >= kNumOri)
    return fail(BIMP_ERR_INVALID, "bad complex-map arguments");
  const ScaleDev& d = c->eng.h_sd[scale];
  if (ld < (size_t)d.cCols) return fail(BIMP_ERR_INVALID, "ld smaller than data width + 1");
  BIMP_CUDA(cudaSetDevice(c->eng.device));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const float* src = d.C + (size_t)o * d.cStride;
  BIMP_CUDA(cudaMemcpy2DAsync(d_out, ld * sizeof(float), src, d.cPitch * sizeof(float),
                              d.cCols * sizeof(float), d.dataH + 1, cudaMemcpyDeviceToDevice, s));
  return BIMP_OK;
}

int bimp_ctx_kernel_launches(const bimp_context* c) { return c ? c->eng.kernel_launches() : 0; }

int bimp_ctx_run_stage(bimp_context* c, int stage, void* stream) {
  if (!c) return fail(BIMP_ERR_INVALID, "ctx is null");
  BIMP_CUDA(cudaSetDevice(c->eng.device));
  return c->eng.stage(stage, static_cast<cudaStream_t>(stream));
}

int bimp_download_keypoints(const float* d_kp, size_t ld, int n, bimp_keypoint* out, void* stream) {
  if (n < 0 || (n > 0 && (!d_kp || !out || ld < (size_t)n)))
    return fail(BIMP_ERR_INVALID, "bad download arguments");
  if (n == 0) return BIMP_OK;
  std::vector<float> h((size_t)BIMP_KP_VECTOR_LENGTH * n);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  BIMP_CUDA(cudaMemcpy2DAsync(h.data(), sizeof(float) * n, d_kp, sizeof(float) * ld, sizeof(float) * n,
                              BIMP_KP_VECTOR_LENGTH, cudaMemcpyDeviceToHost, s));
  BIMP_CUDA(cudaStreamSynchronize(s));
  for (int j = 0; j < n; ++j) {
    bimp_keypoint& k = out[j];
    k.x = h[BIMP_X_ROW * n + j];
    k.y = h[BIMP_Y_ROW * n + j];
    std::memcpy(&k.class_id, &h[BIMP_LAPLACIAN_ROW * n + j], 4);
    std::memcpy(&k.octave, &h[BIMP_OCTAVE_ROW * n + j], 4);
    k.size = h[BIMP_SIZE_ROW * n + j];
    k.angle = h[BIMP_ANGLE_ROW * n + j];
    k.response = h[BIMP_HESSIAN_ROW * n + j];
  }
  return BIMP_OK;
}

int bimp_upload_keypoints(const bimp_keypoint* kps, int n, float* d_kp, size_t ld, void* stream) {
  if (n < 0 || (n > 0 && (!kps || !d_kp || ld < (size_t)n)))
    return fail(BIMP_ERR_INVALID, "bad upload arguments");
  if (n == 0) return BIMP_OK;
  std::vector<float> h((size_t)BIMP_KP_VECTOR_LENGTH * n);
  for (int j = 0; j < n; ++j) {
    const bimp_keypoint& k = kps[j];
    h[BIMP_X_ROW * n + j] = k.x;
    h[BIMP_Y_ROW * n + j] = k.y;
    h[BIMP_SIZE_ROW * n + j] = k.size;
    h[BIMP_ANGLE_ROW * n + j] = k.angle;
    h[BIMP_HESSIAN_ROW * n + j] = k.response;
    std::memcpy(&h[BIMP_OCTAVE_ROW * n + j], &k.octave, 4);
    const int one = 1;   // utils.cpp:126 writes LAPLACIAN = 1
    std::memcpy(&h[BIMP_LAPLACIAN_ROW * n + j], &one, 4);
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  BIMP_CUDA(cudaMemcpy2DAsync(d_kp, sizeof(float) * ld, h.data(), sizeof(float) * n, sizeof(float) * n,
                              BIMP_KP_VECTOR_LENGTH, cudaMemcpyHostToDevice, s));
  BIMP_CUDA(cudaStreamSynchronize(s));
  return BIMP_OK;
}

// ---------------------------------------------------------------------------
// batches
// ---------------------------------------------------------------------------
int bimp_batch_create(bimp_batch** out, const int* widths, const int* heights, int n_images,
                      const float* lambdas, int n_lambdas, const bimp_params* params, int kp_capacity) {
  if (!out) return fail(BIMP_ERR_INVALID, "batch is null");
  *out = nullptr;
  if (!widths || !heights || n_images <= 0 || !lambdas || n_lambdas <= 0 || kp_capacity <= 0)
    return fail(BIMP_ERR_INVALID, "bad batch arguments");
  int dev = 0;
  BIMP_CUDA(cudaGetDevice(&dev));
  int rc = ensure_device_configured(dev);
  if (rc != BIMP_OK) return rc;
  bimp_batch* b = new bimp_batch();
  const bimp_params p = params ? *params : default_params();
  rc = b->eng.build(dev, widths, heights, n_images, lambdas, n_lambdas, p, kp_capacity);
  if (rc != BIMP_OK) {
    b->eng.release();
    delete b;
    return rc;
  }
  cudaError_t e = cudaMallocHost(&b->h_totals, sizeof(int) * (n_images + 1));
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->capStream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    const std::string msg = std::string("batch setup: ") + cudaGetErrorString(e);
    bimp_batch_destroy(b);
    return fail(BIMP_ERR_CUDA, msg);
  }
  rc = capture_batch(b);
  if (rc != BIMP_OK) {
    const std::string msg = g_last_error;
    bimp_batch_destroy(b);
    return fail(rc, msg);
  }
  *out = b;
  return BIMP_OK;
}

int bimp_batch_destroy(bimp_batch* b) {
  if (!b) return BIMP_OK;
  cudaSetDevice(b->eng.device);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->capStream) cudaStreamDestroy(b->capStream);
  if (b->h_totals) cudaFreeHost(b->h_totals);
  b->eng.release();
  delete b;
  return BIMP_OK;
}

int bimp_batch_num_images(const bimp_batch* b) { return b ? b->eng.nImages : 0; }

int bimp_batch_image(bimp_batch* b, int i, uint8_t** d_image, size_t* pitch) {
  if (!b || i < 0 || i >= b->eng.nImages || !d_image || !pitch)
    return fail(BIMP_ERR_INVALID, "bad batch image arguments");
  *d_image = b->eng.lvl[i][0];
  *pitch = (size_t)b->eng.lvlP[i][0];
  return BIMP_OK;
}

int bimp_batch_set_tile_plan(bimp_batch* b, int policy, int order, int grid, int kernel) {
  if (!b || policy < 0 || policy > 1 || order < 0 || order > 1 || kernel < 0 || kernel > 1)
    return fail(BIMP_ERR_INVALID, "bad tile plan");
  BIMP_CUDA(cudaSetDevice(b->eng.device));
  const int rc = b->eng.retile(policy, order, grid, kernel);
  if (rc != BIMP_OK) return rc;
  return capture_batch(b);
}

int bimp_batch_autotune(bimp_batch* b, void* stream, int reps, bimp_tile_plan* chosen, bimp_tile_plan* tried,
                        int max_tried, int* n_tried) {
  if (!b || reps <= 0 || (max_tried > 0 && !tried)) return fail(BIMP_ERR_INVALID, "bad autotune arguments");
  BIMP_CUDA(cudaSetDevice(b->eng.device));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int sms = 148;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->eng.device) != cudaSuccess || sms <= 0)
    sms = 148;
  const int grids[3] = {0, sms, 2 * sms};
  // the pipelined kernel takes every scale only when its valid blocks fit
  const int kernels = b->eng.pipelined_fits() ? 2 : 1;
  cudaEvent_t e0, e1;
  BIMP_CUDA(cudaEventCreate(&e0));
  BIMP_CUDA(cudaEventCreate(&e1));
  bimp_tile_plan best{};
  best.ms = -1.f;
  int count = 0, rc = BIMP_OK;
  for (int kernel = kernels - 1; kernel >= 0 && rc == BIMP_OK; --kernel)
    for (int policy = 0; policy < 2 && rc == BIMP_OK; ++policy)
      for (int order = 0; order < 2 && rc == BIMP_OK; ++order)
        for (int g = 0; g < 3 && rc == BIMP_OK; ++g) {
          rc = b->eng.retile(policy, order, grids[g], kernel);
          for (int i = 0; i < 2 && rc == BIMP_OK; ++i) rc = b->eng.enqueue(s);
          if (rc != BIMP_OK) break;
          cudaEventRecord(e0, s);
          for (int i = 0; i < reps && rc == BIMP_OK; ++i) rc = b->eng.enqueue(s);
          cudaEventRecord(e1, s);
          if (rc != BIMP_OK) break;
          if (cudaEventSynchronize(e1) != cudaSuccess) {
            rc = fail(BIMP_ERR_CUDA, "autotune timing failed");
            break;
          }
          float ms = 0.f;
          cudaEventElapsedTime(&ms, e0, e1);
          const bimp_tile_plan pl{policy, order, b->eng.tilePipelined ? 1 : 0, b->eng.tileGridReq, b->eng.nTiles,
                                  ms / reps};
          if (count < max_tried) tried[count] = pl;
          ++count;
          if (best.ms < 0.f || pl.ms < best.ms) best = pl;
        }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != BIMP_OK) return rc;
  rc = b->eng.retile(best.policy, best.order, best.grid, best.kernel);
  if (rc == BIMP_OK) rc = capture_batch(b);
  if (rc != BIMP_OK) return rc;
  if (chosen) *chosen = best;
  if (n_tried) *n_tried = count;
  return BIMP_OK;
}

int bimp_batch_run(bimp_batch* b, void* stream) {
  if (!b) return fail(BIMP_ERR_INVALID, "batch is null");
  BIMP_CUDA(cudaSetDevice(b->eng.device));
  BIMP_CUDA(cudaGraphLaunch(b->exec, static_cast<cudaStream_t>(stream)));
  return BIMP_OK;
}

int bimp_batch_counts(bimp_batch* b, int* d_counts, void* stream) {
  if (!b || !d_counts) return fail(BIMP_ERR_INVALID, "bad batch count arguments");
  BIMP_CUDA(cudaMemcpyAsync(d_counts, b->eng.d_totals, sizeof(int) * b->eng.nImages,
                            cudaMemcpyDeviceToDevice, static_cast<cudaStream_t>(stream)));
  return BIMP_OK;
}

int bimp_batch_scale_info(const bimp_batch* b, int i, int scale, bimp_scale_info* out) {
  if (!b || !out || i < 0 || i >= b->eng.nImages || scale < 0 || scale >= b->eng.nScales)
    return fail(BIMP_ERR_INVALID, "bad batch scale index");
  const ScaleHost& h = b->eng.geo[i][scale];
  out->lambda_full = h.lambda2;
  out->lambda_level = h.lambda;
  out->pyrstep = h.pyrstep;
  out->kernel_w = h.kW;
  out->kernel_x = h.kX;
  out->data_w = h.dataW;
  out->data_h = h.dataH;
  out->fft_w = h.fftW;
  out->fft_h = h.fftH;
  out->margin = h.off;
  return BIMP_OK;
}

int bimp_batch_dense_map(bimp_batch* b, int i, int scale, float* d_out, size_t ld, void* stream) {
  if (!b || !d_out || i < 0 || i >= b->eng.nImages || scale < 0 || scale >= b->eng.nScales)
    return fail(BIMP_ERR_INVALID, "bad batch dense-map arguments");
  const ScaleDev& d = b->eng.h_sd[(size_t)i * b->eng.nScales + scale];
  if (ld < (size_t)d.dataW) return fail(BIMP_ERR_INVALID, "ld smaller than data width");
  BIMP_CUDA(cudaSetDevice(b->eng.device));
  BIMP_CUDA(cudaMemcpy2DAsync(d_out, ld * sizeof(float), d.D, d.dPitch * sizeof(float), d.dataW * sizeof(float),
                              d.dataH, cudaMemcpyDeviceToDevice, static_cast<cudaStream_t>(stream)));
  return BIMP_OK;
}

int bimp_batch_keypoints_device(bimp_batch* b, int i, const float** d_kp, size_t* ld) {
  if (!b || i < 0 || i >= b->eng.nImages || !d_kp || !ld)
    return fail(BIMP_ERR_INVALID, "bad batch keypoint arguments");
  *d_kp = b->eng.d_kpInternal + (size_t)i * BIMP_KP_VECTOR_LENGTH * b->eng.kpCapInternal;
  *ld = (size_t)b->eng.kpCapInternal;
  return BIMP_OK;
}

int bimp_batch_detect_host(bimp_batch* b, const uint8_t* const* images, const size_t* pitches,
                           bimp_keypoint* const* outs, const int* capacities, int* n_found,
                           void* stream) {
  if (!b || !images || !pitches || !n_found) return fail(BIMP_ERR_INVALID, "bad batch arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Engine& e = b->eng;
  BIMP_CUDA(cudaSetDevice(e.device));
  for (int i = 0; i < e.nImages; ++i) {
    if (!images[i]) return fail(BIMP_ERR_INVALID, "null image");
    BIMP_CUDA(cudaMemcpy2DAsync(e.lvl[i][0], e.lvlP[i][0], images[i], pitches[i], e.widths[i],
                                e.heights[i], cudaMemcpyHostToDevice, s));
  }
  BIMP_CUDA(cudaGraphLaunch(b->exec, s));
  BIMP_CUDA(cudaMemcpyAsync(b->h_totals, e.d_totals, sizeof(int) * e.nImages, cudaMemcpyDeviceToHost, s));
  BIMP_CUDA(cudaMemcpyAsync(b->h_totals + e.nImages, e.d_fault, sizeof(int), cudaMemcpyDeviceToHost, s));
  BIMP_CUDA(cudaStreamSynchronize(s));
  if (b->h_totals[e.nImages]) return fail(BIMP_ERR_CUDA, "a bounded device wait expired in the tile kernel");
  int status = BIMP_OK;
  for (int i = 0; i < e.nImages; ++i) {
    n_found[i] = b->h_totals[i];
    const int cap = std::min(capacities ? capacities[i] : 0, e.kpCapInternal);
    const int n = std::min(n_found[i], cap);
    if (n_found[i] > cap) status = BIMP_ERR_CAPACITY;
    if (n > 0 && outs && outs[i]) {
      const float* dk = e.d_kpInternal + (size_t)i * BIMP_KP_VECTOR_LENGTH * e.kpCapInternal;
      const int rc = bimp_download_keypoints(dk, e.kpCapInternal, n, outs[i], stream);
      if (rc != BIMP_OK) return rc;
    }
  }
  if (status != BIMP_OK) return fail(status, "keypoints exceed capacity for some image");
  return BIMP_OK;
}

// ---------------------------------------------------------------------------
// pipelined host frames
// ---------------------------------------------------------------------------
int bimp_pipeline_destroy(bimp_pipeline* p) {
  if (!p) return BIMP_OK;
  cudaSetDevice(p->device);
  for (cudaStream_t st : p->streams)
    if (st) cudaStreamSynchronize(st);
  for (bimp_context* c : p->ctx) bimp_ctx_destroy(c);
  for (cudaStream_t st : p->streams)
    if (st) cudaStreamDestroy(st);
  for (cudaEvent_t ev : p->done)
    if (ev) cudaEventDestroy(ev);
  delete p;
  return BIMP_OK;
}

int bimp_pipeline_create(bimp_pipeline** out, int width, int height, const float* lambdas, int n_lambdas,
                         const bimp_params* params, int depth, int capacity) {
  if (!out) return fail(BIMP_ERR_INVALID, "pipeline is null");
  *out = nullptr;
  if (depth < 1 || depth > 8 || capacity < 1) return fail(BIMP_ERR_INVALID, "depth must be 1..8, capacity >= 1");
  bimp_pipeline* p = new bimp_pipeline();
  cudaGetDevice(&p->device);
  p->depth = depth;
  p->capacity = capacity;
  p->ctx.assign(depth, nullptr);
  p->streams.assign(depth, nullptr);
  p->done.assign(depth, nullptr);
  p->spec.assign(depth, 0);
  for (int k = 0; k < depth; ++k) {
    int rc = bimp_ctx_create(&p->ctx[k], width, height, lambdas, n_lambdas, params);
    if (rc == BIMP_OK) rc = ensure_host_buffers(p->ctx[k], capacity);
    cudaError_t e = cudaSuccess;
    if (rc == BIMP_OK) e = cudaStreamCreateWithFlags(&p->streams[k], cudaStreamNonBlocking);
    if (rc == BIMP_OK && e == cudaSuccess) e = cudaEventCreateWithFlags(&p->done[k], cudaEventDisableTiming);
    if (rc == BIMP_OK && e != cudaSuccess) rc = fail(BIMP_ERR_CUDA, std::string("pipeline setup: ") + cudaGetErrorString(e));
    if (rc != BIMP_OK) {
      const std::string msg = g_last_error;
      bimp_pipeline_destroy(p);
      return fail(rc, msg);
    }
  }
  *out = p;
  return BIMP_OK;
}

int bimp_pipeline_in_flight(const bimp_pipeline* p) { return p ? p->inFlight : 0; }

int bimp_pipeline_push(bimp_pipeline* p, const uint8_t* image, size_t pitch, int width, int height) {
  if (!p || !image) return fail(BIMP_ERR_INVALID, "null argument");
  if (p->inFlight == p->depth) return fail(BIMP_ERR_INVALID, "pipeline full: pop a frame first");
  const int k = (p->head + p->inFlight) % p->depth;
  int rc = host_enqueue(p->ctx[k], image, pitch, width, height, p->capacity, p->streams[k], &p->spec[k]);
  if (rc != BIMP_OK) return rc;
  BIMP_CUDA(cudaEventRecord(p->done[k], p->streams[k]));
  ++p->inFlight;
  return BIMP_OK;
}

int bimp_pipeline_pop(bimp_pipeline* p, bimp_keypoint* out, int capacity, int* n_found) {
  if (!p || !n_found || capacity < 0 || (capacity > 0 && !out)) return fail(BIMP_ERR_INVALID, "null argument");
  if (p->inFlight == 0) return fail(BIMP_ERR_INVALID, "no frame in flight");
  const int k = p->head;
  p->head = (p->head + 1) % p->depth;
  --p->inFlight;
  BIMP_CUDA(cudaSetDevice(p->device));
  BIMP_CUDA(cudaEventSynchronize(p->done[k]));
  int total = 0;
  const int rc = host_finish(p->ctx[k], p->spec[k], out, std::min(capacity, p->capacity), &total, p->streams[k]);
  *n_found = total;
  if (rc == BIMP_ERR_CAPACITY && total <= capacity) {
    // more than the pipeline's own capacity was found: the records beyond it
    // were never written
    return fail(BIMP_ERR_CAPACITY, "keypoints exceed the pipeline capacity (" + std::to_string(total) + ")");
  }
  return rc;
}

// ---------------------------------------------------------------------------
// device memory helpers (for callers without the CUDA runtime headers)
// ---------------------------------------------------------------------------
int bimp_device_alloc(void** ptr, size_t bytes) {
  if (!ptr) return fail(BIMP_ERR_INVALID, "ptr is null");
  *ptr = nullptr;
  if (bytes == 0) return BIMP_OK;
  BIMP_CUDA(cudaMalloc(ptr, bytes));
  return BIMP_OK;
}

int bimp_device_free(void* ptr) {
  if (ptr) BIMP_CUDA(cudaFree(ptr));
  return BIMP_OK;
}

int bimp_copy_2d(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width_bytes, size_t rows,
                 void* stream) {
  if (rows == 0 || width_bytes == 0) return BIMP_OK;
  if (!dst || !src || dpitch < width_bytes || spitch < width_bytes) return fail(BIMP_ERR_INVALID, "bad copy arguments");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  BIMP_CUDA(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width_bytes, rows, cudaMemcpyDefault, s));
  BIMP_CUDA(cudaStreamSynchronize(s));
  return BIMP_OK;
}

}  // extern "C"

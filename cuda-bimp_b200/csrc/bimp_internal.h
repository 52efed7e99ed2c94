// Internal structures shared by the host bank builder, the kernels and the
// C ABI.  Not part of the public interface.
#pragma once

#include <vector_types.h>   // float2, int2 (CUDA headers, also for the host compiler)

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "bimp_b200.h"

namespace bimp_b200 {

constexpr int kNumOri = 8;
// Overlap-save tile: 128 x 128 complex FFT held in shared memory.
constexpr int kTile = 128;
constexpr int kXhCols = 65;                // Hermitian half: kx = 0..64
constexpr int kTileThreads = 512;
constexpr int kMaxHalf = 56;               // largest supported kernel half size
constexpr int kSpecFloats = kTile * kTile; // one orientation's real spectrum
constexpr int kSpecHalf = kTile * kXhCols;  // Hermitian half of a tile spectrum
// Forward stencil blocks: 32 columns x kStencilBlockH rows of D per block
// (the host's block lists and the kernel share this).
constexpr int kStencilBlockH = 32;

// Per (image, scale) descriptor read by every kernel.  Plain old data.
struct ScaleDev {
  // geometry (cuda_bimp.cu:249-256)
  int dataW, dataH, fftW, fftH;
  int kX;          // kernel half size == kernelX == kernelY
  int V;           // valid outputs per tile side = kTile - 2*kX
  int tilesX, tilesY;
  int cRows, cCols;  // complex-cell window stored: (dataH+2) x (dataW+1)
  int wrapW;         // fftW == dataW: column dataW reads the next row's column 0
  // level image (uint8, full pyrDown size lvlW x lvlH)
  const uint8_t* lvl;
  int lvlPitch, lvlW, lvlH;
  // real tile spectra, kNumOri x kTile x kTile floats in (py, px) order
  const float* G;
  // complex-cell maps: kNumOri maps, each cRows x cPitch floats
  float* C;
  int cPitch;
  long long cStride;
  const void* cMap;       // 3-D TMA tensor map of C (device memory, 128 B)
  // stencil offsets (cuda_bimp.cu:533-550)
  int es1[kNumOri], es2[kNumOri];   // end-stop (row, col)
  int in1[kNumOri], in2[kNumOri];   // inhibition (row, col)
  int ih1[kNumOri], ih2[kNumOri];   // radial half offsets round(0.5*in)
  float radialGain, wTan, wRad;
  // dense maps: dataH x dPitch floats
  float* D;
  float* S;
  int dPitch;
  unsigned int* maxKey;   // order-preserving key of max(D)
  // keypoints (cuda_bimp.cu:737-740)
  int off;                // (int)lambda
  float pyrstep;
  float kpSize;           // lambda*pyrstep
  int kpOctave;           // (int)(lambda*pyrstep)
  double threshRatio;     // double, as the reference multiplies max by the literal 0.104
  int rowBase;            // first entry of this scale in the per-row count array
  unsigned int* nmsMask;  // keypoint decisions per candidate row, nmsChunks words of 32 pixels (or null)
  int nmsChunks;
  int image;              // image index inside a batch
  int pattern;            // stencil offsets: 0 = runtime, k > 0 = kOffsetSets[k-1]
  // differentiable path (float pyramid, saved responses, adjoint buffers)
  const float* lvlF;      // float level (X scale), lvlPitchF floats per row
  int lvlPitchF;
  float2* Z;              // saved e + i o, C layout in float2
  const float* M;         // loss weights, dataH x dataW (row pitch dataW)
  float* gC;              // d loss / d complex cell, C layout
  float* gWrap;           // fftW == dataW: d loss / d window (r, dataW), kNumOri x (dataH + 1)
  float* gLvl;            // d loss / d float level, lvlPitchF floats per row
  float* T;               // tangential inhibition map, dataH x dPitch
  float* R;               // radial inhibition map, dataH x dPitch
  unsigned int* bits;     // ReLU states, 4 bits per orientation, dataH x dPitch
  const float4* bwA;      // per orientation, kSpecHalf entries {G(k), G(-k), dGa(k), dGr(k)}
  const float2* bwB;      //   {dGa(-k), dGr(-k)}; dG* = spectra of d taps / d alpha, d rho
};

// Stencil offset sets of the two level wavelengths the default bank uses
// (lambda ~ 4 and ~ 5.657 at every pyramid level); scales whose offsets equal
// one of them run a kernel specialised with compile-time offsets.
// Layout per set: es1[8], es2[8], in1[8], in2[8], ih1[8], ih2[8].
constexpr int kNumOffsetSets = 2;
#define BIMP_OFFSET_SETS                                   \
  {                                                        \
    {{2, 2, 2, 1, 0, -1, -2, -2}, {0, 1, 2, 2, 2, 2, 2, 1}, \
     {0, 1, 2, 2, 2, 2, 2, 1}, {2, 2, 2, 1, 0, -1, -2, -2}, \
     {0, 1, 1, 1, 1, 1, 1, 1}, {1, 1, 1, 1, 0, -1, -1, -1}},\
    {{3, 3, 2, 1, 0, -1, -2, -3}, {0, 1, 2, 3, 3, 3, 2, 1}, \
     {0, 1, 2, 3, 3, 3, 2, 1}, {3, 3, 2, 1, 0, -1, -2, -3}, \
     {0, 1, 1, 2, 2, 2, 1, 1}, {2, 2, 1, 1, 0, -1, -1, -2}} \
  }
constexpr int kOffsetSets[kNumOffsetSets][6][8] = BIMP_OFFSET_SETS;

// One unit of tiled-FFT work: orientations [oBegin, oEnd) of tile `tile` of
// descriptor `entry`.  oBegin == oEnd is an empty slot of a padded plan.
struct TileWork {
  int entry;
  int tile;
  int oBegin = 0;
  int oEnd = kNumOri;
};

// Host-side description of one scale (geometry + bank).
struct ScaleHost {
  float lambda2, lambda, pyrstep, filtersize;
  int kW, kX, dataW, dataH, fftW, fftH, level, off;
  int es1[kNumOri], es2[kNumOri], in1[kNumOri], in2[kNumOri];
  std::vector<float> even[kNumOri], odd[kNumOri];   // kW x kW taps
  std::vector<float> spectrum;                       // kNumOri x kTile x kTile
};

// Reference-equivalent helpers (bank.cpp).
int snap_transform_size(int n);
std::vector<float> make_lambdas_log(float start, float end, int spo);
std::vector<float> make_lambdas_lin(float start, float end, int n);
bool build_scales(int width, int height, const std::vector<float>& lambdas,
                  const bimp_params& p, std::vector<ScaleHost>& out, std::string& err);
void tile_spectrum(const std::vector<float>* even, const std::vector<float>* odd, int kW, int kX,
                   std::vector<float>& out);
void derivative_taps(const ScaleHost& s, const bimp_params& p, std::vector<float>* de_da, std::vector<float>* do_da,
                     std::vector<float>* de_dr, std::vector<float>* do_dr);

// Sets the message returned by bimp_last_error() on the calling thread.
void record_error(const std::string& msg);
// Sets the kernels' attributes and constants on device `dev` once.
int configure_device(int dev);

// Position of natural frequency k in the digit-permuted 128-point layout.
inline int perm128(int k) { return 8 * (k & 15) + (k >> 4); }

}  // namespace bimp_b200

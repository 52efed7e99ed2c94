// Host-side filter-bank builder: per-scale geometry, Gabor taps and the real
// 128x128 tile spectra consumed by the tiled-FFT kernel.
//
// Geometry and taps follow the CudaStuff constructor of daniel-koudouna/
// cuda-bimp (bimp/src/cuda_bimp.cu:222-331) including its float arithmetic,
// so the taps are the same float32 numbers the reference uploads.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "bimp_internal.h"

namespace bimp_b200 {

// snapTransformSize, bimp/src/cuda_bimp.cu:200-219: align to 16, keep a power
// of two as is, else the next power of two up to 1024, else align to 512.
int snap_transform_size(int n) {
  if (n <= 0) return 0;
  n = (n + 15) / 16 * 16;
  int hi = 31;
  while (hi >= 0 && !(static_cast<unsigned>(n) & (1u << hi))) --hi;
  const unsigned lo = 1u << hi;
  if (lo == static_cast<unsigned>(n)) return n;
  const unsigned up = 1u << (hi + 1);
  if (up <= 1024u) return static_cast<int>(up);
  return (n + 511) / 512 * 512;
}

// makeLambdasLog, bimp/src/cuda_bimp.cu:927-937 (float accumulation, the
// loop bound compared in double).
std::vector<float> make_lambdas_log(float start, float end, int spo) {
  std::vector<float> out;
  if (spo <= 0 || !(start > 0.f)) return out;
  const float mult = static_cast<float>(std::pow(2.0, 1.0 / spo));
  for (float l = start; l <= end * 1.05 && out.size() < 4096; l *= mult) out.push_back(l);
  return out;
}

// makeLambdasLin, bimp/src/cuda_bimp.cu:905-921.
std::vector<float> make_lambdas_lin(float start, float end, int n) {
  std::vector<float> out;
  float step = 1.f;
  if (n > 1) step = (end - start) / (n - 1);
  for (float s = 1; s <= n; s++) out.push_back(start + (s - 1) * step);
  return out;
}

static int round_half_away(double v) {
  return static_cast<int>(v >= 0 ? std::floor(v + 0.5) : -std::floor(-v + 0.5));
}

bool build_scales(int width, int height, const std::vector<float>& lambdas_in,
                  const bimp_params& p, std::vector<ScaleHost>& out, std::string& err) {
  out.clear();
  if (lambdas_in.empty()) { err = "empty wavelength list"; return false; }
  std::vector<float> lambdas(lambdas_in);
  std::sort(lambdas.begin(), lambdas.end());                    // :224
  for (float l2 : lambdas) {
    if (!(l2 > 0.f) || !std::isfinite(l2)) { err = "wavelengths must be positive"; return false; }
    ScaleHost s;
    s.lambda2 = l2;
    float pyr = 1.f;
    while (l2 / pyr >= p.level_max) pyr *= 2;                   // :236-238
    s.pyrstep = pyr;
    s.lambda = l2 / pyr;                                        // :239
    float fs = static_cast<float>(p.size_ratio * static_cast<double>(s.lambda));  // :245
    if (static_cast<int>(fs) % 2 == 0) fs += 1;                 // :246
    s.filtersize = fs;
    s.kX = static_cast<int>(std::floor(fs / 2));                // :249
    s.kW = static_cast<int>(fs);                                // :250
    s.dataH = static_cast<int>(height / pyr);                   // :253
    s.dataW = static_cast<int>(width / pyr);                    // :254
    s.fftH = snap_transform_size(s.dataH);                      // :255
    s.fftW = snap_transform_size(s.dataW);                      // :256
    int lev = 0;
    for (float q = pyr; q > 1.f; q /= 2) ++lev;
    s.level = lev;
    s.off = static_cast<int>(s.lambda);                         // :737
    if (s.dataW < 2 || s.dataH < 2) { err = "image too small for wavelength"; return false; }
    if (s.kX > kMaxHalf || s.kW != 2 * s.kX + 1) {
      err = "Gabor kernel larger than the tile supports"; return false;
    }
    for (int o = 0; o < kNumOri; ++o) {
      const float theta = static_cast<float>(o * M_PI / kNumOri);
      const double c = std::cos(theta), sn = std::sin(theta);
      s.es1[o] = round_half_away(p.offset_ratio * s.lambda * c);   // :535
      s.es2[o] = round_half_away(p.offset_ratio * s.lambda * sn);  // :536
      s.in1[o] = round_half_away(p.offset_ratio * s.lambda * sn);  // :546
      s.in2[o] = round_half_away(p.offset_ratio * s.lambda * c);   // :547
      // the stencil kernel stages an 8-pixel halo: |2*offset| <= 8
      if (std::abs(s.es1[o]) > 4 || std::abs(s.es2[o]) > 4 || std::abs(s.in1[o]) > 4 ||
          std::abs(s.in2[o]) > 4) {
        err = "end-stop/inhibition offset larger than 4 pixels"; return false;
      }
    }
    // Gabor taps, cuda_bimp.cu:241-250 and :304-331 (float arithmetic).
    const float gamma = static_cast<float>(p.gamma);
    const float phi = static_cast<float>(-M_PI / 2);
    const float sigma = static_cast<float>(s.lambda * p.sigma_ratio);
    const float sigmasq = sigma * sigma;
    const int n = s.kW;
    for (int o = 0; o < kNumOri; ++o) {
      const float theta = static_cast<float>(o * M_PI / kNumOri);
      const float st = std::sin(theta), ct = std::cos(theta);
      std::vector<float>& ev = s.even[o];
      std::vector<float>& od = s.odd[o];
      ev.assign(static_cast<size_t>(n) * n, 0.f);
      od.assign(static_cast<size_t>(n) * n, 0.f);
      float evensum = 0;
      for (int row = 0; row < n; ++row) {
        for (int col = 0; col < n; ++col) {
          const int x = col - s.kX, y = row - s.kX;
          const float a = x * ct + y * st;
          const float b = y * ct - x * st;
          const float env = std::exp(-1 / (2 * sigmasq) * (a * a + gamma * b * b));
          const float freq = static_cast<float>(2 * M_PI * a / s.lambda);
          ev[row * n + col] = env * std::cos(freq);
          od[row * n + col] = env * std::cos(freq + phi);
          evensum += ev[row * n + col];
        }
      }
      for (int m = 0; m < n * n; ++m) ev[m] -= evensum / (fs * fs);   // :330-331
    }
    tile_spectrum(s.even, s.odd, s.kW, s.kX, s.spectrum);
    out.push_back(std::move(s));
  }
  return true;
}

// Real spectrum of the complex Gabor kernel q = even + i*odd placed with its
// centre at (0,0) of a 128x128 torus, scaled by 1/128^2:
//   G(k) = Re sum_d q(d) exp(-2 pi i k.d / 128) / 128^2
// The even taps are point-symmetric and the odd taps antisymmetric, so the
// imaginary part is only the float rounding of the taps and is dropped.
// Stored at [o][perm128(ky)][perm128(kx)], the digit-permuted order in which
// the kernel's forward transform leaves the image spectrum.
void tile_spectrum(const std::vector<float>* even, const std::vector<float>* odd, int kW, int kX,
                   std::vector<float>& out) {
  const int T = kTile, n = kW, h = kX;
  std::vector<double> cs(T), sn(T);
  for (int m = 0; m < T; ++m) {
    cs[m] = std::cos(2.0 * M_PI * m / T);
    sn[m] = std::sin(2.0 * M_PI * m / T);
  }
  out.assign(static_cast<size_t>(kNumOri) * T * T, 0.f);
  std::vector<double> rre(static_cast<size_t>(n) * T), rim(static_cast<size_t>(n) * T);
  for (int o = 0; o < kNumOri; ++o) {
    // row transforms: R[row][kx] = sum_dx q[row][dx] e^{-i a kx dx}
    for (int row = 0; row < n; ++row) {
      for (int kx = 0; kx < T; ++kx) {
        double re = 0, im = 0;
        for (int col = 0; col < n; ++col) {
          const double qr = even[o][row * n + col], qi = odd[o][row * n + col];
          const int m = ((kx * (col - h)) % T + T) % T;
          // (qr + i qi)(c - i s)
          re += qr * cs[m] + qi * sn[m];
          im += qi * cs[m] - qr * sn[m];
        }
        rre[row * T + kx] = re;
        rim[row * T + kx] = im;
      }
    }
    for (int ky = 0; ky < T; ++ky) {
      for (int kx = 0; kx < T; ++kx) {
        double re = 0;
        for (int row = 0; row < n; ++row) {
          const int m = ((ky * (row - h)) % T + T) % T;
          re += rre[row * T + kx] * cs[m] + rim[row * T + kx] * sn[m];
        }
        out[(static_cast<size_t>(o) * T + perm128(ky)) * T + perm128(kx)] =
            static_cast<float>(re / (double(T) * T));
      }
    }
  }
}

// Derivatives of the taps with respect to the wavelength scale alpha
// (lambda = alpha * lambda_level, sigma = rho * lambda, filtersize =
// size_ratio * lambda + its frozen odd-size increment) and to rho, at the
// nominal point alpha = 1, rho = sigma_ratio, from the Gabor formula of
// bimp/src/cuda_bimp.cu:318-331 in double.  Kernel size and centre stay at
// the nominal geometry.
void derivative_taps(const ScaleHost& s, const bimp_params& p, std::vector<float>* de_da, std::vector<float>* do_da,
                     std::vector<float>* de_dr, std::vector<float>* do_dr) {
  const int n = s.kW;
  const double lam = s.lambda, rho = p.sigma_ratio, sig = rho * lam;
  const double fs = s.filtersize;
  for (int o = 0; o < kNumOri; ++o) {
    const double th = static_cast<float>(o * M_PI / kNumOri);
    const double c = std::cos(th), sn = std::sin(th);
    std::vector<double> e_raw(n * n), ea(n * n), er(n * n), oa(n * n), orr(n * n);
    double S = 0, Sa = 0, Sr = 0;
    for (int row = 0; row < n; ++row) {
      for (int col = 0; col < n; ++col) {
        const double x = col - s.kX, y = row - s.kX;
        const double a = x * c + y * sn, b = y * c - x * sn;
        const double Q = a * a + p.gamma * b * b;
        const double env = std::exp(-Q / (2 * sig * sig));
        const double f = 2 * M_PI * a / lam;
        const double cf = std::cos(f), sf = std::sin(f);
        const double e_l = env * sf * (f / lam), o_l = -env * cf * (f / lam);
        const double env_s = env * Q / (sig * sig * sig);
        const double e_s = env_s * cf, o_s = env_s * sf;
        const int k = row * n + col;
        e_raw[k] = env * cf;
        ea[k] = lam * e_l + rho * lam * e_s;
        oa[k] = lam * o_l + rho * lam * o_s;
        er[k] = lam * e_s;
        orr[k] = lam * o_s;
        S += e_raw[k];
        Sa += ea[k];
        Sr += er[k];
      }
    }
    de_da[o].resize(n * n);
    do_da[o].resize(n * n);
    de_dr[o].resize(n * n);
    do_dr[o].resize(n * n);
    for (int k = 0; k < n * n; ++k) {
      de_da[o][k] = static_cast<float>(ea[k] - Sa / (fs * fs) + 2 * S * p.size_ratio * lam / (fs * fs * fs));
      do_da[o][k] = static_cast<float>(oa[k]);
      de_dr[o][k] = static_cast<float>(er[k] - Sr / (fs * fs));
      do_dr[o][k] = static_cast<float>(orr[k]);
    }
  }
}

}  // namespace bimp_b200

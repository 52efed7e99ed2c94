/*
 * cbimp.c -- FP32 C restatement of BIMP keypoint extraction with its own
 * mixed-radix FFT and OpenMP threads.
 *
 * TEST INFRASTRUCTURE AND CPU BASELINE ONLY.  The tests check it against the
 * FP64 oracle (bimp_oracle.py) and the benchmark times it on the host cores
 * as the CPU baseline.  The product never links, loads or calls it.
 *
 * It computes the per-scale pipeline of daniel-koudouna/cuda-bimp the way the
 * reference does, on the whole fftH x fftW torus of every scale:
 *   wavelengths  bimp/src/cuda_bimp.cu:927-937 (makeLambdasLog, caller's list)
 *   geometry     bimp/src/cuda_bimp.cu:222-256, snapTransformSize :200-219
 *   taps         bimp/src/cuda_bimp.cu:304-331 (float arithmetic)
 *   pyramid      bimp/src/cuda_bimp.cu:473-486 (pyrDown on u8, then
 *                convertTo(CV_32F, 255/65536))
 *   padding      bimp/include/detection/convolutionFFT2D.cuh:31-49 (kernel,
 *                centre at (0,0)) and :56-85 (data: copy/clamp-last/clamp-first)
 *   filtering    bimp/include/detection/cuda_bimp.cuh:226-248 with the
 *                R2C/C2R transforms of bimp/src/cuda_bimp.cu:498-515; the
 *                product of the spectra is scaled by 1/F
 *   |e + i o|    bimp/include/detection/cuda_bimp.cuh:165-180
 *   end-stop     bimp/include/detection/cuda_bimp.cuh:436-467
 *   inhibition   bimp/include/detection/cuda_bimp.cuh:469-502
 *   D -= T + R   bimp/include/detection/cuda_bimp.cuh:504-517
 *   keypoints    bimp/src/cuda_bimp.cu:714-743, cuda_bimp.cuh:86-148
 *
 * Two differences of form, not of result: the e and o responses of one
 * orientation come out of ONE complex inverse transform (for real X, Ke, Ko,
 * IFFT(X (Ke + i Ko)) = e + i o), and keypoints are listed in (scale, y, x)
 * order instead of the reference's atomic-slot order.  Where the reference
 * is undefined the choices are the FP64 oracle's: the stencils' flat index
 * wraps modulo fftH*fftW, oversize kernels wrap onto the torus and add, and
 * pyrDown rounds exact .5 ties to even.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define CB_NORI 8
#define CB_VB 8      /* sequences transformed together (one AVX register of floats) */
#define CB_MAXR 64   /* largest prime radix */
#define CB_MAXST 40

typedef struct {
  double gamma, sigma_ratio, size_ratio, offset_ratio, level_max, radial_gain, w_tan, w_rad, thresh_ratio;
} cb_params;

/* cv::KeyPoint field order: pt.x, pt.y, size, angle, response, octave, class_id */
typedef struct {
  float x, y, size, angle, response;
  int octave, class_id;
} cb_keypoint;

/* ------------------------------------------------------------------------- */
/* FFT: mixed-radix Stockham (self-sorting), batched over CB_VB sequences    */
/* stored interleaved: element i of sequence b at [i * CB_VB + b], re and im  */
/* in separate arrays.  Stage with radix R after Ns = product of the earlier  */
/* radices: for j in [0, N/R), v_r = x[j + r N/R] * w^(r (j mod Ns)),         */
/* w = exp(-2 pi i / (Ns R)); DFT-R of v; y[(j - j mod Ns) R + j mod Ns +    */
/* r Ns] = V_r.                                                               */
/* ------------------------------------------------------------------------- */
typedef struct {
  int n, nst;
  int rad[CB_MAXST];
  float* twr[CB_MAXST];
  float* twi[CB_MAXST];
  float* rtr[CB_MAXST]; /* exp(-2 pi i k / R), k < R */
  float* rti[CB_MAXST];
} cb_plan;

static void plan_free(cb_plan* p) {
  for (int s = 0; s < p->nst; ++s) {
    free(p->twr[s]);
    free(p->twi[s]);
    free(p->rtr[s]);
    free(p->rti[s]);
  }
  memset(p, 0, sizeof *p);
}

static int plan_init(cb_plan* p, int n) {
  memset(p, 0, sizeof *p);
  p->n = n;
  int m = n, ns = 0;
  while (m % 4 == 0 && ns < CB_MAXST) { p->rad[ns++] = 4; m /= 4; }
  while (m % 2 == 0 && ns < CB_MAXST) { p->rad[ns++] = 2; m /= 2; }
  for (int f = 3; m > 1 && ns < CB_MAXST; f += 2) {
    while (m % f == 0) {
      if (f > CB_MAXR) return -1;
      p->rad[ns++] = f;
      m /= f;
    }
  }
  if (m != 1) return -1;
  p->nst = ns;
  int Ns = 1;
  for (int s = 0; s < ns; ++s) {
    const int R = p->rad[s];
    p->twr[s] = (float*)malloc(sizeof(float) * (size_t)Ns * R);
    p->twi[s] = (float*)malloc(sizeof(float) * (size_t)Ns * R);
    p->rtr[s] = (float*)malloc(sizeof(float) * R);
    p->rti[s] = (float*)malloc(sizeof(float) * R);
    if (!p->twr[s] || !p->twi[s] || !p->rtr[s] || !p->rti[s]) return -1;
    for (int jm = 0; jm < Ns; ++jm)
      for (int r = 0; r < R; ++r) {
        const double a = -2.0 * M_PI * (double)r * jm / ((double)Ns * R);
        p->twr[s][jm * R + r] = (float)cos(a);
        p->twi[s][jm * R + r] = (float)sin(a);
      }
    for (int k = 0; k < R; ++k) {
      p->rtr[s][k] = (float)cos(-2.0 * M_PI * k / R);
      p->rti[s][k] = (float)sin(-2.0 * M_PI * k / R);
    }
    Ns *= R;
  }
  return 0;
}

static void fft_stage(const cb_plan* p, int s, int Ns, const float* restrict xr, const float* restrict xi,
                      float* restrict yr, float* restrict yi) {
  const int N = p->n, R = p->rad[s], NR = N / R;
  const float* twr = p->twr[s];
  const float* twi = p->twi[s];
  float vr[CB_MAXR][CB_VB], vi[CB_MAXR][CB_VB];
  float ur[CB_MAXR][CB_VB], ui[CB_MAXR][CB_VB];
  for (int j = 0; j < NR; ++j) {
    const int jm = j % Ns;
    const int d = (j - jm) * R + jm;
    for (int r = 0; r < R; ++r) {
      const float wr = twr[jm * R + r], wi = twi[jm * R + r];
      const float* ar = xr + (size_t)(j + r * NR) * CB_VB;
      const float* ai = xi + (size_t)(j + r * NR) * CB_VB;
      for (int b = 0; b < CB_VB; ++b) {
        vr[r][b] = ar[b] * wr - ai[b] * wi;
        vi[r][b] = ar[b] * wi + ai[b] * wr;
      }
    }
    if (R == 4) {
      for (int b = 0; b < CB_VB; ++b) {
        const float s0r = vr[0][b] + vr[2][b], s0i = vi[0][b] + vi[2][b];
        const float d0r = vr[0][b] - vr[2][b], d0i = vi[0][b] - vi[2][b];
        const float s1r = vr[1][b] + vr[3][b], s1i = vi[1][b] + vi[3][b];
        const float d1r = vr[1][b] - vr[3][b], d1i = vi[1][b] - vi[3][b];
        ur[0][b] = s0r + s1r; ui[0][b] = s0i + s1i;
        ur[2][b] = s0r - s1r; ui[2][b] = s0i - s1i;
        /* X1 = d0 - i d1, X3 = d0 + i d1 */
        ur[1][b] = d0r + d1i; ui[1][b] = d0i - d1r;
        ur[3][b] = d0r - d1i; ui[3][b] = d0i + d1r;
      }
    } else if (R == 2) {
      for (int b = 0; b < CB_VB; ++b) {
        ur[0][b] = vr[0][b] + vr[1][b]; ui[0][b] = vi[0][b] + vi[1][b];
        ur[1][b] = vr[0][b] - vr[1][b]; ui[1][b] = vi[0][b] - vi[1][b];
      }
    } else {
      const float* rr = p->rtr[s];
      const float* ri = p->rti[s];
      for (int k = 0; k < R; ++k) {
        float accr[CB_VB], acci[CB_VB];
        for (int b = 0; b < CB_VB; ++b) { accr[b] = vr[0][b]; acci[b] = vi[0][b]; }
        for (int q = 1; q < R; ++q) {
          const int e = (q * k) % R;
          const float cr = rr[e], ci = ri[e];
          for (int b = 0; b < CB_VB; ++b) {
            accr[b] += vr[q][b] * cr - vi[q][b] * ci;
            acci[b] += vr[q][b] * ci + vi[q][b] * cr;
          }
        }
        for (int b = 0; b < CB_VB; ++b) { ur[k][b] = accr[b]; ui[k][b] = acci[b]; }
      }
    }
    for (int r = 0; r < R; ++r) {
      float* orr = yr + (size_t)(d + r * Ns) * CB_VB;
      float* oii = yi + (size_t)(d + r * Ns) * CB_VB;
      for (int b = 0; b < CB_VB; ++b) { orr[b] = ur[r][b]; oii[b] = ui[r][b]; }
    }
  }
}

/* Forward DFT of CB_VB interleaved sequences; returns 0 when the result is
 * in (ar, ai), 1 when it is in (br, bi). */
static int fft_batch(const cb_plan* p, float* ar, float* ai, float* br, float* bi) {
  int Ns = 1, cur = 0;
  for (int s = 0; s < p->nst; ++s) {
    if (cur == 0) fft_stage(p, s, Ns, ar, ai, br, bi);
    else fft_stage(p, s, Ns, br, bi, ar, ai);
    cur ^= 1;
    Ns *= p->rad[s];
  }
  return cur;
}

/* In-place 2-D DFT of an H x W complex array (rows of W).  inverse != 0
 * gives the unnormalised inverse (conjugate in, forward, conjugate out).
 * H and W are multiples of CB_VB. */
static void fft2(const cb_plan* pw, const cb_plan* ph, float* re, float* im, int H, int W, int inverse) {
  const float sg = inverse ? -1.f : 1.f;
  const int nmax = W > H ? W : H;
#pragma omp parallel
  {
    float* buf = (float*)malloc(sizeof(float) * 4 * (size_t)nmax * CB_VB);
    float* ar = buf;
    float* ai = buf + (size_t)nmax * CB_VB;
    float* br = ai + (size_t)nmax * CB_VB;
    float* bi = br + (size_t)nmax * CB_VB;
#pragma omp for schedule(static)
    for (int r0 = 0; r0 < H; r0 += CB_VB) {
      for (int b = 0; b < CB_VB; ++b) {
        const float* sr = re + (size_t)(r0 + b) * W;
        const float* si = im + (size_t)(r0 + b) * W;
        for (int x = 0; x < W; ++x) {
          ar[x * CB_VB + b] = sr[x];
          ai[x * CB_VB + b] = sg * si[x];
        }
      }
      const int w = fft_batch(pw, ar, ai, br, bi);
      const float* orr = w ? br : ar;
      const float* oii = w ? bi : ai;
      for (int b = 0; b < CB_VB; ++b) {
        float* dr = re + (size_t)(r0 + b) * W;
        float* di = im + (size_t)(r0 + b) * W;
        for (int x = 0; x < W; ++x) {
          dr[x] = orr[x * CB_VB + b];
          di[x] = oii[x * CB_VB + b];
        }
      }
    }
#pragma omp for schedule(static)
    for (int c0 = 0; c0 < W; c0 += CB_VB) {
      for (int y = 0; y < H; ++y) {
        const float* sr = re + (size_t)y * W + c0;
        const float* si = im + (size_t)y * W + c0;
        for (int b = 0; b < CB_VB; ++b) {
          ar[y * CB_VB + b] = sr[b];
          ai[y * CB_VB + b] = si[b];
        }
      }
      const int w = fft_batch(ph, ar, ai, br, bi);
      const float* orr = w ? br : ar;
      const float* oii = w ? bi : ai;
      for (int y = 0; y < H; ++y) {
        float* dr = re + (size_t)y * W + c0;
        float* di = im + (size_t)y * W + c0;
        for (int b = 0; b < CB_VB; ++b) {
          dr[b] = orr[y * CB_VB + b];
          di[b] = sg * oii[y * CB_VB + b];
        }
      }
    }
    free(buf);
  }
}

/* In-place 2-D DFT of an H x W complex array for the tests (H, W multiples
 * of 8 whose prime factors are <= 64); returns -1 on unsupported sizes. */
int cbimp_fft2(float* re, float* im, int H, int W, int inverse) {
  if (H <= 0 || W <= 0 || H % CB_VB || W % CB_VB) return -1;
  cb_plan pw, ph;
  if (plan_init(&pw, W) || plan_init(&ph, H)) return -1;
  fft2(&pw, &ph, re, im, H, W, inverse);
  plan_free(&pw);
  plan_free(&ph);
  return 0;
}

/* ------------------------------------------------------------------------- */
/* geometry and bank                                                          */
/* ------------------------------------------------------------------------- */
typedef struct {
  float lambda2, lambda, pyrstep, filtersize;
  int kW, kX, dataW, dataH, fftW, fftH, level, off;
  int es1[CB_NORI], es2[CB_NORI], in1[CB_NORI], in2[CB_NORI], ih1[CB_NORI], ih2[CB_NORI];
  cb_plan pw, ph;
  float* Wr; /* CB_NORI x F: spectrum of even taps + i * spectrum of odd taps */
  float* Wi;
  float* D;  /* dataH x dataW */
  float* S;
} cb_scale;

typedef struct {
  int w, h, ns, nlev;
  cb_params p;
  cb_scale* sc;
  uint8_t* lv[32];
  int lw[32], lh[32];
  size_t fmax;
  float *Xr, *Xi, *Yr, *Yi, *C;
} cb_ctx;

static const cb_params kDefaults = {0.5, 0.56, 7.0, 0.6, 7.5, 16.0, 1.0, 1.0, 0.104};

int cbimp_snap_transform_size(int n) {
  if (n <= 0) return 0;
  n = (n + 15) / 16 * 16;
  int hi = 30;
  while (hi > 0 && !(n & (1 << hi))) --hi;
  if ((1 << hi) == n) return n;
  if ((1 << (hi + 1)) <= 1024) return 1 << (hi + 1);
  return (n + 511) / 512 * 512;
}

static int round_half_away(double v) { return (int)(v >= 0 ? floor(v + 0.5) : -floor(-v + 0.5)); }

static int cmp_float(const void* a, const void* b) {
  const float x = *(const float*)a, y = *(const float*)b;
  return (x > y) - (x < y);
}

/* Real taps of orientation o (cuda_bimp.cu:304-331), float arithmetic. */
static void gabor_taps(const cb_scale* s, const cb_params* p, int o, float* ev, float* od) {
  const float gamma = (float)p->gamma;
  const float phi = (float)(-M_PI / 2);
  const float sigma = (float)(s->lambda * p->sigma_ratio);
  const float sigsq = sigma * sigma;
  const float theta = (float)(o * M_PI / CB_NORI);
  const float st = sinf(theta), ct = cosf(theta);
  const int n = s->kW;
  float evensum = 0.f;
  for (int row = 0; row < n; ++row)
    for (int col = 0; col < n; ++col) {
      const float x = (float)(col - s->kX), y = (float)(row - s->kX);
      const float a = x * ct + y * st;
      const float b = y * ct - x * st;
      const float coef = -1.f / (2.f * sigsq);
      const float env = expf(coef * (a * a + gamma * b * b));
      const float freq = (float)(2.0 * M_PI * a / s->lambda);
      ev[row * n + col] = env * cosf(freq);
      od[row * n + col] = env * cosf(freq + phi);
      evensum += ev[row * n + col];
    }
  const float fs = s->filtersize;
  for (int m = 0; m < n * n; ++m) ev[m] -= evensum / (fs * fs);
}

static int build_scale(cb_ctx* c, cb_scale* s, float l2) {
  const cb_params* p = &c->p;
  s->lambda2 = l2;
  float pyr = 1.f;
  while (l2 / pyr >= p->level_max) pyr *= 2;   /* cuda_bimp.cu:236-238 */
  s->pyrstep = pyr;
  s->lambda = l2 / pyr;
  float fs = (float)(p->size_ratio * (double)s->lambda);
  if ((int)fs % 2 == 0) fs += 1;
  s->filtersize = fs;
  s->kX = (int)floorf(fs / 2);
  s->kW = (int)fs;
  s->dataH = (int)(c->h / pyr);
  s->dataW = (int)(c->w / pyr);
  s->fftH = cbimp_snap_transform_size(s->dataH);
  s->fftW = cbimp_snap_transform_size(s->dataW);
  s->level = 0;
  for (float q = pyr; q > 1.f; q /= 2) s->level++;
  s->off = (int)s->lambda;
  if (s->dataW < 2 || s->dataH < 2 || s->level >= 31) return -1;
  for (int o = 0; o < CB_NORI; ++o) {
    const float th = (float)(o * M_PI / CB_NORI);
    const double cth = cosf(th), sth = sinf(th);
    s->es1[o] = round_half_away(p->offset_ratio * s->lambda * cth);
    s->es2[o] = round_half_away(p->offset_ratio * s->lambda * sth);
    s->in1[o] = round_half_away(p->offset_ratio * s->lambda * sth);
    s->in2[o] = round_half_away(p->offset_ratio * s->lambda * cth);
    s->ih1[o] = round_half_away(0.5 * s->in1[o]);
    s->ih2[o] = round_half_away(0.5 * s->in2[o]);
  }
  if (plan_init(&s->pw, s->fftW) || plan_init(&s->ph, s->fftH)) return -1;
  const size_t F = (size_t)s->fftH * s->fftW;
  if (F > c->fmax) c->fmax = F;
  s->Wr = (float*)malloc(sizeof(float) * CB_NORI * F);
  s->Wi = (float*)malloc(sizeof(float) * CB_NORI * F);
  s->D = (float*)malloc(sizeof(float) * (size_t)s->dataW * s->dataH);
  s->S = (float*)malloc(sizeof(float) * (size_t)s->dataW * s->dataH);
  float* er = (float*)calloc(F, sizeof(float));
  float* ei = (float*)calloc(F, sizeof(float));
  float* orr = (float*)calloc(F, sizeof(float));
  float* oi = (float*)calloc(F, sizeof(float));
  float* te = (float*)malloc(sizeof(float) * s->kW * s->kW);
  float* to = (float*)malloc(sizeof(float) * s->kW * s->kW);
  if (!s->Wr || !s->Wi || !s->D || !s->S || !er || !ei || !orr || !oi || !te || !to) return -1;
  for (int o = 0; o < CB_NORI; ++o) {
    gabor_taps(s, p, o, te, to);
    memset(er, 0, sizeof(float) * F);
    memset(ei, 0, sizeof(float) * F);
    memset(orr, 0, sizeof(float) * F);
    memset(oi, 0, sizeof(float) * F);
    /* convolutionFFT2D.cuh:31-49: tap (ky, kx) at ((ky-kX) mod fftH, (kx-kX) mod fftW) */
    for (int ky = 0; ky < s->kW; ++ky) {
      const int y = ((ky - s->kX) % s->fftH + s->fftH) % s->fftH;
      for (int kx = 0; kx < s->kW; ++kx) {
        const int x = ((kx - s->kX) % s->fftW + s->fftW) % s->fftW;
        er[(size_t)y * s->fftW + x] += te[ky * s->kW + kx];
        orr[(size_t)y * s->fftW + x] += to[ky * s->kW + kx];
      }
    }
    fft2(&s->pw, &s->ph, er, ei, s->fftH, s->fftW, 0);
    fft2(&s->pw, &s->ph, orr, oi, s->fftH, s->fftW, 0);
    float* wr = s->Wr + (size_t)o * F;
    float* wi = s->Wi + (size_t)o * F;
    for (size_t k = 0; k < F; ++k) {
      wr[k] = er[k] - oi[k];
      wi[k] = ei[k] + orr[k];
    }
  }
  free(er); free(ei); free(orr); free(oi); free(te); free(to);
  return 0;
}

void cbimp_destroy(void* h) {
  cb_ctx* c = (cb_ctx*)h;
  if (!c) return;
  for (int i = 0; i < c->ns; ++i) {
    cb_scale* s = &c->sc[i];
    plan_free(&s->pw);
    plan_free(&s->ph);
    free(s->Wr); free(s->Wi); free(s->D); free(s->S);
  }
  free(c->sc);
  for (int l = 0; l < 32; ++l) free(c->lv[l]);
  free(c->Xr); free(c->Xi); free(c->Yr); free(c->Yi); free(c->C);
  free(c);
}

/* params: 9 doubles in the order of cb_params, or NULL for the defaults. */
void* cbimp_create(int width, int height, const float* lambdas, int n, const double* params) {
  if (width < 2 || height < 2 || !lambdas || n <= 0) return NULL;
  cb_ctx* c = (cb_ctx*)calloc(1, sizeof(cb_ctx));
  if (!c) return NULL;
  c->w = width;
  c->h = height;
  c->p = kDefaults;
  if (params) memcpy(&c->p, params, sizeof(cb_params));
  float* lam = (float*)malloc(sizeof(float) * n);
  memcpy(lam, lambdas, sizeof(float) * n);
  qsort(lam, n, sizeof(float), cmp_float);   /* cuda_bimp.cu:224 */
  c->sc = (cb_scale*)calloc(n, sizeof(cb_scale));
  c->ns = n;
  for (int i = 0; i < n; ++i) {
    if (!(lam[i] > 0.f) || build_scale(c, &c->sc[i], lam[i])) {
      free(lam);
      cbimp_destroy(c);
      return NULL;
    }
    if (c->sc[i].level + 1 > c->nlev) c->nlev = c->sc[i].level + 1;
  }
  free(lam);
  int w = width, h = height;
  for (int l = 0; l < c->nlev; ++l) {
    c->lw[l] = w;
    c->lh[l] = h;
    c->lv[l] = (uint8_t*)malloc((size_t)w * h);
    w = (w + 1) / 2;
    h = (h + 1) / 2;
  }
  c->Xr = (float*)malloc(sizeof(float) * c->fmax);
  c->Xi = (float*)malloc(sizeof(float) * c->fmax);
  c->Yr = (float*)malloc(sizeof(float) * c->fmax);
  c->Yi = (float*)malloc(sizeof(float) * c->fmax);
  c->C = (float*)malloc(sizeof(float) * CB_NORI * c->fmax);
  if (!c->Xr || !c->Xi || !c->Yr || !c->Yi || !c->C) {
    cbimp_destroy(c);
    return NULL;
  }
  return c;
}

int cbimp_num_scales(const void* h) { return h ? ((const cb_ctx*)h)->ns : 0; }

/* geometry of scale s: dataW, dataH, fftW, fftH, kW, off, level */
int cbimp_scale_info(const void* h, int s, int* out7) {
  const cb_ctx* c = (const cb_ctx*)h;
  if (!c || s < 0 || s >= c->ns || !out7) return -1;
  const cb_scale* q = &c->sc[s];
  out7[0] = q->dataW; out7[1] = q->dataH; out7[2] = q->fftW; out7[3] = q->fftH;
  out7[4] = q->kW; out7[5] = q->off; out7[6] = q->level;
  return 0;
}

void cbimp_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int cbimp_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* ------------------------------------------------------------------------- */
/* per-image pipeline                                                         */
/* ------------------------------------------------------------------------- */
static inline int reflect101(int i, int n) {
  if (n == 1) return 0;
  const int period = 2 * n - 2;
  i = abs(i) % period;
  return i >= n ? period - i : i;
}

/* cv::cuda::pyrDown on CV_8UC1: 5-tap [1 4 6 4 1] separable, reflect-101,
 * exact integer sum / 256 rounded half to even. */
static void pyr_down(const uint8_t* src, int sw, int sh, int sp, uint8_t* dst, int dw, int dh) {
  static const int w5[5] = {1, 4, 6, 4, 1};
#pragma omp parallel for schedule(static)
  for (int y = 0; y < dh; ++y) {
    int rows[5];
    for (int i = 0; i < 5; ++i) rows[i] = reflect101(2 * y + i - 2, sh);
    for (int x = 0; x < dw; ++x) {
      int acc = 0;
      for (int i = 0; i < 5; ++i) {
        const uint8_t* r = src + (size_t)rows[i] * sp;
        int hsum = 0;
        for (int k = 0; k < 5; ++k) hsum += w5[k] * r[reflect101(2 * x + k - 2, sw)];
        acc += w5[i] * hsum;
      }
      const int q = acc >> 8, rem = acc & 255;
      int v = q + ((rem > 128 || (rem == 128 && (q & 1))) ? 1 : 0);
      dst[(size_t)y * dw + x] = (uint8_t)(v > 255 ? 255 : v);
    }
  }
}

/* convolutionFFT2D.cuh:56-85: padded row/col t reads data t, the last
 * data row/col for t < n + k, else the first (clamp to the border on the
 * torus: the rows/cols after the clamped band wrap to data row/col 0). */
static inline int pad_src(int t, int n, int k) { return t < n ? t : (t < n + k ? n - 1 : 0); }

static void filter_scale(cb_ctx* c, cb_scale* s) {
  const int fw = s->fftW, fh = s->fftH, dw = s->dataW, dh = s->dataH;
  const size_t F = (size_t)fw * fh;
  const uint8_t* lvl = c->lv[s->level];
  const int lw = c->lw[s->level];
  const float conv = (float)(255.0 / 65536.0);
  float* Xr = c->Xr;
  float* Xi = c->Xi;
#pragma omp parallel for schedule(static)
  for (int y = 0; y < fh; ++y) {
    const int sy = pad_src(y, dh, s->kX);
    for (int x = 0; x < fw; ++x) {
      const int sx = pad_src(x, dw, s->kX);
      Xr[(size_t)y * fw + x] = (float)lvl[(size_t)sy * lw + sx] * conv;
      Xi[(size_t)y * fw + x] = 0.f;
    }
  }
  fft2(&s->pw, &s->ph, Xr, Xi, fh, fw, 0);
  const float inv = 1.f / (float)F;
  for (int o = 0; o < CB_NORI; ++o) {
    const float* wr = s->Wr + (size_t)o * F;
    const float* wi = s->Wi + (size_t)o * F;
    float* Yr = c->Yr;
    float* Yi = c->Yi;
#pragma omp parallel for schedule(static)
    for (long long k = 0; k < (long long)F; ++k) {
      Yr[k] = (Xr[k] * wr[k] - Xi[k] * wi[k]) * inv;
      Yi[k] = (Xr[k] * wi[k] + Xi[k] * wr[k]) * inv;
    }
    fft2(&s->pw, &s->ph, Yr, Yi, fh, fw, 1);
    float* Co = c->C + (size_t)o * F;
#pragma omp parallel for schedule(static)
    for (long long k = 0; k < (long long)F; ++k) Co[k] = sqrtf(Yr[k] * Yr[k] + Yi[k] * Yi[k]);
  }
}

/* Complex-cell value at window (r, c): flat index r*fftW + c modulo F. */
static inline float cw(const float* Co, long long r, long long col, long long fw, long long F) {
  long long k = r * fw + col;
  if (k >= F) k -= F;
  return Co[k];
}

static void stencil_scale(cb_ctx* c, cb_scale* s) {
  const int W = s->dataW, H = s->dataH;
  const long long fw = s->fftW, F = (long long)s->fftW * s->fftH;
  const float gain = (float)c->p.radial_gain, wT = (float)c->p.w_tan, wR = (float)c->p.w_rad;
  const float* C = c->C;
#pragma omp parallel for schedule(static)
  for (int y = 0; y < H; ++y) {
    for (int x = 0; x < W; ++x) {
      float S = 0.f, D = 0.f, T = 0.f, R = 0.f;
      for (int o = 0; o < CB_NORI; ++o) {
        const int o1 = s->es1[o], o2 = s->es2[o];
        const int ax = abs(o2), ay = abs(o1);
        if (!(x - 2 * ax >= 0 && x + 2 * ax <= W && y - 2 * ay >= 0 && y + 2 * ay <= H)) continue;
        const float* Co = C + (size_t)o * F;
        float sv = cw(Co, y - o1, x + o2, fw, F) - cw(Co, y + o1, x - o2, fw, F);
        if (sv > 0.f) S += sv;
        float dv = cw(Co, y, x, fw, F) - 0.5f * cw(Co, y - 2 * o1, x + 2 * o2, fw, F) -
                   0.5f * cw(Co, y + 2 * o1, x - 2 * o2, fw, F);
        if (dv > 0.f) D += dv;
      }
      for (int o = 0; o < CB_NORI; ++o) {
        const int o1 = s->in1[o], o2 = s->in2[o];
        const int ax = abs(o2), ay = abs(o1);
        if (!(x - 2 * ax >= 0 && x + 2 * ax <= W && y - 2 * ay >= 0 && y + 2 * ay <= H)) continue;
        const float* Co = C + (size_t)o * F;
        const float* Cp = C + (size_t)((o + CB_NORI / 2) % CB_NORI) * F;
        const float centre = cw(Co, y, x, fw, F);
        float tv = cw(Co, y - o1, x - o2, fw, F) - centre;
        if (tv > 0.f) T += tv;
        const int h1 = s->ih1[o], h2 = s->ih2[o];
        float r = centre - gain * cw(Cp, y + h1, x + h2, fw, F);
        r = r > 0.f ? r : 0.f;
        r += centre - gain * cw(Cp, y - h1, x - h2, fw, F);
        r = r > 0.f ? r : 0.f;
        R += r;
      }
      const float inhib = wT * T + wR * R;
      s->D[(size_t)y * W + x] = D - inhib;
      s->S[(size_t)y * W + x] = S - inhib;
    }
  }
}

/* Threshold, strict 8-neighbour maximum and parabolic subpixel position,
 * appended in (y, x) order (cuda_bimp.cu:714-743, cuda_bimp.cuh:86-148). */
static int keypoints_scale(const cb_ctx* c, const cb_scale* s, cb_keypoint* out, int cap, int n0, int* total) {
  const int W = s->dataW, H = s->dataH;
  const float* Dm = s->D;
  float mx = -INFINITY;
  for (size_t k = 0; k < (size_t)W * H; ++k) mx = Dm[k] > mx ? Dm[k] : mx;
  const float thr = (float)((double)mx * c->p.thresh_ratio);
  const int off = s->off;
  const int y1 = H - off < H - 1 ? H - off : H - 1;
  const int x1 = W - off < W - 1 ? W - off : W - 1;
  int n = n0;
  for (int y = off + 1; y < y1; ++y) {
    const float* r0 = Dm + (size_t)(y - 1) * W;
    const float* r1 = r0 + W;
    const float* r2 = r1 + W;
    for (int x = off + 1; x < x1; ++x) {
      const float v = r1[x];
      float dil = r0[x - 1];
      dil = fmaxf(dil, r0[x]); dil = fmaxf(dil, r0[x + 1]);
      dil = fmaxf(dil, r1[x - 1]); dil = fmaxf(dil, r1[x + 1]);
      dil = fmaxf(dil, r2[x - 1]); dil = fmaxf(dil, r2[x]); dil = fmaxf(dil, r2[x + 1]);
      if (!(v - dil > 0.f && v > thr)) continue;
      if (n < cap && out) {
        const float xv1 = r1[x - 1], xv3 = r1[x + 1], yv1 = r0[x], yv3 = r2[x];
        float xp = (float)x, yp = (float)y;
        const float dx = xv1 + xv3 - 2.f * v, dy = yv1 + yv3 - 2.f * v;
        if (dx != 0.f) xp += 0.5f * (xv1 - xv3) / dx;
        if (dy != 0.f) yp += 0.5f * (yv1 - yv3) / dy;
        cb_keypoint* k = &out[n];
        k->x = xp * s->pyrstep;
        k->y = yp * s->pyrstep;
        k->size = s->lambda * s->pyrstep;
        k->angle = -1.f;
        k->response = v;
        k->octave = (int)(s->lambda * s->pyrstep);
        k->class_id = 1;
      }
      ++n;
    }
  }
  *total += n - n0;
  return n < cap ? n : cap;
}

/* Detects on one u8 image (pitch bytes per row).  Writes up to cap records
 * and returns how many were written; *total receives the number found. */
int cbimp_detect(void* h, const uint8_t* img, int pitch, cb_keypoint* out, int cap, int* total) {
  cb_ctx* c = (cb_ctx*)h;
  if (!c || !img || pitch < c->w || cap < 0) return -1;
  for (int y = 0; y < c->h; ++y) memcpy(c->lv[0] + (size_t)y * c->w, img + (size_t)y * pitch, c->w);
  for (int l = 1; l < c->nlev; ++l)
    pyr_down(c->lv[l - 1], c->lw[l - 1], c->lh[l - 1], c->lw[l - 1], c->lv[l], c->lw[l], c->lh[l]);
  int n = 0, tot = 0;
  for (int i = 0; i < c->ns; ++i) {
    cb_scale* s = &c->sc[i];
    filter_scale(c, s);
    stencil_scale(c, s);
    n = keypoints_scale(c, s, out, cap, n, &tot);
  }
  if (total) *total = tot;
  return n;
}

/* Complex cells of orientation o of the LAST scale of the last detection,
 * fftH x fftW floats. */
int cbimp_last_complex_map(const void* h, int o, float* out) {
  const cb_ctx* c = (const cb_ctx*)h;
  if (!c || o < 0 || o >= CB_NORI || !out) return -1;
  const cb_scale* q = &c->sc[c->ns - 1];
  const size_t F = (size_t)q->fftW * q->fftH;
  memcpy(out, c->C + (size_t)o * F, sizeof(float) * F);
  return 0;
}

/* D (which = 0) or S (which = 1) of scale s from the last detection,
 * dataH x dataW floats. */
int cbimp_dense_map(const void* h, int s, int which, float* out) {
  const cb_ctx* c = (const cb_ctx*)h;
  if (!c || s < 0 || s >= c->ns || !out) return -1;
  const cb_scale* q = &c->sc[s];
  memcpy(out, which ? q->S : q->D, sizeof(float) * (size_t)q->dataW * q->dataH);
  return 0;
}

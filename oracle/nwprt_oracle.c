/* CPU oracle for the neural wavelet PRT relight path -- TEST INFRASTRUCTURE ONLY.
 * See nwprt_oracle.h for what each function restates and its parity status.
 * Build: oracle/Makefile (-O3 -march=x86-64-v3 -fopenmp -ffp-contract=off). */
#include "nwprt_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

static void set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* ------------------------------------------------------------------------ */
/* Haar transform + top-K                                                    */
/* ------------------------------------------------------------------------ */

/* Selection key: |luminance| of the coefficient's RGB with the reference's
 * luminance weights (EnvironmentMap.cpp:149-151), evaluated left to right in
 * FP32 without contraction.  NaN keys sort as 0 (lowest priority). */
float orc_wavelet_key(float r, float g, float b) {
  float t = 0.212671f * r;
  t = t + 0.715160f * g;
  t = t + 0.072169f * b;
  t = fabsf(t);
  if (t != t) t = 0.0f;
  return t;
}

/* Non-standard 2-D Haar decomposition with orthonormal 1/2 factors, Mallat
 * layout, recursive down to 1x1.  For each 2x2 block (a b / c d) of the
 * current n x n low-pass square:
 *   LL=(a+b+c+d)/2 -> (i, j)        HL=(a-b+c-d)/2 -> (i, j+n/2)
 *   LH=(a+b-c-d)/2 -> (i+n/2, j)    HH=(a-b-c+d)/2 -> (i+n/2, j+n/2)
 * evaluated as s0=a+b, d0=a-b, s1=c+d, d1=c-d and (x+y)*0.5f. */
void orc_haar_face(float* face, int S) {
  float* tmp = (float*)malloc(sizeof(float) * (size_t)S * S * 3);
  for (int n = S; n >= 2; n >>= 1) {
    const int h = n >> 1;
    for (int i = 0; i < h; ++i)
      for (int j = 0; j < h; ++j)
        for (int c = 0; c < 3; ++c) {
          const float a = face[((2 * i) * S + 2 * j) * 3 + c];
          const float b = face[((2 * i) * S + 2 * j + 1) * 3 + c];
          const float cc = face[((2 * i + 1) * S + 2 * j) * 3 + c];
          const float d = face[((2 * i + 1) * S + 2 * j + 1) * 3 + c];
          const float s0 = a + b, d0 = a - b, s1 = cc + d, d1 = cc - d;
          tmp[(i * S + j) * 3 + c] = (s0 + s1) * 0.5f;
          tmp[(i * S + j + h) * 3 + c] = (d0 + d1) * 0.5f;
          tmp[((i + h) * S + j) * 3 + c] = (s0 - s1) * 0.5f;
          tmp[((i + h) * S + j + h) * 3 + c] = (d0 - d1) * 0.5f;
        }
    for (int i = 0; i < n; ++i)
      memcpy(&face[(size_t)i * S * 3], &tmp[(size_t)i * S * 3], sizeof(float) * n * 3);
  }
  free(tmp);
}

void orc_haar_inverse_face_f64(double* face, int S) {
  double* tmp = (double*)malloc(sizeof(double) * (size_t)S * S * 3);
  for (int n = 2; n <= S; n <<= 1) {
    const int h = n >> 1;
    for (int i = 0; i < h; ++i)
      for (int j = 0; j < h; ++j)
        for (int c = 0; c < 3; ++c) {
          const double LL = face[(i * S + j) * 3 + c], HL = face[(i * S + j + h) * 3 + c];
          const double LH = face[((i + h) * S + j) * 3 + c], HH = face[((i + h) * S + j + h) * 3 + c];
          const double s0 = LL + LH, s1 = LL - LH, d0 = HL + HH, d1 = HL - HH;
          tmp[((2 * i) * S + 2 * j) * 3 + c] = 0.5 * (s0 + d0);
          tmp[((2 * i) * S + 2 * j + 1) * 3 + c] = 0.5 * (s0 - d0);
          tmp[((2 * i + 1) * S + 2 * j) * 3 + c] = 0.5 * (s1 + d1);
          tmp[((2 * i + 1) * S + 2 * j + 1) * 3 + c] = 0.5 * (s1 - d1);
        }
    for (int i = 0; i < n; ++i)
      memcpy(&face[(size_t)i * S * 3], &tmp[(size_t)i * S * 3], sizeof(double) * n * 3);
  }
  free(tmp);
}

typedef struct {
  float key;
  int32_t idx;
} orc_keyed;

/* Total order: key descending, then flat index ascending. */
static int cmp_keyed(const void* pa, const void* pb) {
  const orc_keyed* a = (const orc_keyed*)pa;
  const orc_keyed* b = (const orc_keyed*)pb;
  if (a->key > b->key) return -1;
  if (a->key < b->key) return 1;
  return (a->idx > b->idx) - (a->idx < b->idx);
}

/* faces: [6][S][S][3] in the reference face order (+X,-X,+Y,-Y,-Z,+Z).
 * Flat coefficient index = face*S*S + row*S + col (the index space of the
 * wavelet embedding, utils_kernels.h:110-127).  Outputs in selection order. */
int orc_haar_topk(const float* faces, int S, int K, int32_t* idx, float* strength) {
  const int64_t per = (int64_t)S * S;
  const int64_t n = 6 * per;
  if (S < 1 || (S & (S - 1)) || K < 1 || K > n) return -1;
  float* c = (float*)malloc(sizeof(float) * n * 3);
  memcpy(c, faces, sizeof(float) * n * 3);
  for (int f = 0; f < 6; ++f) orc_haar_face(c + f * per * 3, S);
  orc_keyed* kv = (orc_keyed*)malloc(sizeof(orc_keyed) * n);
  for (int64_t i = 0; i < n; ++i) {
    kv[i].key = orc_wavelet_key(c[i * 3 + 0], c[i * 3 + 1], c[i * 3 + 2]);
    kv[i].idx = (int32_t)i;
  }
  qsort(kv, (size_t)n, sizeof(orc_keyed), cmp_keyed);
  for (int k = 0; k < K; ++k) {
    const int32_t j = kv[k].idx;
    idx[k] = j;
    strength[k * 3 + 0] = c[(int64_t)j * 3 + 0];
    strength[k * 3 + 1] = c[(int64_t)j * 3 + 1];
    strength[k * 3 + 2] = c[(int64_t)j * 3 + 2];
  }
  free(kv);
  free(c);
  return 0;
}

int orc_haar_topk_batch(const float* faces, int n_env, int S, int K, int32_t* idx,
                        float* strength, int n_threads) {
  int bad = 0;
  set_threads(n_threads);
#pragma omp parallel for schedule(dynamic, 1) reduction(| : bad)
  for (int e = 0; e < n_env; ++e)
    bad |= orc_haar_topk(faces + (int64_t)e * 6 * S * S * 3, S, K, idx + (int64_t)e * K,
                         strength + (int64_t)e * K * 3) != 0;
  return bad ? -1 : 0;
}

/* ------------------------------------------------------------------------ */
/* Spherical harmonics (pbrt-v2 real SH, as in shaderUtils.h:231-338)        */
/* ------------------------------------------------------------------------ */

static int sh_index(int l, int m) { return l * l + l + m; }

void orc_sh_eval_f64(double x, double y, double z, int lmax, double* out) {
  /* associated Legendre P(l,m), m >= 0, with the Condon-Shortley phase */
  double P[(ORC_MAX_LAYERS + 1) * (ORC_MAX_LAYERS + 1)];
  const double s = sqrt(fmax(0.0, 1.0 - z * z));
  for (int m = 0; m <= lmax; ++m) {
    /* P(m,m) = (-1)^m (2m-1)!! s^m */
    double pmm = 1.0;
    for (int i = 1; i <= m; ++i) pmm *= -(2.0 * i - 1.0) * s;
    P[sh_index(m, m)] = pmm;
    if (m + 1 <= lmax) P[sh_index(m + 1, m)] = z * (2.0 * m + 1.0) * pmm;
    for (int l = m + 2; l <= lmax; ++l)
      P[sh_index(l, m)] =
          ((2.0 * l - 1.0) * z * P[sh_index(l - 1, m)] - (l + m - 1.0) * P[sh_index(l - 2, m)]) /
          (double)(l - m);
  }
  double sn[ORC_MAX_LAYERS + 1], cs[ORC_MAX_LAYERS + 1];
  if (s == 0.0) {
    for (int m = 0; m <= lmax; ++m) { sn[m] = 0.0; cs[m] = 1.0; }
  } else {
    const double phi = atan2(y / s, x / s);
    for (int m = 0; m <= lmax; ++m) { sn[m] = sin(m * phi); cs[m] = cos(m * phi); }
  }
  for (int l = 0; l <= lmax; ++l)
    for (int m = 0; m <= l; ++m) {
      /* K(l,m) = sqrt((2l+1)/(4 pi) * (l-m)!/(l+m)!) */
      double ratio = 1.0;
      for (int t = l - m + 1; t <= l + m; ++t) ratio /= (double)t;
      const double K = sqrt((2.0 * l + 1.0) / (4.0 * M_PI) * ratio);
      const double p = P[sh_index(l, m)];
      if (m == 0) {
        out[sh_index(l, 0)] = K * p;
      } else {
        out[sh_index(l, m)] = M_SQRT2 * K * p * cs[m];
        out[sh_index(l, -m)] = M_SQRT2 * K * p * sn[m];
      }
    }
}

/* Direction of the texel centre (row, col) of face f: the cubemap texture's
 * (u, v) = ((col+0.5)/S, (row+0.5)/S) mapped by the reference's EnvUVToDirec
 * (device_functions/cubeMap.cu:97-113). */
static void face_dir(int f, double uc, double vc, double* d) {
  double x = 0, y = 0, z = 0;
  switch (f) {
    case 0: x = 1.0; y = vc; z = uc; break;
    case 1: x = -1.0; y = vc; z = -uc; break;
    case 2: x = uc; y = 1.0; z = vc; break;
    case 3: x = uc; y = -1.0; z = -vc; break;
    case 4: x = uc; y = vc; z = -1.0; break;
    default: x = -uc; y = vc; z = 1.0; break;
  }
  const double n = sqrt(x * x + y * y + z * z);
  d[0] = x / n; d[1] = y / n; d[2] = z / n;
}

/* L[k][c] = sum_texels f_c * Y_k(w) * dA,  dA = (uc^2+vc^2+1)^(-3/2) * 4/S^2
 * (the cube projection of device_functions/sh.h:59-103).  L_abs accumulates
 * |f_c * Y_k * dA| (error scale for tests), may be NULL. */
void orc_sh_project_f64(const float* faces, int S, int lmax, double* L, double* L_abs) {
  const int nc = (lmax + 1) * (lmax + 1);
  double Y[(ORC_MAX_LAYERS + 1) * (ORC_MAX_LAYERS + 1)];
  memset(L, 0, sizeof(double) * nc * 3);
  if (L_abs) memset(L_abs, 0, sizeof(double) * nc * 3);
  for (int f = 0; f < 6; ++f)
    for (int r = 0; r < S; ++r)
      for (int c = 0; c < S; ++c) {
        const double uc = 2.0 * (c + 0.5) / S - 1.0, vc = 2.0 * (r + 0.5) / S - 1.0;
        double d[3];
        face_dir(f, uc, vc, d);
        orc_sh_eval_f64(d[0], d[1], d[2], lmax, Y);
        const double q = uc * uc + vc * vc + 1.0;
        const double dA = 1.0 / (q * sqrt(q)) * (4.0 / ((double)S * S));
        const float* t = faces + (((int64_t)f * S + r) * S + c) * 3;
        for (int k = 0; k < nc; ++k)
          for (int ch = 0; ch < 3; ++ch) {
            const double v = (double)t[ch] * Y[k] * dA;
            L[k * 3 + ch] += v;
            if (L_abs) L_abs[k * 3 + ch] += fabs(v);
          }
      }
}

/* out_px = |sum_j T[px][j] * L[j]| per channel (the per-pixel form of
 * devicePrograms.cu:479-490; abs as at :490), fmaf in j order. */
void orc_sh_dot_f32(const float* T, int64_t N, int nc, const float* L, int abs_out,
                    float* out4, int n_threads) {
  set_threads(n_threads);
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < N; ++p) {
    float a0 = 0.f, a1 = 0.f, a2 = 0.f;
    const float* t = T + p * nc;
    for (int j = 0; j < nc; ++j) {
      a0 = fmaf(t[j], L[j * 3 + 0], a0);
      a1 = fmaf(t[j], L[j * 3 + 1], a1);
      a2 = fmaf(t[j], L[j * 3 + 2], a2);
    }
    if (abs_out) { a0 = fabsf(a0); a1 = fabsf(a1); a2 = fabsf(a2); }
    out4[p * 4 + 0] = a0; out4[p * 4 + 1] = a1; out4[p * 4 + 2] = a2; out4[p * 4 + 3] = 1.0f;
  }
}

void orc_sh_dot_f64(const float* T, int64_t N, int nc, const double* L, int abs_out, double* out3) {
  for (int64_t p = 0; p < N; ++p) {
    double a[3] = {0, 0, 0};
    for (int j = 0; j < nc; ++j)
      for (int c = 0; c < 3; ++c) a[c] += (double)T[p * nc + j] * L[j * 3 + c];
    for (int c = 0; c < 3; ++c) out3[p * 3 + c] = abs_out ? fabs(a[c]) : a[c];
  }
}

/* ------------------------------------------------------------------------ */
/* Relight                                                                   */
/* ------------------------------------------------------------------------ */

/* ln(x) of a float, evaluated in double by the atanh series
 *   ln m = 2 artanh((m-1)/(m+1)) = 2 (s + s^3/3 + s^5/5 + ...)   (Abramowitz & Stegun 4.1.27)
 * after the reduction x = 2^e m, m in [sqrt(1/2), sqrt(2)], and rounded once to float.
 * Only IEEE double +, -, *, / and fma in a fixed order, so the GPU's copy of this
 * routine (relight_common.cu) returns the same bits; its result is the correctly rounded
 * float logarithm except in rare ties.  Used for the roughness remap in place of logf,
 * whose last bit differs between C libraries and the GPU. */
float orc_logf_series(float xf) {
  if (xf != xf) return xf;
  if (xf < 0.0f) return NAN;
  if (xf == 0.0f) return -INFINITY;
  if (isinf(xf)) return xf;
  double x = (double)xf;
  uint64_t b;
  memcpy(&b, &x, 8);
  int e = (int)((b >> 52) & 0x7ff) - 1023;
  b = (b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL;
  double m;
  memcpy(&m, &b, 8);
  if (m > 1.4142135623730951) { m = m * 0.5; e += 1; }
  const double s = (m - 1.0) / (m + 1.0);
  const double z = s * s;
  double p = 1.0 / 23.0;
  p = fma(p, z, 1.0 / 21.0);
  p = fma(p, z, 1.0 / 19.0);
  p = fma(p, z, 1.0 / 17.0);
  p = fma(p, z, 1.0 / 15.0);
  p = fma(p, z, 1.0 / 13.0);
  p = fma(p, z, 1.0 / 11.0);
  p = fma(p, z, 1.0 / 9.0);
  p = fma(p, z, 1.0 / 7.0);
  p = fma(p, z, 1.0 / 5.0);
  p = fma(p, z, 1.0 / 3.0);
  p = fma(p, z, 1.0);
  const double lm = (2.0 * s) * p;
  return (float)fma((double)e, 0.6931471805599453, lm);
}

/* x^y = exp(y ln x) in IEEE double, rounded once to float: the logarithm by the atanh
 * series of orc_logf_series (Abramowitz & Stegun 4.1.27), the exponential by reduction
 * t = k ln2 + r, |r| <= ln2/2, and the Taylor series of e^r up to r^18.  The reference's
 * final-colour pass calls powf (Renderer/toneMap.cu:33-39,61); this is the restatement
 * the library evaluates on host and device. */
float orc_powf_series(float xf, float yf) {
  if (xf != xf || xf < 0.0f) return NAN;
  if (xf == 0.0f) return 0.0f;
  if (isinf(xf)) return xf;
  double x = (double)xf;
  uint64_t b;
  memcpy(&b, &x, 8);
  int e = (int)((b >> 52) & 0x7ff) - 1023;
  b = (b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL;
  double m;
  memcpy(&m, &b, 8);
  if (m > 1.4142135623730951) { m = m * 0.5; e += 1; }
  const double s = (m - 1.0) / (m + 1.0);
  const double z = s * s;
  double p = 1.0 / 23.0;
  p = fma(p, z, 1.0 / 21.0);
  p = fma(p, z, 1.0 / 19.0);
  p = fma(p, z, 1.0 / 17.0);
  p = fma(p, z, 1.0 / 15.0);
  p = fma(p, z, 1.0 / 13.0);
  p = fma(p, z, 1.0 / 11.0);
  p = fma(p, z, 1.0 / 9.0);
  p = fma(p, z, 1.0 / 7.0);
  p = fma(p, z, 1.0 / 5.0);
  p = fma(p, z, 1.0 / 3.0);
  p = fma(p, z, 1.0);
  const double lm = (2.0 * s) * p;
  const double t = fma((double)e, 0.6931471805599453, lm) * (double)yf;
  const double kd = floor(fma(t, 1.4426950408889634, 0.5));
  const double r = fma(-kd, 0.6931471805599453, t);
  /* 1/n! for n = 18 .. 0 */
  static const double inv_fact[19] = {
      1.0 / 6402373705728000.0, 1.0 / 355687428096000.0, 1.0 / 20922789888000.0, 1.0 / 1307674368000.0,
      1.0 / 87178291200.0, 1.0 / 6227020800.0, 1.0 / 479001600.0, 1.0 / 39916800.0, 1.0 / 3628800.0,
      1.0 / 362880.0, 1.0 / 40320.0, 1.0 / 5040.0, 1.0 / 720.0, 1.0 / 120.0, 1.0 / 24.0, 1.0 / 6.0,
      0.5, 1.0, 1.0};
  double q = inv_fact[0];
  for (int i = 1; i < 19; ++i) q = fma(q, r, inv_fact[i]);
  return (float)ldexp(q, (int)kd);
}

/* One linear channel -> byte, Renderer/toneMap.cu:57-69: f = 1.055 (x + 1e-6)^(1/2.4) - 0.055
 * (the multiply-subtract contracted to one fma, as nvcc compiles it), clamped to [0, 1] with
 * NaN -> 0, times 255.9, truncated. */
static uint32_t orc_srgb_byte(float x) {
  const float coeff = 1.055f;
  const float p = orc_powf_series(x + 1e-6f, 1.0f / 2.4f);
  float f = fmaf(coeff, p, -(coeff - 1.0f));
  f = f > 0.0f ? f : 0.0f;
  f = f < 1.0f ? f : 1.0f;
  return (uint32_t)(f * 255.9f);
}

/* computeFinalPixelColorsKernel (Renderer/toneMap.cu:47-71): float4 -> r | g<<8 | b<<16 | 255<<24. */
void orc_tonemap_srgb(const float* src, int64_t n, uint32_t* dst) {
  for (int64_t i = 0; i < n; ++i)
    dst[i] = orc_srgb_byte(src[i * 4]) | (orc_srgb_byte(src[i * 4 + 1]) << 8) |
             (orc_srgb_byte(src[i * 4 + 2]) << 16) | (255u << 24);
}

/* The 255 step thresholds of orc_srgb_byte: t[j] = the smallest float x >= 0 whose byte is
 * >= j, by bisection over the ordered bit patterns of non-negative floats. */
void orc_srgb_thresholds(float* t) {
  t[0] = 0.0f;
  for (int j = 1; j < 256; ++j) {
    uint32_t lo = 0, hi = 0x7f800000u;
    while (lo < hi) {
      const uint32_t mid = lo + (hi - lo) / 2;
      float x;
      memcpy(&x, &mid, 4);
      if (orc_srgb_byte(x) >= (uint32_t)j) hi = mid;
      else lo = mid + 1;
    }
    memcpy(&t[j], &lo, 4);
  }
}

/* Floats within `radius` ulps of every threshold (and all negative/NaN/inf specials) whose
 * byte from the threshold count differs from the direct evaluation: 0 means the step table
 * and the formula agree wherever the byte can change. */
int64_t orc_srgb_threshold_mismatches(const float* t, int radius) {
  int64_t bad = 0;
  for (int j = 1; j < 256; ++j) {
    uint32_t c;
    memcpy(&c, &t[j], 4);
    for (int64_t d = -radius; d <= radius; ++d) {
      const int64_t b = (int64_t)c + d;
      if (b < 0 || b > 0x7f800000LL) continue;
      const uint32_t ub = (uint32_t)b;
      float x;
      memcpy(&x, &ub, 4);
      uint32_t k = 0;
      for (int i = 1; i < 256; ++i) k += t[i] <= x;
      bad += k != orc_srgb_byte(x);
    }
  }
  return bad;
}

/* SH shading of mesh vertices (Renderer/device_functions/devicePrograms.cu:476-486):
 * light[k] = sum_j T[v][k][j] L[j] accumulated with one fma per term in j order
 * (lightResponse[k] += T * light_vector[j]), then c = sum_k light[k] * brdf[v][k] in k order
 * (colorTriangleVertices += lightResponse * brdf), and its absolute value per channel. */
void orc_sh_vertex_radiance(const float* T, const float* brdf, const float* L, int64_t V, int n, float* out) {
  for (int64_t v = 0; v < V; ++v) {
    const float* t = T + v * (int64_t)n * n;
    const float* b = brdf + v * (int64_t)n * 3;
    float c[3] = {0.f, 0.f, 0.f};
    for (int k = 0; k < n; ++k) {
      float l[3] = {0.f, 0.f, 0.f};
      for (int j = 0; j < n; ++j)
        for (int ch = 0; ch < 3; ++ch) l[ch] = fmaf(t[k * n + j], L[j * 3 + ch], l[ch]);
      for (int ch = 0; ch < 3; ++ch) c[ch] = fmaf(l[ch], b[k * 3 + ch], c[ch]);
    }
    for (int ch = 0; ch < 3; ++ch) out[v * 3 + ch] = fabsf(c[ch]);
  }
}

/* Barycentric pixel colour (devicePrograms.cu:488-490): ((1 - u) - v) c0 + u c1 + v c2 as
 * fma(v, c2, fma(u, c1, w c0)); output float4 (rgb, 1).  Returns the number of pixels whose
 * triangle named a vertex outside [0, V) (those read (0, 0, 0, 1)). */
int64_t orc_sh_interpolate(const float* vc, int64_t V, const int32_t* tri, const float* uv, int64_t P, float* out) {
  int64_t bad = 0;
  for (int64_t p = 0; p < P; ++p) {
    const int32_t i0 = tri[p * 3], i1 = tri[p * 3 + 1], i2 = tri[p * 3 + 2];
    float* o = out + p * 4;
    o[3] = 1.f;
    if (i0 < 0 || i1 < 0 || i2 < 0 || i0 >= V || i1 >= V || i2 >= V) {
      o[0] = o[1] = o[2] = 0.f;
      ++bad;
      continue;
    }
    const float u = uv[p * 2], w = uv[p * 2 + 1];
    const float b0 = (1.f - u) - w;
    for (int ch = 0; ch < 3; ++ch)
      o[ch] = fmaf(w, vc[i2 * 3 + ch], fmaf(u, vc[i1 * 3 + ch], b0 * vc[i0 * 3 + ch]));
  }
  return bad;
}

/* The reference's per-pixel 16-float input row (waveletDataCopy,
 * utils_kernels.h:7-49; layout prt_globals.h:4-13):
 * pos(3) normal(3) reflect(3) log(25r+1)/log(26) 2kd-1(3) 2ks-1(3). */
void orc_remap_f32(const orc_gbuf* g, int64_t px, float row[16]) {
  const float rgh_den = 1.f / orc_logf_series(25.f + 1.f);
  for (int i = 0; i < 3; ++i) {
    row[0 + i] = g->pos[px * 4 + i];
    row[3 + i] = g->normal[px * 4 + i];
    row[6 + i] = g->reflect[px * 4 + i];
    row[10 + i] = 2.f * g->kd[px * 4 + i] - 1.f;
    row[13 + i] = 2.f * g->ks[px * 4 + i] - 1.f;
  }
  row[9] = orc_logf_series(fmaf(25.f, g->roughness[px], 1.f)) * rgh_den;
}

static float clamp01f(float x) { return fminf(fmaxf(x, 0.f), 1.f); }

/* Per level l: x_l = x * N_l, corner i0 = min(floor(x_l), N_l - 1), weight
 * w = x_l - i0.  Vertex (i,j,k) of the (N_l+1)^3 lattice indexes the level's
 * table densely (i + j(N+1) + k(N+1)^2) when the lattice fits, else by the
 * Instant-NGP spatial hash (i*1 ^ j*2654435761 ^ k*805459861) mod T.
 * Corner c: bit0 -> x, bit1 -> y, bit2 -> z; weight ((wx*wy)*wz);
 * features accumulated with fmaf in corner order. */
static void hash_corner_setup(const orc_net* net, int l, const float pos[3], uint32_t i0[3],
                              float w[3]) {
  const int N = net->level_res[l];
  for (int d = 0; d < 3; ++d) {
    const float xl = clamp01f(pos[d]) * (float)N;
    int i = (int)floorf(xl);
    if (i > N - 1) i = N - 1;
    i0[d] = (uint32_t)i;
    w[d] = xl - (float)i;
  }
}

static uint32_t hash_index(const orc_net* net, int l, uint32_t x, uint32_t y, uint32_t z) {
  const uint32_t N1 = (uint32_t)net->level_res[l] + 1u;
  const uint32_t T = (uint32_t)net->level_size[l];
  const uint64_t V = (uint64_t)N1 * N1 * N1;
  if (V <= (uint64_t)T) return x + y * N1 + z * N1 * N1;
  return (x ^ (y * 2654435761u) ^ (z * 805459861u)) & (T - 1u);
}

void orc_hash_encode_f32(const orc_net* net, const float* hash, const float pos[3], float* out) {
  const int F = net->n_features;
  for (int l = 0; l < net->n_levels; ++l) {
    uint32_t i0[3];
    float w[3];
    hash_corner_setup(net, l, pos, i0, w);
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int c = 0; c < 8; ++c) {
      const int bx = c & 1, by = (c >> 1) & 1, bz = (c >> 2) & 1;
      const float wx = bx ? w[0] : 1.f - w[0];
      const float wy = by ? w[1] : 1.f - w[1];
      const float wz = bz ? w[2] : 1.f - w[2];
      const float wc = (wx * wy) * wz;
      const uint32_t e = hash_index(net, l, i0[0] + bx, i0[1] + by, i0[2] + bz);
      const float* th = hash + ((int64_t)net->level_offset[l] + e) * F;
      for (int f = 0; f < F; ++f) acc[f] = fmaf(wc, th[f], acc[f]);
    }
    for (int f = 0; f < F; ++f) out[l * F + f] = acc[f];
  }
}

void orc_hash_encode_f64(const orc_net* net, const float* hash, const float pos[3], double* out) {
  const int F = net->n_features;
  for (int l = 0; l < net->n_levels; ++l) {
    uint32_t i0[3];
    float w[3];
    hash_corner_setup(net, l, pos, i0, w);
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int c = 0; c < 8; ++c) {
      const int bx = c & 1, by = (c >> 1) & 1, bz = (c >> 2) & 1;
      const double wx = bx ? w[0] : 1.0 - w[0];
      const double wy = by ? w[1] : 1.0 - w[1];
      const double wz = bz ? w[2] : 1.0 - w[2];
      const uint32_t e = hash_index(net, l, i0[0] + bx, i0[1] + by, i0[2] + bz);
      const float* th = hash + ((int64_t)net->level_offset[l] + e) * F;
      for (int f = 0; f < F; ++f) acc[f] += wx * wy * wz * (double)th[f];
    }
    for (int f = 0; f < F; ++f) out[l * F + f] = acc[f];
  }
}

/* y = act(W x) with W given transposed, Wt[i][out]; every y_j accumulates
 * fmaf(W[j][i], x_i, .) from 0 in ascending i (the GPU FP32 kernel's order).  The
 * j loop is innermost so the compiler vectorises across outputs without changing
 * any output's operation sequence. */
static void dense_f32(const float* Wt, int n_in, int n_out, const float* x, float* y, int relu) {
  float acc[ORC_MAX_WIDTH];
  for (int j = 0; j < n_out; ++j) acc[j] = 0.f;
  for (int i = 0; i < n_in; ++i) {
    const float xi = x[i];
    const float* wr = Wt + (int64_t)i * n_out;
    for (int j = 0; j < n_out; ++j) acc[j] = fmaf(wr[j], xi, acc[j]);
  }
  for (int j = 0; j < n_out; ++j) y[j] = relu ? fmaxf(acc[j], 0.f) : acc[j];
}

/* Transposes each row-major [out][in] layer of a network to [in][out]. */
static float* transpose_layers(const float* W, int nl, const int* in, const int* out) {
  size_t n = 0;
  for (int l = 0; l < nl; ++l) n += (size_t)in[l] * out[l];
  float* t = (float*)malloc(sizeof(float) * (n ? n : 1));
  size_t o = 0;
  for (int l = 0; l < nl; ++l) {
    for (int j = 0; j < out[l]; ++j)
      for (int i = 0; i < in[l]; ++i) t[o + (size_t)i * out[l] + j] = W[o + (size_t)j * in[l] + i];
    o += (size_t)in[l] * out[l];
  }
  return t;
}

static void dense_f64(const float* W, int n_in, int n_out, const double* x, double* y, int relu) {
  for (int j = 0; j < n_out; ++j) {
    double acc = 0.0;
    const float* wr = W + (int64_t)j * n_in;
    for (int i = 0; i < n_in; ++i) acc += (double)wr[i] * x[i];
    y[j] = relu ? (acc > 0.0 ? acc : 0.0) : acc;
  }
}

static int net_ok(const orc_net* net) {
  if (net->n_levels * net->n_features > ORC_MAX_WIDTH) return 0;
  if (net->op_nl < 1 || net->cn_nl < 1 || net->op_nl > ORC_MAX_LAYERS || net->cn_nl > ORC_MAX_LAYERS)
    return 0;
  for (int i = 0; i < net->op_nl; ++i)
    if (net->op_in[i] > ORC_MAX_WIDTH || net->op_out[i] > ORC_MAX_WIDTH) return 0;
  for (int i = 0; i < net->cn_nl; ++i)
    if (net->cn_in[i] > ORC_MAX_WIDTH || net->cn_out[i] > ORC_MAX_WIDTH) return 0;
  if (net->cn_out[net->cn_nl - 1] != 3) return 0;
  if (net->cn_in[0] != net->op_out[net->op_nl - 1] + net->aux_width) return 0;
  return 1;
}

/* Transport of one pixel from its 16-float input row (the layout of prt_globals.h:4-13). */
static void transport_f32_row(const orc_net* net, const orc_weights* w, const float* op_t,
                              const float* cn_t, const float row[16], const int32_t* idx, int K,
                              float* out) {
  float enc[ORC_MAX_WIDTH], aux[ORC_MAX_WIDTH];
  float xa[ORC_MAX_WIDTH], xb[ORC_MAX_WIDTH];
  orc_hash_encode_f32(net, w->hash, row, enc);
  for (int i = 0; i < net->aux_width; ++i) aux[i] = i < 13 ? row[3 + i] : 1.0f;
  const int D = net->n_levels * net->n_features;
  const int op_out = net->op_out[net->op_nl - 1];
  for (int k = 0; k < K; ++k) {
    for (int d = 0; d < D; ++d) xa[d] = enc[d] * w->emb[(int64_t)d * net->n_coeffs + idx[k]];
    const float* W = op_t;
    float *x = xa, *y = xb, *t;
    for (int li = 0; li < net->op_nl; ++li) {
      dense_f32(W, net->op_in[li], net->op_out[li], x, y, li < net->op_nl - 1);
      W += (int64_t)net->op_in[li] * net->op_out[li];
      t = x; x = y; y = t;
    }
    for (int i = 0; i < net->aux_width; ++i) x[op_out + i] = aux[i];
    W = cn_t;
    for (int li = 0; li < net->cn_nl; ++li) {
      dense_f32(W, net->cn_in[li], net->cn_out[li], x, y, li < net->cn_nl - 1);
      W += (int64_t)net->cn_in[li] * net->cn_out[li];
      t = x; x = y; y = t;
    }
    out[k * 3 + 0] = x[0]; out[k * 3 + 1] = x[1]; out[k * 3 + 2] = x[2];
  }
}

static void transport_f32_t(const orc_net* net, const orc_weights* w, const float* op_t,
                            const float* cn_t, const orc_gbuf* g, int64_t px, const int32_t* idx,
                            int K, float* out) {
  float row[16];
  orc_remap_f32(g, px, row);
  transport_f32_row(net, w, op_t, cn_t, row, idx, K, out);
}

int orc_transport_f32(const orc_net* net, const orc_weights* w, const orc_gbuf* g, int64_t px,
                      const int32_t* idx, int K, float* out) {
  if (!net_ok(net)) return -1;
  float* op_t = transpose_layers(w->op, net->op_nl, net->op_in, net->op_out);
  float* cn_t = transpose_layers(w->cn, net->cn_nl, net->cn_in, net->cn_out);
  transport_f32_t(net, w, op_t, cn_t, g, px, idx, K, out);
  free(op_t);
  free(cn_t);
  return 0;
}

int orc_transport_f64(const orc_net* net, const orc_weights* w, const orc_gbuf* g, int64_t px,
                      const int32_t* idx, int K, double* out) {
  if (!net_ok(net)) return -1;
  float row[16];
  double enc[ORC_MAX_WIDTH], aux[ORC_MAX_WIDTH], xa[ORC_MAX_WIDTH], xb[ORC_MAX_WIDTH];
  orc_remap_f32(g, px, row);
  /* remap in FP64 for the accuracy reference */
  double row64[16];
  for (int i = 0; i < 3; ++i) {
    row64[0 + i] = g->pos[px * 4 + i];
    row64[3 + i] = g->normal[px * 4 + i];
    row64[6 + i] = g->reflect[px * 4 + i];
    row64[10 + i] = 2.0 * g->kd[px * 4 + i] - 1.0;
    row64[13 + i] = 2.0 * g->ks[px * 4 + i] - 1.0;
  }
  row64[9] = log(25.0 * (double)g->roughness[px] + 1.0) / log(26.0);
  orc_hash_encode_f64(net, w->hash, row, enc);
  for (int i = 0; i < net->aux_width; ++i) aux[i] = i < 13 ? row64[3 + i] : 1.0;
  const int D = net->n_levels * net->n_features;
  const int op_out = net->op_out[net->op_nl - 1];
  for (int k = 0; k < K; ++k) {
    for (int d = 0; d < D; ++d) xa[d] = enc[d] * (double)w->emb[(int64_t)d * net->n_coeffs + idx[k]];
    const float* W = w->op;
    double *x = xa, *y = xb, *t;
    for (int li = 0; li < net->op_nl; ++li) {
      dense_f64(W, net->op_in[li], net->op_out[li], x, y, li < net->op_nl - 1);
      W += (int64_t)net->op_in[li] * net->op_out[li];
      t = x; x = y; y = t;
    }
    for (int i = 0; i < net->aux_width; ++i) x[op_out + i] = aux[i];
    W = w->cn;
    for (int li = 0; li < net->cn_nl; ++li) {
      dense_f64(W, net->cn_in[li], net->cn_out[li], x, y, li < net->cn_nl - 1);
      W += (int64_t)net->cn_in[li] * net->cn_out[li];
      t = x; x = y; y = t;
    }
    out[k * 3 + 0] = x[0]; out[k * 3 + 1] = x[1]; out[k * 3 + 2] = x[2];
  }
  return 0;
}

/* Radiance sum of computeResponse (utils_kernels.h:52-91): only pixels whose
 * env-map flag is set get sum_k max(L_k * T_k, 0); indirect = (rgb, 1),
 * with_direct = (rgb + direct.rgb, 1). */
static int relight_f32_impl(const orc_net* net, const orc_weights* w, const orc_gbuf* g,
                            const float* rows, const int32_t* idx, const float* strength, int K,
                            int clamp, int kahan, int64_t px_begin, int64_t px_end, int n_threads,
                            float* indirect4, float* with_direct4) {
  if (!net_ok(net) || K < 0) return -1;
  int bad = 0;
  set_threads(n_threads);
  float* op_t = transpose_layers(w->op, net->op_nl, net->op_in, net->op_out);
  float* cn_t = transpose_layers(w->cn, net->cn_nl, net->cn_in, net->cn_out);
#pragma omp parallel reduction(| : bad)
  {
    float* T = (float*)malloc(sizeof(float) * 3 * (K > 0 ? K : 1));
#pragma omp for schedule(dynamic, 8)
    for (int64_t p = px_begin; p < px_end; ++p) {
      float s[3] = {0.f, 0.f, 0.f}, comp[3] = {0.f, 0.f, 0.f};
      if (g->flag[p]) {
        if (rows)
          transport_f32_row(net, w, op_t, cn_t, rows + (p - px_begin) * 16, idx, K, T);
        else
          transport_f32_t(net, w, op_t, cn_t, g, p, idx, K, T);
        for (int k = 0; k < K; ++k)
          for (int c = 0; c < 3; ++c) {
            float term = strength[k * 3 + c] * T[k * 3 + c];
            if (clamp) term = fmaxf(term, 0.0f);
            if (kahan) {
              const float y = term - comp[c];
              const float t = s[c] + y;
              comp[c] = (t - s[c]) - y;
              s[c] = t;
            } else {
              s[c] += term;
            }
          }
      }
      for (int c = 0; c < 3; ++c) {
        indirect4[p * 4 + c] = s[c];
        with_direct4[p * 4 + c] = s[c] + g->direct[p * 4 + c];
      }
      indirect4[p * 4 + 3] = 1.0f;
      with_direct4[p * 4 + 3] = 1.0f;
    }
    free(T);
  }
  free(op_t);
  free(cn_t);
  return bad ? -1 : 0;
}

int orc_relight_f32(const orc_net* net, const orc_weights* w, const orc_gbuf* g,
                    const int32_t* idx, const float* strength, int K, int clamp, int kahan,
                    int64_t px_begin, int64_t px_end, int n_threads,
                    float* indirect4, float* with_direct4) {
  return relight_f32_impl(net, w, g, NULL, idx, strength, K, clamp, kahan, px_begin, px_end,
                          n_threads, indirect4, with_direct4);
}

int orc_relight_rows_f32(const orc_net* net, const orc_weights* w, const orc_gbuf* g,
                         const float* rows, const int32_t* idx, const float* strength, int K,
                         int clamp, int kahan, int64_t px_begin, int64_t px_end, int n_threads,
                         float* indirect4, float* with_direct4) {
  if (!rows) return -1;
  return relight_f32_impl(net, w, g, rows, idx, strength, K, clamp, kahan, px_begin, px_end,
                          n_threads, indirect4, with_direct4);
}

int orc_relight_f64(const orc_net* net, const orc_weights* w, const orc_gbuf* g,
                    const int32_t* idx, const float* strength, int K, int clamp,
                    int64_t px_begin, int64_t px_end, int n_threads, double* rgb3) {
  if (!net_ok(net) || K < 0) return -1;
  int bad = 0;
  set_threads(n_threads);
#pragma omp parallel reduction(| : bad)
  {
    double* T = (double*)malloc(sizeof(double) * 3 * (K > 0 ? K : 1));
#pragma omp for schedule(dynamic, 8)
    for (int64_t p = px_begin; p < px_end; ++p) {
      double s[3] = {0, 0, 0};
      if (g->flag[p]) {
        if (orc_transport_f64(net, w, g, p, idx, K, T) != 0) bad = 1;
        for (int k = 0; k < K; ++k)
          for (int c = 0; c < 3; ++c) {
            double term = (double)strength[k * 3 + c] * T[k * 3 + c];
            if (clamp && term < 0.0) term = 0.0;
            s[c] += term;
          }
      }
      for (int c = 0; c < 3; ++c) rgb3[(p - px_begin) * 3 + c] = s[c];
    }
    free(T);
  }
  return bad ? -1 : 0;
}

/* ------------------------------------------------------------------------ */
/* Env-map rotation (point-sampled cubemap lookup, cubeMap.cu:23-113)        */
/* ------------------------------------------------------------------------ */

/* dst texel (f, r, c) = src texel seen in direction R^T d, d = EnvUVToDirec of the
 * texel centre (unnormalised), face/uv by EnvDirecToUV with its six tests applied in
 * order (a later match overrides), point sampling with wrap addressing.  FP32 ops
 * without contraction, in the same order as the GPU kernel. */
void orc_env_rotate(const float* src, int S, const float R[9], float* dst) {
  const float fs = (float)S;
  for (int f = 0; f < 6; ++f)
    for (int r = 0; r < S; ++r)
      for (int c = 0; c < S; ++c) {
        const float uc = 2.f * (((float)c + 0.5f) / fs) - 1.f;
        const float vc = 2.f * (((float)r + 0.5f) / fs) - 1.f;
        float x, y, z;
        switch (f) {
          case 0: x = 1.f; y = vc; z = uc; break;
          case 1: x = -1.f; y = vc; z = -uc; break;
          case 2: x = uc; y = 1.f; z = vc; break;
          case 3: x = uc; y = -1.f; z = -vc; break;
          case 4: x = uc; y = vc; z = -1.f; break;
          default: x = -uc; y = vc; z = 1.f; break;
        }
        const float sx = (R[0] * x + R[3] * y) + R[6] * z;
        const float sy = (R[1] * x + R[4] * y) + R[7] * z;
        const float sz = (R[2] * x + R[5] * y) + R[8] * z;
        const float ax = fabsf(sx), ay = fabsf(sy), az = fabsf(sz);
        float maxa = 1.f, su = 0.f, sv = 0.f;
        int sf = 0;
        if (sx > 0.f && ax >= ay && ax >= az) { maxa = ax; su = sz; sv = sy; sf = 0; }
        if (!(sx > 0.f) && ax >= ay && ax >= az) { maxa = ax; su = -sz; sv = sy; sf = 1; }
        if (sy > 0.f && ay >= ax && ay >= az) { maxa = ay; su = sx; sv = sz; sf = 2; }
        if (!(sy > 0.f) && ay >= ax && ay >= az) { maxa = ay; su = sx; sv = -sz; sf = 3; }
        if (!(sz > 0.f) && az >= ax && az >= ay) { maxa = az; su = sx; sv = sy; sf = 4; }
        if (sz > 0.f && az >= ax && az >= ay) { maxa = az; su = -sx; sv = sy; sf = 5; }
        if (!(maxa > 0.f)) { maxa = 1.f; su = -1.f; sv = -1.f; sf = 0; }
        const float u = 0.5f * (su / maxa + 1.f);
        const float v = 0.5f * (sv / maxa + 1.f);
        int col = (int)floorf(u * fs) % S;
        int row = (int)floorf(v * fs) % S;
        if (col < 0) col += S;
        if (row < 0) row += S;
        const float* s = src + (((int64_t)sf * S + row) * S + col) * 3;
        float* d = dst + (((int64_t)f * S + r) * S + c) * 3;
        d[0] = s[0]; d[1] = s[1]; d[2] = s[2];
      }
}

// me_device.cuh -- device functions of the per-pixel Milne-Eddington inversion.
//
// Everything here is written for sm_100a and templated on the synthesis type
// T (float for the FP32 path, double for the FP64 path).  The 9x9 SVD solve
// and the chi^2 accept test are always FP64.
//
// Reference functions restated (HaoLi-70/Milne-Eddington, Src/):
//   voigt / voigt_alg916 / voigt_hui6 / voigt_humlicek_w4 / erfcx / dawson
//       FADDEEVA.c:440-590, 286-402, 112-163, 167-281, 83-108, 29-79
//   me_point               ME_SOLVER.c:101-366 (one wavelength of Milne_Eddington_Single)
//   bounds_fold            ME_SOLVER.c:370-406 (bounds_check)
//   init_guess             ME_SOLVER.c:445-676 (Init_Guess)
//   gr_svd / gr_backsub    SVD_TEMPLATE.h:49-406 (svdcmp / svbksb, Golub-Reinsch)
//   svd_solve              LM_FIT.c:400-469 (SVD_solve_mem)
//   restart draws          LM_FIT.c:157-201 (Random_Jump) with per-(pixel, run)
//                          Philox4x32-10 draws instead of a process-wide stream
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <type_traits>

#include "../../include/me_b200.h"

namespace me {

constexpr double kPi = 3.14159265358979323846;
constexpr double kLightSpeed = 299792458.0;
constexpr double kSqrtPi = 1.77245385090551588191;
constexpr int kMaxNl = 512;

// Plan constants the kernels read (passed by value as a kernel parameter).
struct DevPlan {
  int nl, ncut, ic, i0, i1, npar;
  int nfigures, row, fnmax;
  int niter, nruns, hmi_ref, regul_any;
  int fixed[9], regul[9];
  int free_idx[9];  // reduced index -> full parameter index
  // variant of the one-thread-per-slot Jacobian and trial kernels (pixels
  // per CTA, grid staging, reciprocal table; me_kernels.h kKernelVariants)
  int kvar;
  // SVD solves with all nine parameters free: 0 = matrix in shared memory,
  // 1 = in registers (svd9_kernel) in the one-thread-per-slot rounds, 2 = in
  // registers in the lane-split rounds as well
  int svd_regs;
  // Faddeeva evaluation of the FP32 syntheses: 0 = the reference's regions
  // and Alg-916, 1 = Weideman's 16-term rational series (FP64 plans: 0)
  int faddeeva;
  // Givens rotations of the SVD's QR sweeps from one reciprocal square root
  // (givens_radius<true>; FP32 plans) or as the reference forms them (FP64)
  int fastg;
  double lambda0, bshift;
  double limits[9][2];
  double step[9];
  double w2[4], weights[4];
  double icriteria, convg, chisq_crit, damp, lam_accept, lam_reject, lam_lim[2], svd_thr;
  double vcoeffi, lcoeffi;
  double regul_value[9], regul_weight[9];
  unsigned long long seed;
  // Alg-916 constants (Faddeeva_init, FADDEEVA.c:406-436)
  double fa, faa, flog_rmin0, fsqrt_log_rmin0;
  double exp_a2n2[50];
  double thr[5];  // |z|^2 region boundaries of this Nfigures row
  const double *lambda;   // [nl] wavelength grid [A]
  const double *dlambda;  // [nl] lambda - lambda0 [A]
  // instrument filter (no reference counterpart): observed wavelength i is
  // sum_k sub_w[k] * synthesis at flambda[i * nsub + k]; nsub = 1: none
  int nsub;
  double sub_w[ME_MAX_FILTER];
  const double *flambda;   // [nl * nsub] sub-wavelengths [A]
  const double *fdlambda;  // [nl * nsub] minus lambda0 [A]
};

// ---------------------------------------------------------------------------
// precision-generic math
// ---------------------------------------------------------------------------
__device__ __forceinline__ float m_exp(float x) { return expf(x); }
__device__ __forceinline__ double m_exp(double x) { return exp(x); }
__device__ __forceinline__ float m_sin(float x) { return sinf(x); }
__device__ __forceinline__ double m_sin(double x) { return sin(x); }
__device__ __forceinline__ float m_cos(float x) { return cosf(x); }
__device__ __forceinline__ double m_cos(double x) { return cos(x); }
__device__ __forceinline__ float m_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double m_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float m_erfc(float x) { return erfcf(x); }
__device__ __forceinline__ double m_erfc(double x) { return erfc(x); }
__device__ __forceinline__ float m_abs(float x) { return fabsf(x); }
__device__ __forceinline__ double m_abs(double x) { return fabs(x); }
__device__ __forceinline__ float m_round(float x) { return roundf(x); }
__device__ __forceinline__ double m_round(double x) { return round(x); }
__device__ __forceinline__ float m_copysign(float a, float b) { return copysignf(a, b); }
__device__ __forceinline__ double m_copysign(double a, double b) { return copysign(a, b); }
__device__ __forceinline__ void m_sincos(float x, float *s, float *c) { sincosf(x, s, c); }
__device__ __forceinline__ void m_sincos(double x, double *s, double *c) { sincos(x, s, c); }

// ---------------------------------------------------------------------------
// Voigt H(nu, a) and Faraday-Voigt L(nu, a) = Re, Im of w(nu + i a)
// ---------------------------------------------------------------------------
constexpr int kRden = 32;  // reciprocal table 1 / (a^2 n^2 + y^2), n < kRden

template <class T>
struct VoigtK {
  T a, aa, inv_a, log_rmin0, sqrt_log_rmin0;
  T ema2, em2a2;  // exp(-a^2), exp(-2 a^2)
  int nmax, nfig;
  int weid;  // FP32: Weideman's series (voigt_weideman_f32) in place of the regions
  T thr[5];
  const T *ea2n2;  // exp(-a^2 n^2), n = 0..49 (shared memory, per block)
  const T *e2an;   // exp(-2 a^2 n), n = 0..49 (shared memory, per block)
  // per synthesis (FP32 path): y = damping and this thread's reciprocal table
  T yy, inv_y;
  const T *rden;   // rden[n * rstride] = 1 / (a^2 n^2 + y^2)
  int rstride;
};

// Fills the y-dependent part of K for one synthesis at damping y.  On the FP32
// path every Alg-916 series term 1 / (a^2 n^2 + y^2) then comes from this
// thread's table instead of a division (the damping is one number per
// synthesis).  `rden` is this thread's base in shared memory, stride `stride`.
template <class T>
__device__ __forceinline__ void voigt_prepare(VoigtK<T> &K, T y, T *rden, int stride) {
  K.yy = y * y;
  K.inv_y = T(1) / y;
  K.rden = rden;
  K.rstride = stride;
  if (sizeof(T) == sizeof(float) && rden && !K.weid) {
#pragma unroll 4
    for (int n = 0; n < kRden; n++) rden[n * stride] = T(1) / (K.aa * T(n * n) + K.yy);
  }
}

// (H, L) pair returned by the Voigt evaluators.
template <class T>
struct HL {
  T h, l;
};

// erfcx(a) = exp(a^2) erfc(a) with the a > 26.6 asymptotic series (FADDEEVA.c:83-108).
template <class T>
__device__ __forceinline__ T erfcx_t(T a) {
  if (a > T(26.6)) {
    T a2 = a * a;
    return ((((((T(162.421875) / a2 - T(29.53125)) / a2 + T(6.5625)) / a2 - T(1.875)) / a2 +
              T(0.75)) / a2 - T(0.5)) / a2 + T(1)) / T(kSqrtPi) / a;
  }
  return m_exp(a * a) * m_erfc(a);
}

// Dawson's integral by Rybicki's method (FADDEEVA.c:29-79); only reached for a == 0.
// Out of line, like the two evaluators below that the default accuracy row
// (Nfigures 6, damping below 1) never reaches: the synthesis kernels' hot code
// stays smaller, and their instruction fetch stalls less.
template <class T>
__device__ __noinline__ T dawson_t(T x) {
  const T H = T(0.4);
  T ax = m_abs(x);
  if (ax < T(0.2)) {
    T x2 = x * x;
    return x * (T(1) - T(2.0 / 3.0) * x2 * (T(1) - T(0.4) * x2 * (T(1) - T(2.0 / 7.0) * x2)));
  }
  int n0 = 2 * (int)m_round(ax / (2 * H));
  T xp = ax - n0 * H;
  T e1 = m_exp(T(2) * xp * H);
  T e2 = e1 * e1;
  T d1 = T(n0 + 1);
  T d2 = d1 - T(2);
  T sum = 0;
#pragma unroll
  for (int i = 1; i <= 6; i++) {
    T t = (T(2) * i - T(1)) * H;
    sum += m_exp(-t * t) * (e1 / d1 + T(1) / (d2 * e1));
    d1 += T(2);
    d2 -= T(2);
    e1 *= e2;
  }
  return T(0.5641895835) * m_copysign(m_exp(-xp * xp), x) * sum;
}

// Hui, Armstrong & Wray (1978) 6-pole rational approximation (FADDEEVA.c:112-163).
template <class T>
__device__ __noinline__ HL<T> voigt_hui6(T nu, T y) {
  const T A[7] = {T(122.607931777104326), T(214.382388694706425), T(181.928533092181549),
                  T(93.155580458138441),  T(30.180142196210589),  T(5.912626209773153),
                  T(0.564189583562615)};
  const T B[7] = {T(122.60793177387535),  T(352.730625110963558), T(457.334478783897737),
                  T(348.703917719495792), T(170.354001821091472), T(53.992906912940207),
                  T(10.479857114260399)};
  const T zr = y, zi = -nu;
  T pr = A[6], pi = 0, qr = B[6] + zr, qi = zi;
#pragma unroll
  for (int k = 5; k >= 0; k--) {
    T tr = pr * zr - pi * zi + A[k];
    T ti = pr * zi + pi * zr;
    pr = tr;
    pi = ti;
    tr = qr * zr - qi * zi + B[k];
    ti = qr * zi + qi * zr;
    qr = tr;
    qi = ti;
  }
  T den = qr * qr + qi * qi;
  return {(pr * qr + pi * qi) / den, (pi * qr - pr * qi) / den};
}

// Humlicek (1982) W4 (FADDEEVA.c:167-281).  Reached only for Nfigures <= 5.
template <class T>
__device__ __noinline__ HL<T> voigt_humlicek_w4(T nu, T y) {
  T H, L;
  const T anu = m_abs(nu);
  const T s = anu + y;
  const T tr = y, ti = -nu;
  if (s >= T(15)) {
    T ur = tr * tr - ti * ti, ui = T(2) * tr * ti;
    T dr = T(0.5) + ur, di = ui;
    T den = dr * dr + di * di;
    H = T(0.56418958355) * (tr * dr + ti * di) / den;
    L = T(0.56418958355) * (ti * dr - tr * di) / den;
  } else if (s >= T(5.5)) {
    T ur = tr * tr - ti * ti, ui = T(2) * tr * ti;
    T nr = T(1.4104739589) + T(0.5641896) * ur, ni = T(0.5641896) * ui;
    T dr = T(0.75) + T(3) * ur + (ur * ur - ui * ui);
    T di = T(3) * ui + T(2) * ur * ui;
    T den = dr * dr + di * di;
    T qr = (nr * dr + ni * di) / den, qi = (ni * dr - nr * di) / den;
    H = tr * qr - ti * qi;
    L = tr * qi + ti * qr;
  } else if (y >= T(1.95) * anu - T(0.176)) {
    const T c[5] = {T(0.5642236), T(3.778987), T(11.96482), T(20.20933), T(16.4955)};
    const T d[6] = {T(1.0), T(6.699398), T(21.69274), T(39.27121), T(38.82363), T(16.4955)};
    T nr = c[0], ni = 0, dr = d[0], di = 0;
    for (int k = 1; k < 5; k++) {
      T r = nr * tr - ni * ti + c[k], i = nr * ti + ni * tr;
      nr = r;
      ni = i;
    }
    for (int k = 1; k < 6; k++) {
      T r = dr * tr - di * ti + d[k], i = dr * ti + di * tr;
      dr = r;
      di = i;
    }
    T den = dr * dr + di * di;
    H = (nr * dr + ni * di) / den;
    L = (ni * dr - nr * di) / den;
  } else {
    const T c[7] = {T(0.5641900381), T(1.320521697), T(35.7668278), T(219.0312964),
                    T(1540.786893),  T(3321.990492), T(36183.30536)};
    const T d[8] = {T(1),           T(1.841438936), T(61.57036588), T(364.2190727),
                    T(2186.181081), T(9022.227659), T(24322.84021), T(32066.59372)};
    T ur = tr * tr - ti * ti, ui = T(2) * tr * ti;
    T eu = m_exp(ur), sn, cs;
    m_sincos(ui, &sn, &cs);
    T er = eu * cs, ei = eu * sn;
    T nr = c[0], ni = 0, dr = d[0], di = 0;
    for (int k = 1; k < 7; k++) {
      T r = -(nr * ur - ni * ui) + c[k], i = -(nr * ui + ni * ur);
      nr = r;
      ni = i;
    }
    T r = nr * tr - ni * ti, i = nr * ti + ni * tr;
    nr = r;
    ni = i;
    for (int k = 1; k < 8; k++) {
      r = -(dr * ur - di * ui) + d[k];
      i = -(dr * ui + di * ur);
      dr = r;
      di = i;
    }
    T den = dr * dr + di * di;
    H = er - (nr * dr + ni * di) / den;
    L = ei - (ni * dr - nr * di) / den;
  }
  return {H, L};
}

// FP32 form of Alg 916 with the same series, terms and cut-offs, arranged for
// the GPU: the 1 / (a^2 n^2 + y^2) factors come from the per-synthesis table;
// with d_b = x - a n_b and d_f = a - d_b (n_f = n_b + 1), exp(-d_f^2) and
// exp(-2 a d_f) follow from exp(-d_b^2) and exp(-2 a d_b) and the constants
// exp(-a^2), exp(-2 a^2); exp(-2 a x) = exp(-2 a^2 n_b) exp(-2 a d_b); and
// 2 a x sin(xy)^2 / (xy pi) = 2 a sin(xy)^2 / (y pi).
__device__ __forceinline__ HL<float> voigt_alg916_f32(float nu, float y, float erfcx_y,
                                                      const VoigtK<float> &K) {
  if (nu == 0.f) return {erfcx_y, 0.f};
  if (y == 0.f) return {expf(-nu * nu), float(2.0 / kSqrtPi) * dawson_t(nu)};
  const float x = fabsf(nu), ya = fabsf(y);
  if (x + ya > 1e7f) {
    if (x < ya) {
      const float xs = __fdividef(x, ya), r = __fdividef(float(1.0 / kSqrtPi), xs * xs + 1.f);
      return {r, xs * r};
    }
    const float ys = __fdividef(ya, x), r = __fdividef(float(1.0 / kSqrtPi), ys * ys + 1.f);
    return {ys * r, r};
  }
  const float a = K.a;
  const float xx = x * x, xy = x * y;
  float sxy, cxy;
  sincosf(xy, &sxy, &cxy);
  const float s2 = 2.f * sxy * cxy;
  const float c2 = (cxy - sxy) * (cxy + sxy);
  const float exx = expf(-xx);
  const float k1 = exx * erfcx_y;
  const float r2 = K.log_rmin0 - xx;
  const int nmax1 = r2 >= 0.f ? (int)(sqrtf(r2) * K.inv_a + 0.5f) : -2147483647;
  const int nmax2 = (int)((K.sqrt_log_rmin0 - x) * K.inv_a + 0.5f);
  int nmax = nmax1 > nmax2 ? nmax1 : nmax2;
  if (nmax >= K.nmax) nmax = K.nmax - 1;
  const int nb = (int)(x * K.inv_a + 0.5f);
  const int nf = nb + 1;
  const float dxb = x - a * nb;
  const float dxf = a - dxb;
  int nmaxf = (int)((K.sqrt_log_rmin0 - dxf) * K.inv_a);
  int nmaxb = (int)((K.sqrt_log_rmin0 - dxb) * K.inv_a);
  if (nmaxf >= K.nmax) nmaxf = K.nmax - 1;
  if (nmaxb >= K.nmax) nmaxb = K.nmax - 1;
  const int nlo = (nb - nmaxb) > 1 ? (nb - nmaxb) : 1;
  const float inv_pi = float(1.0 / kPi);
  const float ay = a * K.inv_y * inv_pi * exx;
  float re = k1 * c2 + 2.f * ay * sxy * sxy;
  float im = -k1 * s2 + ay * s2;
  const float e1b = expf(-dxb * dxb);
  const float e2b = expf(-2.f * a * dxb);
  const float ie2b = __fdividef(1.f, e2b);
  const float e1f = K.ema2 * e1b * ie2b;
  const float e2f = K.em2a2 * ie2b;
  // 1 / (a^2 n^2 + y^2): from the per-synthesis table, or (no table) the
  // same correctly rounded reciprocal computed in place
  auto rd = [&](int n) {
    if (n < kRden) return K.rden ? K.rden[n * K.rstride] : 1.f / (K.aa * float(n * n) + K.yy);
    return __fdividef(1.f, K.aa * float(n * n) + K.yy);
  };
  float s1 = 0.f, s2s = 0.f, s3 = 0.f, s4 = 0.f, s5 = 0.f, ep = 1.f;
  for (int n = nf; n <= nf + nmaxf; n++) {
    const float t = e1f * K.ea2n2[n - nf] * rd(n) * ep;
    s3 += t;
    s5 += t * float(n);
    ep *= e2f;
  }
  ep = 1.f;
  for (int n = nb; n >= nlo; n--) {
    const float t = e1b * K.ea2n2[nb - n] * rd(n) * ep;
    s3 += t;
    s5 += t * float(n);
    ep *= e2b;
  }
  re += a * y * s3 * inv_pi;
  im += a * a * s5 * inv_pi;
  if (x < K.sqrt_log_rmin0 || x < 10.f) {
    const float q = (nb < 50 ? K.e2an[nb] : expf(-2.f * K.aa * nb)) * e2b;  // exp(-2 a x)
    ep = 1.f;
    for (int n = 1; n <= nmax; n++) {
      const float t = exx * K.ea2n2[n] * rd(n);
      s1 += t;
      ep *= q;
      s2s += t * ep;
      s4 += t * ep * float(n);
    }
    re += a * y * (-2.f * c2 * s1 + s2s) * inv_pi;
    im += a * (2.f * y * s2 * s1 - a * s4) * inv_pi;
  }
  return {re, nu > 0.f ? im : -im};
}

template <class T>
__device__ __forceinline__ HL<T> voigt_alg916(T nu, T y, T erfcx_y, const VoigtK<T> &K) {
  if constexpr (sizeof(T) == sizeof(float)) return voigt_alg916_f32(nu, y, erfcx_y, K);
  if (nu == T(0)) {
    return {erfcx_y, T(0)};
  } else if (y == T(0)) {
    return {m_exp(-nu * nu), T(2.0 / kSqrtPi) * dawson_t(nu)};
  }
  const T x = m_abs(nu), ya = m_abs(y);
  if (x + ya > T(1e7)) {
    if (x < ya) {
      T xs = x / ya;
      return {T(1) / T(kSqrtPi) / (xs * xs + T(1)), xs / T(kSqrtPi) / (xs * xs + T(1))};
    }
    T ys = ya / x;
    return {ys / T(kSqrtPi) / (ys * ys + T(1)), T(1) / T(kSqrtPi) / (ys * ys + T(1))};
  }
  const T xx = x * x, yy = y * y, xy = x * y;
  const T xy2 = T(2) * xy;
  T sin_xy, cos_xy;
  m_sincos(xy, &sin_xy, &cos_xy);
  // sin(2xy), cos(2xy) by the double-angle identities
  const T sin_2xy = T(2) * sin_xy * cos_xy;
  const T cos_2xy = (cos_xy - sin_xy) * (cos_xy + sin_xy);
  const T exp_xx = m_exp(-xx);
  const T k1 = exp_xx * erfcx_y;
  const T a = K.a;
  int nmax1 = (int)(m_sqrt(K.log_rmin0 - x * x) / a + T(0.5));
  if (!(K.log_rmin0 - x * x >= T(0))) nmax1 = -2147483647;  // sqrt(<0) = NaN -> INT_MIN in C
  const int nmax2 = (int)((K.sqrt_log_rmin0 - x) / a + T(0.5));
  int nmax = nmax1 > nmax2 ? nmax1 : nmax2;
  if (nmax >= K.nmax) nmax = K.nmax - 1;
  const int nb = (int)(x / a + T(0.5));
  const int nf = nb + 1;
  const T dxf = a * nf - x;
  const T dxb = x - a * nb;
  int nmaxf = (int)((K.sqrt_log_rmin0 - dxf) / a);
  int nmaxb = (int)((K.sqrt_log_rmin0 - dxb) / a);
  if (nmaxf >= K.nmax) nmaxf = K.nmax - 1;
  if (nmaxb >= K.nmax) nmaxb = K.nmax - 1;
  const int nlo = (nb - nmaxb) > 1 ? (nb - nmaxb) : 1;
  const T inv_pi = T(1.0 / kPi);
  T re = k1 * cos_2xy + T(2) * a * x * sin_xy * exp_xx * sin_xy / xy * inv_pi;
  T im = -k1 * sin_2xy + T(2) * a * x * exp_xx * sin_2xy / xy2 * inv_pi;
  T s1 = 0, s2 = 0, s3 = 0, s4 = 0, s5 = 0;
  T e1 = m_exp(-dxf * dxf);
  T e2 = m_exp(T(-2) * a * dxf);
  T ep = 1;
  for (int n = nf; n <= nf + nmaxf; n++) {
    T t = e1 * K.ea2n2[n - nf] / (K.aa * T(n * n) + yy);
    s3 += t * ep;
    s5 += t * ep * a * T(n);
    ep *= e2;
  }
  e1 = m_exp(-dxb * dxb);
  e2 = m_exp(T(-2) * a * dxb);
  ep = 1;
  for (int n = nb; n >= nlo; n--) {
    T t = e1 * K.ea2n2[nb - n] / (K.aa * T(n * n) + yy);
    s3 += t * ep;
    s5 += t * ep * a * T(n);
    ep *= e2;
  }
  re += a * y * s3 * inv_pi;
  im += a * s5 * inv_pi;
  if (x < K.sqrt_log_rmin0 || x < T(10)) {
    const T q = m_exp(T(-2) * a * x);  // 1 / exp(2 a x)
    ep = 1;
    for (int n = 1; n <= nmax; n++) {
      T t = exp_xx * K.ea2n2[n] / (K.aa * T(n * n) + yy);
      s1 += t;
      ep *= q;
      s2 += t * ep;
      s4 += t * ep * a * T(n);
    }
    re += a * y * (T(-2) * cos_2xy * s1 + s2) * inv_pi;
    im += a * (T(2) * y * sin_2xy * s1 - s4) * inv_pi;
  }
  return {re, nu > T(0) ? im : -im};
}

// Weideman's rational series for the Faddeeva function (J. A. C. Weideman,
// "Computation of the complex error function", SIAM J. Numer. Anal. 31 (1994)
// 1497-1518) with N = 16 terms, for Im z >= 0:
//   L = (N / sqrt 2)^(1/2),  d = L - i z,  Z = (L + i z) / d,
//   w(z) = 2 p(Z) / d^2 + 1 / (sqrt(pi) d),  p(Z) = sum_{n < N} c_n Z^n,
// where c_1..c_N (here c_0..c_15) are the real parts of the discrete Fourier
// transform (length 4N, divided by 4N) of f(t) = exp(-t^2) (L^2 + t^2) sampled
// at t = L tan(theta / 2), theta = k pi / (2N), k = -2N+1 .. 2N-1, as the
// paper constructs them.  In FP32 the result is within 6e-7 of w for every
// z with Im z >= 0 (the evaluation's rounding; the series' own error at
// N = 16 is 1.3e-7): no branch, one reciprocal, 4N multiply-adds.  The
// coefficients, highest power first (me_weideman16 returns them to tests):
#define ME_WEIDEMAN16_L 3.36358566101485856f
#define ME_WEIDEMAN16(X)                                                               \
  X(15, 9.939322536e-07f) X(14, 3.981287575e-06f) X(13, -5.584233411e-06f)            \
  X(12, -2.734640462e-05f) X(11, 2.170986793e-05f) X(10, 2.107105640e-04f)             \
  X(9, 8.703158428e-05f) X(8, -1.527659740e-03f) X(7, -3.881015189e-03f)               \
  X(6, 3.682567317e-03f) X(5, 5.182240243e-02f) X(4, 1.912417267e-01f)                 \
  X(3, 4.692909009e-01f) X(2, 8.864478302e-01f) X(1, 1.362240822e+00f)                 \
  X(0, 1.748395886e+00f)

__device__ __forceinline__ HL<float> voigt_weideman_f32(float nu, float y) {
  constexpr float L = ME_WEIDEMAN16_L;
  // 1 / d = conj(d) / |d|^2 with d = (L + y) - i nu
  const float dre = L + y;
  const float r = __fdividef(1.f, fmaf(dre, dre, nu * nu));
  const float ire = dre * r, iim = nu * r;
  // Z = (L + i z) / d, L + i z = (L - y) + i nu
  const float nre = L - y;
  const float zre = fmaf(nre, ire, -nu * iim), zim = fmaf(nre, iim, nu * ire);
  float pre = 0.f, pim = 0.f;
#define ME_WEID_STEP(n, c)                                   \
  {                                                          \
    const float t = fmaf(pre, zre, fmaf(-pim, zim, c));      \
    pim = fmaf(pre, zim, pim * zre);                         \
    pre = t;                                                 \
  }
  ME_WEIDEMAN16(ME_WEID_STEP)
#undef ME_WEID_STEP
  // 2 p / d^2 + (1 / sqrt(pi)) / d
  const float i2re = fmaf(ire, ire, -iim * iim), i2im = 2.f * ire * iim;
  const float rsp = float(1.0 / kSqrtPi);
  const float h = fmaf(2.f, fmaf(pre, i2re, -pim * i2im), ire * rsp);
  const float l = fmaf(2.f, fmaf(pre, i2im, pim * i2re), iim * rsp);
  return {h, l};
}

// Reciprocal: the MUFU approximation on the FP32 path (<= 2 ulp), exact
// division in FP64.
__device__ __forceinline__ float rcp_t(float x) { return __fdividef(1.f, x); }
__device__ __forceinline__ double rcp_t(double x) { return 1.0 / x; }

template <class T>
__device__ __forceinline__ HL<T> voigt(T nu, T y, T erfcx_y, const VoigtK<T> &K) {
  if constexpr (sizeof(T) == sizeof(float)) {
    if (K.weid) return voigt_weideman_f32(nu, y);
  }
  T H, L;
  if (nu == T(0)) {
    return {erfcx_y, T(0)};
  } else if (y == T(0)) {
    return {m_exp(-nu * nu), T(2.0 / kSqrtPi) * dawson_t(nu)};
  }
  const T zr = nu, zi = y;
  const T z2r = zr * zr - zi * zi;
  const T z2i = T(2) * zr * zi;
  const T r2 = zr * zr + zi * zi;
  const T y2 = y * y;
  if (r2 >= K.thr[0]) {
    const T rden = rcp_t(T(kSqrtPi) * r2);
    H = zi * rden;
    L = zr * rden;
  } else if (r2 >= K.thr[1]) {
    T wr = z2r - T(0.5);
    const T rden = rcp_t(T(kSqrtPi) * (wr * wr + z2i * z2i));
    H = (-zi * wr + zr * z2i) * rden;
    L = (zr * wr + zi * z2i) * rden;
  } else if (r2 >= K.thr[2]) {
    T wr = z2r - T(1.5);
    T pr = wr * zr - z2i * zi, pi = wr * zi + z2i * zr;
    const T rden = rcp_t(T(kSqrtPi) * (pr * pr + pi * pi));
    wr = z2r - T(1);
    H = (-z2i * pr + wr * pi) * rden;
    L = (wr * pr + z2i * pi) * rden;
  } else if (r2 >= K.thr[3]) {
    if ((K.nfig <= 4 && y2 < T(6e-14)) || (K.nfig == 5 && r2 < T(39) && y2 < T(1e-9))) {
      return voigt_humlicek_w4(nu, y);
    }
    T wr = z2r - T(2.5);
    T ar = -(wr * zi + z2i * zr), ai = wr * zr - z2i * zi;
    wr = z2r - T(3);
    T br = wr * z2r - z2i * z2i + T(0.75), bi = (wr + z2r) * z2i;
    const T rden = rcp_t(T(kSqrtPi) * (br * br + bi * bi));
    H = (ar * br + ai * bi) * rden;
    L = (-ar * bi + ai * br) * rden;
  } else if (r2 >= K.thr[4]) {
    if (K.nfig <= 4) {
      if (y2 < T(0.026))
        return voigt_humlicek_w4(nu, y);
      else
        return voigt_hui6(nu, y);
    } else if (K.nfig == 5) {
      if (y2 >= T(0.27))
        return voigt_hui6(nu, y);
      else if (y2 >= T(1e-9))
        return voigt_alg916(nu, y, erfcx_y, K);
      else
        return voigt_humlicek_w4(nu, y);
    } else if (K.nfig == 6) {
      if (y2 >= T(1))
        return voigt_hui6(nu, y);
      else
        return voigt_alg916(nu, y, erfcx_y, K);
    }
    T wr = z2r - T(4.5);
    T ar = -(wr + z2r) * z2i, ai = wr * z2r - z2i * z2i + T(2);
    wr = z2r - T(5);
    T br = wr * z2r - z2i * z2i + T(3.75), bi = (wr + z2r) * z2i;
    T cr = br * zr - bi * zi, ci = br * zi + bi * zr;
    T den = T(kSqrtPi) * (cr * cr + ci * ci);
    H = (ar * cr + ai * ci) / den;
    L = (-ar * ci + ai * cr) / den;
  } else {
    if (K.nfig <= 4)
      return voigt_hui6(nu, y);
    else
      return voigt_alg916(nu, y, erfcx_y, K);
  }
  return {H, L};
}


// Block-wide Voigt tables in shared memory (s_tab: [100] = exp(-a^2 n^2), then
// exp(-2 a^2 n)) and the per-block constants; call once per block (syncs).
template <class T>
__device__ __forceinline__ void voigt_block_setup(VoigtK<T> &K, const DevPlan &P, T *s_tab) {
  for (int i = threadIdx.x; i < 50; i += blockDim.x) {
    s_tab[i] = T(P.exp_a2n2[i]);
    s_tab[50 + i] = T(exp(-2.0 * P.faa * i));
  }
  __syncthreads();
  K.a = T(P.fa);
  K.aa = T(P.faa);
  K.inv_a = T(1.0 / P.fa);
  K.log_rmin0 = T(P.flog_rmin0);
  K.sqrt_log_rmin0 = T(P.fsqrt_log_rmin0);
  K.ema2 = T(exp(-P.faa));
  K.em2a2 = T(exp(-2.0 * P.faa));
  K.nmax = P.fnmax;
  K.nfig = P.nfigures;
  K.weid = sizeof(T) == sizeof(float) && P.faddeeva == 1;
#pragma unroll
  for (int i = 0; i < 5; i++) K.thr[i] = T(P.thr[i]);
  K.ea2n2 = s_tab;
  K.e2an = s_tab + 50;
  K.rden = nullptr;
  K.rstride = 0;
  K.yy = T(0);
  K.inv_y = T(0);
}

// ---------------------------------------------------------------------------
// Milne-Eddington synthesis at one wavelength (ME_SOLVER.c:189-362)
// ---------------------------------------------------------------------------
template <class T>
struct SynthCall {
  T p4, p5, p6, p7, p8, inv_p4, inv_p6;
  T eta_half, b0, b1, bsh_n, lam_n;
  T sth, cth, sth2, cth2p1, c2p, s2p, kq, ku, kt, kv;
  T shift_b, vshift;  // Zeeman and Doppler shifts
  T erfcx_y;
  T step[9];
  // the observed (or, with a filter, sub-) wavelength grid staged in shared
  // memory as shift_w reads it, or null: read through the L1 cache
  const T *grid;
};

template <class T>
__device__ __forceinline__ void synth_setup(SynthCall<T> &c, const double *mp, const DevPlan &P,
                                            const double *step) {
  c.p4 = T(mp[4]);
  c.p5 = T(mp[5]);
  c.p6 = T(mp[6]);
  c.p7 = T(mp[7]);
  c.p8 = T(mp[8]);
  c.inv_p4 = T(1.0 / mp[4]);
  c.inv_p6 = T(1.0 / mp[6]);
  c.eta_half = T(0.5) * c.p6;
  c.b0 = c.p7 * c.p8;
  c.b1 = c.p7 - c.b0;
  c.bsh_n = T(P.bshift / mp[4]);
  c.lam_n = T(P.lambda0 / mp[4]);
  double s1, c1, s2, c2;
  sincos(mp[1], &s1, &c1);
  sincos(2. * mp[2], &s2, &c2);
  c.sth = T(s1);
  c.cth = T(c1);
  c.sth2 = c.sth * c.sth;
  c.cth2p1 = c.cth * c.cth + T(1);
  c.c2p = T(c2);
  c.s2p = T(s2);
  c.kq = c.eta_half * c.sth2 * c.c2p;
  c.ku = c.eta_half * c.sth2 * c.s2p;
  c.kt = c.eta_half * T(2) * c.sth * c.cth;
  c.kv = c.eta_half * c.cth;
  c.shift_b = T(mp[0] * (P.bshift / mp[4]));
  if (sizeof(T) == sizeof(double)) {
    // FP64: the reference's own form, ShiftW = 1e3 lambda / width + ShiftV
    // (Src/ME_SOLVER.c:160-161, 190)
    c.vshift = T(1e3 * (-1e3 * mp[3] / kLightSpeed * P.lambda0 - P.lambda0) / mp[4]);
  } else {
    // FP32: the same quantity without its cancellation,
    // ShiftW = (1e3 (lambda - lambda0) - 1e6 v lambda0 / c) / width
    c.vshift = T(1e6 * mp[3] * P.lambda0 / kLightSpeed);
  }
  c.erfcx_y = erfcx_t<T>(c.p5);
#pragma unroll
  for (int k = 0; k < 9; k++) c.step[k] = T(step[k]);
  c.grid = nullptr;
}

// The grid values shift_w / shift_wf read, for staging: FP32 the offsets from
// lambda0 converted to float, FP64 the wavelengths; entry i of the filter's
// sub-grid when it has one.
template <class T>
__device__ __forceinline__ T grid_value(const DevPlan &P, int i);
template <>
__device__ __forceinline__ float grid_value<float>(const DevPlan &P, int i) {
  return float(P.nsub > 1 ? P.fdlambda[i] : P.dlambda[i]);
}
template <>
__device__ __forceinline__ double grid_value<double>(const DevPlan &P, int i) {
  return P.nsub > 1 ? P.flambda[i] : P.lambda[i];
}

// Reduced wavelength of grid point iw.
template <class T>
__device__ __forceinline__ T shift_w(const SynthCall<T> &c, const DevPlan &P, int iw);
template <>
__device__ __forceinline__ float shift_w<float>(const SynthCall<float> &c, const DevPlan &P,
                                                int iw) {
  const float d = c.grid ? c.grid[iw] : float(__ldg(P.dlambda + iw));
  return (1e3f * d - c.vshift) * c.inv_p4;
}
template <>
__device__ __forceinline__ double shift_w<double>(const SynthCall<double> &c, const DevPlan &P,
                                                  int iw) {
  const double l = c.grid ? c.grid[iw] : __ldg(P.lambda + iw);
  return 1e3 * l / c.p4 + c.vshift;
}

// shift_w at sub-wavelength j of the instrument filter
template <class T>
__device__ __forceinline__ T shift_wf(const SynthCall<T> &c, const DevPlan &P, int j);
template <>
__device__ __forceinline__ float shift_wf<float>(const SynthCall<float> &c, const DevPlan &P,
                                                 int j) {
  const float d = c.grid ? c.grid[j] : float(__ldg(P.fdlambda + j));
  return (1e3f * d - c.vshift) * c.inv_p4;
}
template <>
__device__ __forceinline__ double shift_wf<double>(const SynthCall<double> &c, const DevPlan &P,
                                                   int j) {
  const double l = c.grid ? c.grid[j] : __ldg(P.flambda + j);
  return 1e3 * l / c.p4 + c.vshift;
}

// One wavelength of Milne_Eddington_Single.  syn[4] = I, Q, U, V.  With
// DERIV also J[s][k] = d syn_s / d p_k * step[k] * sw[s] (sw: per-Stokes
// weights the caller wants folded in, 1 for the plain Jacobian).
//
// The analytic Jacobian is organised by the chain rule: the Stokes vector
// depends on the parameters only through the seven absorption-matrix
// elements x = (eta_I, eta_Q, eta_U, eta_V, rho_Q, rho_U, rho_V), so
// J = G (dx/dp) with G = dS/dx (4 x 7) formed once per wavelength from the
// Unno-Rachkovsky solution, and dx/dp from the profile derivatives
// (LL04 9.110; the same derivatives as Src/ME_SOLVER.c:249-361, regrouped).
// The three Zeeman components are visited in a loop that accumulates their
// contributions, so the Voigt evaluation appears once in the code.
template <class T, bool DERIV>
__device__ __forceinline__ void me_point(const SynthCall<T> &c, T w0, const VoigtK<T> &K,
                                         const T sw[4], T syn[4], T J[4][9]) {
  const T rsp = T(1.0 / kSqrtPi);
  // sums over the components: "1" = pi (q = 0), "s" = half the sigma sum,
  // "d" = sigma_b - sigma_r; for the profiles and for the derivative slots
  // j = B, v, Doppler width, damping
  T f1 = 0, fs = 0, fd = 0, g1 = 0, gs = 0, gd = 0;
  T df1[4], dfs[4], dfd[4], dg1[4], dgs[4], dgd[4];
  if (DERIV) {
#pragma unroll
    for (int j = 0; j < 4; j++) df1[j] = dfs[j] = dfd[j] = dg1[j] = dgs[j] = dgd[j] = 0;
  }
#pragma unroll 1
  for (int k = 0; k < 3; k++) {
    const int q = k - 1;
    const T v = w0 + T(q) * c.shift_b;
    const HL<T> hl = voigt<T>(v, c.p5, c.erfcx_y, K);
    const T phi = hl.h * rsp, psi = hl.l * rsp;
    const T w1 = q == 0 ? T(1) : T(0);
    const T ws = q == 0 ? T(0) : T(0.5);
    const T wd = T(-q);  // +1 for sigma_b (q = -1), -1 for sigma_r
    f1 += w1 * phi;
    fs += ws * phi;
    fd += wd * phi;
    g1 += w1 * psi;
    gs += ws * psi;
    gd += wd * psi;
    if (DERIV) {
      const T dH = T(2) * (-v * hl.h + c.p5 * hl.l) * rsp;
      const T dL = T(-2) * (-rsp + c.p5 * hl.h + v * hl.l) * rsp;
      const T fac[3] = {T(q) * c.bsh_n, T(-1e6 / kLightSpeed) * c.lam_n, -v * c.inv_p4};
#pragma unroll
      for (int j = 0; j < 3; j++) {
        const T dp = fac[j] * dH, dq = fac[j] * dL;
        df1[j] += w1 * dp;
        dfs[j] += ws * dp;
        dfd[j] += wd * dp;
        dg1[j] += w1 * dq;
        dgs[j] += ws * dq;
        dgd[j] += wd * dq;
      }
      // d/da: dH/da = -dL/dv, dL/da = dH/dv
      df1[3] -= w1 * dL;
      dfs[3] -= ws * dL;
      dfd[3] -= wd * dL;
      dg1[3] += w1 * dH;
      dgs[3] += ws * dH;
      dgd[3] += wd * dH;
    }
  }
  const T phit = f1 - fs, psit = g1 - gs;
  T x[7];  // eta_I, eta_Q, eta_U, eta_V, rho_Q, rho_U, rho_V
  x[0] = c.eta_half * (f1 * c.sth2 + fs * c.cth2p1);
  x[1] = phit * c.kq;
  x[2] = phit * c.ku;
  x[3] = fd * c.kv;
  x[4] = psit * c.kq;
  x[5] = psit * c.ku;
  x[6] = gd * c.kv;
  const T a1 = T(1) + x[0];
  const T a1s = a1 * a1;
  const T e2 = x[1] * x[1] + x[2] * x[2] + x[3] * x[3];
  const T r2 = x[4] * x[4] + x[5] * x[5] + x[6] * x[6];
  const T er = x[1] * x[4] + x[2] * x[5] + x[3] * x[6];
  const T del = a1s * (a1s - e2 + r2) - er * er;
  const T idel = rcp_t(del);
  const T b1d = c.b1 * idel;
  // cc_s: (eta x rho) components of the solution
  const T cc[3] = {x[3] * x[5] - x[2] * x[6], x[1] * x[6] - x[3] * x[4],
                   x[2] * x[4] - x[1] * x[5]};
  T num[4];
  num[0] = a1 * (a1s + r2);
#pragma unroll
  for (int s = 0; s < 3; s++) num[s + 1] = a1s * x[1 + s] + a1 * cc[s] + x[4 + s] * er;
  syn[0] = c.b0 + b1d * num[0];
#pragma unroll
  for (int s = 1; s < 4; s++) syn[s] = -b1d * num[s];
  if (!DERIV) return;

  // G = dS/dx: dS_I = b1 (dnum0 - R0 dDel) / Del, dS_P = -b1 (dnum_P - R_P dDel) / Del
  T dDel[7];
  dDel[0] = T(2) * a1 * (T(2) * a1s - e2 + r2);
#pragma unroll
  for (int s = 0; s < 3; s++) {
    dDel[1 + s] = T(-2) * (a1s * x[1 + s] + er * x[4 + s]);
    dDel[4 + s] = T(2) * (a1s * x[4 + s] - er * x[1 + s]);
  }
  T G[4][7];
  {
    const T R0 = num[0] * idel;
    const T cI = b1d * sw[0];
    G[0][0] = cI * (T(3) * a1s + r2 - R0 * dDel[0]);
#pragma unroll
    for (int m = 1; m < 4; m++) G[0][m] = cI * (-R0 * dDel[m]);
#pragma unroll
    for (int m = 4; m < 7; m++) G[0][m] = cI * (T(2) * a1 * x[m] - R0 * dDel[m]);
  }
  // d cc_s / d eta_t and d cc_s / d rho_t (s, t over Q, U, V); cc_Q = eV rU - eU rV, ...
#pragma unroll
  for (int s = 0; s < 3; s++) {
    const T Rs = num[s + 1] * idel;
    const T cs = -b1d * sw[s + 1];
    const T es = x[1 + s], rs = x[4 + s];
    // d num_s / d a1
    G[s + 1][0] = cs * (T(2) * a1 * es + cc[s] - Rs * dDel[0]);
#pragma unroll
    for (int t = 0; t < 3; t++) {
      // d cc_s / d eta_t = eps(s, t, u) rho_u, d cc_s / d rho_t = -eps(s, t, u) eta_u
      T dce = 0, dcr = 0;
      const int u = 3 - s - t;
      if (s != t) {
        const T sgn = ((t - s + 3) % 3 == 1) ? T(-1) : T(1);
        dce = sgn * x[4 + u];
        dcr = -sgn * x[1 + u];
      }
      const T dne = (s == t ? a1s : T(0)) + a1 * dce + rs * x[4 + t];
      const T dnr = a1 * dcr + (s == t ? er : T(0)) + rs * x[1 + t];
      G[s + 1][1 + t] = cs * (dne - Rs * dDel[1 + t]);
      G[s + 1][4 + t] = cs * (dnr - Rs * dDel[4 + t]);
    }
  }

  // dx/dp for p = B, theta, phi, v, width, a, eta0, each scaled by step[p]
  T dx[7][7];
  {
    const int slot_k[4] = {0, 3, 4, 5};
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int k = slot_k[j];
      const T st = c.step[k];
      const T dpt = (df1[j] - dfs[j]) * st, dgt = (dg1[j] - dgs[j]) * st;
      dx[k][0] = c.eta_half * (df1[j] * c.sth2 + dfs[j] * c.cth2p1) * st;
      dx[k][1] = dpt * c.kq;
      dx[k][2] = dpt * c.ku;
      dx[k][3] = dfd[j] * c.kv * st;
      dx[k][4] = dgt * c.kq;
      dx[k][5] = dgt * c.ku;
      dx[k][6] = dgd[j] * c.kv * st;
    }
    const T s1 = c.step[1], s2 = c.step[2], s6 = c.step[6] * c.inv_p6;
    const T ptk = phit * c.kt * s1, gtk = psit * c.kt * s1;
    dx[1][0] = ptk;
    dx[1][1] = ptk * c.c2p;
    dx[1][2] = ptk * c.s2p;
    dx[1][3] = -c.eta_half * fd * c.sth * s1;
    dx[1][4] = gtk * c.c2p;
    dx[1][5] = gtk * c.s2p;
    dx[1][6] = -c.eta_half * gd * c.sth * s1;
    dx[2][0] = 0;
    dx[2][1] = T(-2) * x[2] * s2;
    dx[2][2] = T(2) * x[1] * s2;
    dx[2][3] = 0;
    dx[2][4] = T(-2) * x[5] * s2;
    dx[2][5] = T(2) * x[4] * s2;
    dx[2][6] = 0;
#pragma unroll
    for (int m = 0; m < 7; m++) dx[6][m] = x[m] * s6;
  }
#pragma unroll
  for (int s = 0; s < 4; s++) {
#pragma unroll
    for (int k = 0; k < 7; k++) {
      T acc = G[s][0] * dx[k][0];
#pragma unroll
      for (int m = 1; m < 7; m++) acc += G[s][m] * dx[k][m];
      J[s][k] = acc;
    }
  }
  // S = S0 + S1 and beta = S0 / S
  const T t7 = (T(1) - c.p8) * idel * c.step[7];
  J[0][7] = (c.p8 * c.step[7] + t7 * num[0]) * sw[0];
#pragma unroll
  for (int s = 1; s < 4; s++) J[s][7] = -t7 * num[s] * sw[s];
  const T t8 = c.p7 * idel * c.step[8];
  J[0][8] = (c.p7 * c.step[8] - t8 * num[0]) * sw[0];
#pragma unroll
  for (int s = 1; s < 4; s++) J[s][8] = t8 * num[s] * sw[s];
}

// One observed wavelength of the synthesis: me_point at it, or, with the
// instrument filter (FILT, P.nsub > 1), the weighted sum over its
// sub-wavelengths, in order from zero, of the profiles and Jacobian rows.
template <class T, bool DERIV, bool FILT>
__device__ __forceinline__ void channel_point(const SynthCall<T> &c, const DevPlan &P,
                                              const VoigtK<T> &K, const T sw[4], int iw, T syn[4],
                                              T (*J)[9]) {
  if constexpr (!FILT) {
    me_point<T, DERIV>(c, shift_w<T>(c, P, iw), K, sw, syn, J);
  } else {
#pragma unroll
    for (int s = 0; s < 4; s++) {
      syn[s] = T(0);
      if (DERIV)
#pragma unroll
        for (int k = 0; k < 9; k++) J[s][k] = T(0);
    }
    const int ns = P.nsub;
#pragma unroll 1
    for (int q = 0; q < ns; q++) {
      T ys[4], Jq[4][9];
      me_point<T, DERIV>(c, shift_wf<T>(c, P, iw * ns + q), K, sw, ys, DERIV ? Jq : nullptr);
      const T wq = T(P.sub_w[q]);
#pragma unroll
      for (int s = 0; s < 4; s++) {
        syn[s] += wq * ys[s];
        if (DERIV)
#pragma unroll
          for (int k = 0; k < 9; k++) J[s][k] += wq * Jq[s][k];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// bounds_check (ME_SOLVER.c:370-406)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double clampb(double x, double lo, double hi) {
  return x < lo ? lo : (x > hi ? hi : x);
}
__device__ __forceinline__ void bounds_fold(double *p, const DevPlan &P, double l70, double l71) {
  const double two_pi = 2.0 * kPi;
  p[0] = clampb(p[0], P.limits[0][0], P.limits[0][1]);
  double t = fmod(p[1], two_pi);
  if (t < 0) t += two_pi;
  if (t > kPi) t = two_pi - t;
  p[1] = t;
#pragma unroll
  for (int i = 3; i < 9; i++) {
    double lo = i == 7 ? l70 : P.limits[i][0];
    double hi = i == 7 ? l71 : P.limits[i][1];
    p[i] = clampb(p[i], lo, hi);
  }
  double ph = fmod(p[2], kPi);
  if (ph < 0.0) ph += kPi;
  p[2] = ph;
}

// ---------------------------------------------------------------------------
// Init_Guess (ME_SOLVER.c:445-676), FP64, one thread per pixel
// ---------------------------------------------------------------------------
struct PixelInit {
  double guess[9];
  double norm0, normp, l70, l71, step7;
};

// Returns 1 when mean(I) < Icriteria (or the mean is NaN), as Init_Guess /
// the INVERSION_MULTI gate.
static __device__ __noinline__ int init_guess(const double *prof, const DevPlan &P, PixelInit &o,
                                       bool nan_gate) {
  const int nw = P.nl;
  const double *pI = prof, *pQ = prof + nw, *pU = prof + 2 * nw, *pV = prof + 3 * nw;
  const double lam0 = P.lambda0;
  double isum = 0., imin = 1e10, qsum = 0., usum = 0., vsum = 0.;
  double imax = 0, lmax = 0., vmax = 0., vmin = 0.;
  int i_imin = 0, i_vmax = 0, i_vmin = 0;
  for (int iw = 0; iw < nw; iw++) {
    const double vi = pI[iw];
    if (imax < vi) imax = vi;
    if (imin > vi) {
      i_imin = iw;
      imin = vi;
    }
    isum += vi;
    qsum += fabs(pQ[iw]);
    usum += fabs(pU[iw]);
    vsum += fabs(pV[iw]);
  }
  for (int iw = P.i0; iw <= P.i1; iw++) {
    const double l = sqrt(pQ[iw] * pQ[iw] + pU[iw] * pU[iw]);
    if (lmax < l) lmax = l;
    if (vmin > pV[iw]) {
      i_vmin = iw;
      vmin = pV[iw];
    } else if (vmax < pV[iw]) {
      i_vmax = iw;
      vmax = pV[iw];
    }
  }
  const double imean = isum / nw;
  // Init_Guess tests only Imean < Icriteria; INVERSION_MULTI also rejects a
  // NaN mean before calling it (Src/LM_FIT.c:783)
  if ((nan_gate && isnan(imean)) || imean < P.icriteria) return 1;
  o.norm0 = 1e-2 * imean;
  o.norm0 *= o.norm0;
  const double is2 = isum * isum;
  o.normp = 1 + qsum * qsum / is2 * P.w2[1] + usum * usum / is2 * P.w2[2] +
            vsum * vsum / is2 * P.w2[3];
  lmax = 100 * lmax / imean;
  vmin = 100 * vmin / imean;
  vmax = 100 * vmax / imean;
  const bool ir_line = (lam0 > 15640 && lam0 < 15660);
  const double thr_v = ir_line ? 1.5 : 5.0;
  const double thr_l = ir_line ? 2.5 : 5.0;
  double blos = 0.;
  const double lv = 0.5 * (vmax - vmin);
  const double factor = imin > 0.9 * imax ? 2. : 1.;
  if (lv > 0.1) {
    blos = 20 + P.vcoeffi * lv * factor;
    if (i_vmin < i_vmax) blos = -blos;
  }
  double bpos = 100 + P.lcoeffi * lmax * factor;
  bpos = bpos < 2200 ? bpos : 2200;
  double *g = o.guess;
  double tmp = 0;
  if (lv > thr_v) {
    tmp = 0.5 * (P.lambda[i_vmin] + P.lambda[i_vmax]) - lam0;
  } else {
    bool found = false;
    // the reference reads pI[i_imin-2 .. i_imin+2] unchecked; out-of-grid
    // reads (grids with nl < 10) count as a failed minimum test here
    if (imin < 0.9 * imax && i_imin >= P.ncut && i_imin < nw - P.ncut && i_imin >= 2 &&
        i_imin + 2 <= nw - 1) {
      if (pI[i_imin - 1] < pI[i_imin - 2] && pI[i_imin] < pI[i_imin - 1] &&
          pI[i_imin] < pI[i_imin + 1] && pI[i_imin + 1] < pI[i_imin + 2]) {
        tmp = P.lambda[i_imin] - lam0;
        found = true;
      }
    }
    if (!found) {
      double lsum = 0, wsum = 0.;
      const int lo = (P.ic > 7) ? (P.ic - 7) : 0;
      const int hi = (P.ic + 7 < nw) ? (P.ic + 7) : (nw - 1);
      for (int iw = lo; iw <= hi; iw++) {
        const double d = (imax - pI[iw]);
        lsum += P.lambda[iw] * d;
        wsum += d;
      }
      tmp = lsum / wsum - lam0;
    }
  }
  g[3] = tmp / lam0 * kLightSpeed / 1e3;
  g[0] = sqrt(blos * blos + bpos * bpos);
  g[1] = acos(blos / g[0]);
  if (g[0] > 3000) g[0] = 3000;
  double wsum = 0., phi = 0.;
  for (int iw = P.i0; iw <= P.i1; iw++) {
    const double l = sqrt(pQ[iw] * pQ[iw] + pU[iw] * pU[iw]);
    if (l > thr_l) {
      double t = 0.5 * atan2(pU[iw], pQ[iw]);
      t = t > 0 ? t : kPi + t;
      phi += t * l;
      wsum += l;
    }
  }
  g[2] = (wsum > 2. * thr_l) ? phi / wsum : kPi / 2.;
  if (ir_line) {
    g[4] = 60.;
    g[5] = 0.5;
    g[6] = 15;
    g[8] = 0.7;
  } else if (g[0] > 1100) {
    g[4] = 20;
    g[5] = 0.5;
    g[6] = 20;
    g[8] = 0.3;
  } else {
    g[4] = 30;
    g[5] = 0.5;
    g[6] = 5;
    g[8] = 0.15;
  }
  g[7] = imax;
  o.l70 = imax * 0.6;
  o.l71 = imax * 1.4;
  o.step7 = imax * 0.1;
  bounds_fold(g, P, o.l70, o.l71);
  return 0;
}

// ---------------------------------------------------------------------------
// Golub-Reinsch SVD, FP64 (SVD_TEMPLATE.h:49-406).  a[n*n] -> U in place,
// w[n], v[n*n]; returns 1 when a bidiagonal entry needed more than 50 QR sweeps
// (the reference stops the program there).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double pythag_d(double a, double b) {
  const double aa = fabs(a), ab = fabs(b);
  const double mx = aa > ab ? aa : ab;
  if (mx == 0) return 0;
  if (mx < 1e150) return sqrt(a * a + b * b);
  const double mn = aa > ab ? ab : aa;
  const double r = mn / mx;
  return mx * sqrt(1.0 + r * r);
}

// The radius z = pythag(a, b) of a Givens rotation of the QR sweeps and its
// reciprocal 1 / z, from which the rotation's cosine and sine follow.  FAST:
// both from one reciprocal square root, z = q rsqrt(q) and 1 / z = rsqrt(q)
// with q = a^2 + b^2 -- each within two ulps of the correctly rounded square
// root and quotient, and a third of their dependent latency -- while q lies
// well inside the normal range; otherwise, and always when !FAST, pythag_d
// and a division, as the reference computes them.
template <bool FAST>
__device__ __forceinline__ double givens_radius(double a, double b, double &inv) {
  if constexpr (FAST) {
    const double q = a * a + b * b;
    if (q > 1e-290 && q < 1e290) {
      const double r = rsqrt(q);
      inv = r;
      return q * r;
    }
  }
  const double z = pythag_d(a, b);
  inv = 1.0 / z;
  return z;
}

// The chase's first rotation of each step: the reference divides by the
// radius (c = f / z, s = h / z, SVD_TEMPLATE.h:305-306); FAST multiplies by
// the reciprocal square root givens_radius gave.
template <bool FAST>
__device__ __forceinline__ void chase_cs(double f, double h, double z, double iz, double &c,
                                         double &s) {
  if constexpr (FAST) {
    c = f * iz;
    s = h * iz;
  } else {
    c = f / z;
    s = h / z;
  }
}

static __device__ __noinline__ int gr_svd(double *a, int n, double *w, double *v) {
#define A_(i, j) a[(i) * n + (j)]
#define V_(i, j) v[(i) * n + (j)]
  const int m = n;
  int l = 0, nm = 0;
  double anorm = 0., c, f, g = 0., h, s, scale = 0., x, y, z;
  double rv1[9];
  int hit = 0;
  for (int i = 0; i < n; i++) {
    l = i + 1;
    rv1[i] = scale * g;
    g = s = scale = 0.0;
    for (int k = i; k < m; k++) scale += fabs(A_(k, i));
    if (scale) {
      const double is = 1.0 / scale;
      for (int k = i; k < m; k++) {
        A_(k, i) *= is;
        s += A_(k, i) * A_(k, i);
      }
      f = A_(i, i);
      g = f >= 0 ? -sqrt(s) : sqrt(s);
      h = f * g - s;
      A_(i, i) = f - g;
      const double ih = 1.0 / h;
      for (int j = l; j < n; j++) {
        s = 0.0;
        for (int k = i; k < m; k++) s += A_(k, i) * A_(k, j);
        f = s * ih;
        for (int k = i; k < m; k++) A_(k, j) += f * A_(k, i);
      }
      for (int k = i; k < m; k++) A_(k, i) *= scale;
    }
    w[i] = scale * g;
    g = s = scale = 0.0;
    if (i != n - 1) {
      for (int k = l; k < n; k++) scale += fabs(A_(i, k));
      if (scale) {
        const double is = 1.0 / scale;
        for (int k = l; k < n; k++) {
          A_(i, k) *= is;
          s += A_(i, k) * A_(i, k);
        }
        f = A_(i, l);
        g = f >= 0 ? -sqrt(s) : sqrt(s);
        h = f * g - s;
        A_(i, l) = f - g;
        const double ih = 1.0 / h;
        for (int k = l; k < n; k++) rv1[k] = A_(i, k) * ih;
        for (int j = l; j < m; j++) {
          s = 0.0;
          for (int k = l; k < n; k++) s += A_(j, k) * A_(i, k);
          for (int k = l; k < n; k++) A_(j, k) += s * rv1[k];
        }
        for (int k = l; k < n; k++) A_(i, k) *= scale;
      }
    }
    const double t = fabs(w[i]) + fabs(rv1[i]);
    if (anorm < t) anorm = t;
  }
  for (int i = n - 1; i >= 0; i--) {
    if (i < n - 1) {
      if (g != 0.0) {
        for (int j = l; j < n; j++) V_(j, i) = (A_(i, j) / A_(i, l)) / g;
        for (int j = l; j < n; j++) {
          s = 0.0;
          for (int k = l; k < n; k++) s += A_(i, k) * V_(k, j);
          for (int k = l; k < n; k++) V_(k, j) += s * V_(k, i);
        }
      }
      for (int j = l; j < n; j++) V_(i, j) = V_(j, i) = 0.0;
    }
    V_(i, i) = 1.0;
    g = rv1[i];
    l = i;
  }
  for (int i = n - 1; i >= 0; i--) {
    l = i + 1;
    g = w[i];
    for (int j = l; j < n; j++) A_(i, j) = 0.0;
    if (g != 0.0) {
      g = 1.0 / g;
      for (int j = l; j < n; j++) {
        s = 0.0;
        for (int k = l; k < m; k++) s += A_(k, i) * A_(k, j);
        f = (s / A_(i, i)) * g;
        for (int k = i; k < m; k++) A_(k, j) += f * A_(k, i);
      }
      for (int j = i; j < m; j++) A_(j, i) *= g;
    } else {
      for (int j = i; j < m; j++) A_(j, i) = 0.0;
    }
    A_(i, i) += 1.0;
  }
  for (int k = n - 1; k >= 0; k--) {
    for (int its = 0; its < 50; its++) {
      int flag = 1;
      for (l = k; l >= 0; l--) {
        nm = l - 1;
        if ((fabs(rv1[l]) + anorm) == anorm) {
          flag = 0;
          break;
        }
        if (nm >= 0 && (fabs(w[nm]) + anorm) == anorm) break;
      }
      if (flag) {
        c = 0.0;
        s = 1.0;
        for (int i = l; i <= k; i++) {
          f = s * rv1[i];
          rv1[i] = c * rv1[i];
          if ((fabs(f) + anorm) == anorm) break;
          g = w[i];
          h = pythag_d(f, g);
          w[i] = h;
          h = 1.0 / h;
          c = g * h;
          s = -f * h;
          for (int j = 0; j < m; j++) {
            y = A_(j, nm);
            z = A_(j, i);
            A_(j, nm) = y * c + z * s;
            A_(j, i) = z * c - y * s;
          }
        }
      }
      z = w[k];
      if (l == k) {
        if (z < 0.0) {
          w[k] = -z;
          for (int j = 0; j < n; j++) V_(j, k) = -V_(j, k);
        }
        break;
      }
      if (its == 49) hit = 1;
      x = w[l];
      nm = k - 1;
      y = w[nm];
      g = rv1[nm];
      h = rv1[k];
      f = ((y - z) * (y + z) + (g - h) * (g + h)) / (2.0 * h * y);
      g = pythag_d(f, 1.0);
      f = ((x - z) * (x + z) + h * (y / (f + (f >= 0.0 ? g : -g)) - h)) / x;
      c = s = 1.0;
      for (int j = l; j <= nm; j++) {
        const int i = j + 1;
        g = rv1[i];
        y = w[i];
        h = s * g;
        g *= c;
        z = pythag_d(f, h);
        rv1[j] = z;
        c = f / z;
        s = h / z;
        f = x * c + g * s;
        g = g * c - x * s;
        h = y * s;
        y *= c;
        for (int jj = 0; jj < n; jj++) {
          x = V_(jj, j);
          z = V_(jj, i);
          V_(jj, j) = x * c + z * s;
          V_(jj, i) = z * c - x * s;
        }
        z = pythag_d(f, h);
        w[j] = z;
        if (z) {
          z = 1.0 / z;
          c = f * z;
          s = h * z;
        }
        f = c * g + s * y;
        x = c * y - s * g;
        for (int jj = 0; jj < m; jj++) {
          y = A_(jj, j);
          z = A_(jj, i);
          A_(jj, j) = y * c + z * s;
          A_(jj, i) = z * c - y * s;
        }
      }
      rv1[l] = 0.0;
      rv1[k] = f;
      w[k] = x;
    }
  }
  return hit;
#undef A_
#undef V_
}

// The same Golub-Reinsch decomposition producing U and w only (no V): the
// Householder reduction, the accumulation of the left transformations and the
// implicit-shift QR sweeps of gr_svd with every operation on V left out.  The
// operations on U and w are gr_svd's own, in its order (V's loops only
// overwrite scratch scalars that are reassigned before their next use); the
// compiler may contract multiply-adds differently in the two functions, so U
// and w agree with gr_svd's to rounding (me_svd_u against me_svd in the unit
// tests).  Matrix element (i, j) lives at a[(i * n + j) * STR], w[i] at
// w[i * STR], so one thread's matrix can sit in a column of shared memory.
template <int STR, bool FAST = false>
__device__ __noinline__ int gr_svd_u(double *a, int n, double *w, double *rv1) {
#define A_(i, j) a[((i) * n + (j)) * STR]
#define W_(i) w[(i) * STR]
#define R_(i) rv1[(i) * STR]
  const int m = n;
  int l = 0, nm = 0;
  double anorm = 0., c, f, g = 0., h, s, scale = 0., x, y, z;
  int hit = 0;
  for (int i = 0; i < n; i++) {
    l = i + 1;
    R_(i) = scale * g;
    g = s = scale = 0.0;
    for (int k = i; k < m; k++) scale += fabs(A_(k, i));
    if (scale) {
      const double is = 1.0 / scale;
      for (int k = i; k < m; k++) {
        const double t = A_(k, i) * is;
        A_(k, i) = t;
        s += t * t;
      }
      f = A_(i, i);
      g = f >= 0 ? -sqrt(s) : sqrt(s);
      h = f * g - s;
      A_(i, i) = f - g;
      const double ih = 1.0 / h;
      // columns j and j + 1 side by side: two independent chains, each
      // summed and updated in the order of the one-column loop
      int j = l;
      for (; j + 1 < n; j += 2) {
        double s0 = 0.0, s1 = 0.0;
        for (int k = i; k < m; k++) {
          const double aki = A_(k, i);
          s0 += aki * A_(k, j);
          s1 += aki * A_(k, j + 1);
        }
        const double f0 = s0 * ih, f1 = s1 * ih;
        for (int k = i; k < m; k++) {
          const double aki = A_(k, i);
          A_(k, j) += f0 * aki;
          A_(k, j + 1) += f1 * aki;
        }
      }
      if (j < n) {
        s = 0.0;
        for (int k = i; k < m; k++) s += A_(k, i) * A_(k, j);
        f = s * ih;
        for (int k = i; k < m; k++) A_(k, j) += f * A_(k, i);
      }
      for (int k = i; k < m; k++) A_(k, i) *= scale;
    }
    W_(i) = scale * g;
    g = s = scale = 0.0;
    if (i != n - 1) {
      for (int k = l; k < n; k++) scale += fabs(A_(i, k));
      if (scale) {
        const double is = 1.0 / scale;
        for (int k = l; k < n; k++) {
          const double t = A_(i, k) * is;
          A_(i, k) = t;
          s += t * t;
        }
        f = A_(i, l);
        g = f >= 0 ? -sqrt(s) : sqrt(s);
        h = f * g - s;
        A_(i, l) = f - g;
        const double ih = 1.0 / h;
        for (int k = l; k < n; k++) R_(k) = A_(i, k) * ih;
        int j = l;
        for (; j + 1 < m; j += 2) {  // rows j and j + 1 side by side
          double s0 = 0.0, s1 = 0.0;
          for (int k = l; k < n; k++) {
            const double aik = A_(i, k);
            s0 += A_(j, k) * aik;
            s1 += A_(j + 1, k) * aik;
          }
          for (int k = l; k < n; k++) {
            const double rk = R_(k);
            A_(j, k) += s0 * rk;
            A_(j + 1, k) += s1 * rk;
          }
        }
        if (j < m) {
          s = 0.0;
          for (int k = l; k < n; k++) s += A_(j, k) * A_(i, k);
          for (int k = l; k < n; k++) A_(j, k) += s * R_(k);
        }
        for (int k = l; k < n; k++) A_(i, k) *= scale;
      }
    }
    const double t = fabs(W_(i)) + fabs(R_(i));
    if (anorm < t) anorm = t;
  }
  for (int i = n - 1; i >= 0; i--) {
    l = i + 1;
    g = W_(i);
    for (int j = l; j < n; j++) A_(i, j) = 0.0;
    if (g != 0.0) {
      g = 1.0 / g;
      const double iaii = 1.0 / A_(i, i);
      int j = l;
      for (; j + 1 < n; j += 2) {  // columns j and j + 1 side by side
        double s0 = 0.0, s1 = 0.0;
        for (int k = l; k < m; k++) {
          const double aki = A_(k, i);
          s0 += aki * A_(k, j);
          s1 += aki * A_(k, j + 1);
        }
        const double f0 = (s0 * iaii) * g, f1 = (s1 * iaii) * g;
        for (int k = i; k < m; k++) {
          const double aki = A_(k, i);
          A_(k, j) += f0 * aki;
          A_(k, j + 1) += f1 * aki;
        }
      }
      if (j < n) {
        s = 0.0;
        for (int k = l; k < m; k++) s += A_(k, i) * A_(k, j);
        f = (s * iaii) * g;
        for (int k = i; k < m; k++) A_(k, j) += f * A_(k, i);
      }
      for (int j = i; j < m; j++) A_(j, i) *= g;
    } else {
      for (int j = i; j < m; j++) A_(j, i) = 0.0;
    }
    A_(i, i) += 1.0;
  }
  for (int k = n - 1; k >= 0; k--) {
    for (int its = 0; its < 50; its++) {
      int flag = 1;
      for (l = k; l >= 0; l--) {
        nm = l - 1;
        if ((fabs(R_(l)) + anorm) == anorm) {
          flag = 0;
          break;
        }
        if (nm >= 0 && (fabs(W_(nm)) + anorm) == anorm) break;
      }
      if (flag) {
        c = 0.0;
        s = 1.0;
        for (int i = l; i <= k; i++) {
          f = s * R_(i);
          R_(i) = c * R_(i);
          if ((fabs(f) + anorm) == anorm) break;
          g = W_(i);
          double ih;
          h = givens_radius<FAST>(f, g, ih);
          W_(i) = h;
          c = g * ih;
          s = -f * ih;
          for (int j = 0; j < m; j++) {
            y = A_(j, nm);
            z = A_(j, i);
            A_(j, nm) = y * c + z * s;
            A_(j, i) = z * c - y * s;
          }
        }
      }
      z = W_(k);
      if (l == k) {
        if (z < 0.0) W_(k) = -z;  // (V's column k would change sign here)
        break;
      }
      if (its == 49) hit = 1;
      x = W_(l);
      nm = k - 1;
      y = W_(nm);
      g = R_(nm);
      h = R_(k);
      f = ((y - z) * (y + z) + (g - h) * (g + h)) / (2.0 * h * y);
      g = pythag_d(f, 1.0);
      f = ((x - z) * (x + z) + h * (y / (f + (f >= 0.0 ? g : -g)) - h)) / x;
      c = s = 1.0;
      for (int j = l; j <= nm; j++) {
        const int i = j + 1;
        g = R_(i);
        y = W_(i);
        h = s * g;
        g *= c;
        double iz;
        z = givens_radius<FAST>(f, h, iz);
        R_(j) = z;
        chase_cs<FAST>(f, h, z, iz, c, s);
        f = x * c + g * s;
        g = g * c - x * s;
        h = y * s;
        y *= c;
        z = givens_radius<FAST>(f, h, iz);
        W_(j) = z;
        if (z) {
          c = f * iz;
          s = h * iz;
        }
        f = c * g + s * y;
        x = c * y - s * g;
        for (int jj = 0; jj < m; jj++) {
          y = A_(jj, j);
          z = A_(jj, i);
          A_(jj, j) = y * c + z * s;
          A_(jj, i) = z * c - y * s;
        }
      }
      R_(l) = 0.0;
      R_(k) = f;
      W_(k) = x;
    }
  }
  return hit;
#undef A_
#undef W_
#undef R_
}

// gr_svd_u for a group of G consecutive lanes of a warp (G a power of two,
// `mask` the group's lanes), the matrix row-major in the group's shared
// memory (stride 1): the vector loops of each update are spread over the
// lanes (lane t takes rows or columns t, t + G, ... of it), every sum is
// formed by one lane in gr_svd_u's order, and the scalar recurrences (w, rv1,
// the QR chase) run redundantly in every lane on private copies.  The
// arithmetic is gr_svd_u's operation for operation; only the latency
// changes.  w [n] is private to the lane.  All lanes of the group call it.
template <int G, bool FAST = false>
__device__ __noinline__ int gr_svd_u_grp(double *a, int n, double *w, int lane, unsigned mask) {
#define A_(i, j) a[(i) * n + (j)]
#define GSYNC()                  \
  do {                           \
    if (G > 1) __syncwarp(mask); \
  } while (0)
// k runs over 0 ... 8 unrolled, so that the column or row a lane holds stays in
// registers; the predicate keeps the reference's range and order
#define FOR9(k) _Pragma("unroll") for (int k = 0; k < 9; k++)
  const int m = n;
  int l = 0, nm = 0;
  double anorm = 0., c, f, g = 0., h, s, scale = 0., x, y, z;
  double rv1[9];
  int hit = 0;
  // Householder reduction.  Every lane reads the column (then the row) being
  // reduced into registers and scales it there, so the transforms of the
  // other columns (rows) read it from registers; the scaled vector goes back
  // to shared memory once, after the transforms: one synchronisation per
  // column and per row.
  for (int i = 0; i < n; i++) {
    l = i + 1;
    rv1[i] = scale * g;
    g = s = scale = 0.0;
    double col[9];
    FOR9(k) col[k] = (k >= i && k < m) ? A_(k, i) : 0.0;
    FOR9(k) if (k >= i && k < m) scale += fabs(col[k]);
    if (scale) {
      const double is = 1.0 / scale;
      FOR9(k) if (k >= i && k < m) {
        col[k] *= is;
        s += col[k] * col[k];
      }
      f = A_(i, i) * is;
      g = f >= 0 ? -sqrt(s) : sqrt(s);
      h = f * g - s;
      FOR9(k) if (k == i) col[k] = f - g;
      const double ih = 1.0 / h;
      for (int j = l + lane; j < n; j += G) {
        double sj = 0.0;
        FOR9(k) if (k >= i && k < m) sj += col[k] * A_(k, j);
        const double fj = sj * ih;
        FOR9(k) if (k >= i && k < m) A_(k, j) += fj * col[k];
      }
      GSYNC();
      FOR9(k) if (k >= i && k < m && ((k - i) & (G - 1)) == lane) A_(k, i) = col[k] * scale;
    }
    w[i] = scale * g;
    g = s = scale = 0.0;
    if (i != n - 1) {
      double row[9];
      FOR9(k) row[k] = (k >= l && k < n) ? A_(i, k) : 0.0;
      FOR9(k) if (k >= l && k < n) scale += fabs(row[k]);
      if (scale) {
        const double is = 1.0 / scale;
        FOR9(k) if (k >= l && k < n) {
          row[k] *= is;
          s += row[k] * row[k];
        }
        f = A_(i, l) * is;
        g = f >= 0 ? -sqrt(s) : sqrt(s);
        h = f * g - s;
        const double ih = 1.0 / h;
        FOR9(k) if (k == l) row[k] = f - g;
        double rk[9];  // rv1 = the scaled row / h, in every lane
        FOR9(k) {
          rk[k] = row[k] * ih;
          if (k >= l && k < n) rv1[k] = rk[k];
        }
        for (int j = l + lane; j < m; j += G) {
          double sj = 0.0;
          FOR9(k) if (k >= l && k < n) sj += A_(j, k) * row[k];
          FOR9(k) if (k >= l && k < n) A_(j, k) += sj * rk[k];
        }
        GSYNC();
        FOR9(k) if (k >= l && k < n && ((k - l) & (G - 1)) == lane) A_(i, k) = row[k] * scale;
      }
    }
    const double t = fabs(w[i]) + fabs(rv1[i]);
    if (anorm < t) anorm = t;
  }
  GSYNC();
  // Accumulation of the left-hand transformations.  Column i is read into
  // registers before anything changes it; the lane that owns column j zeroes
  // A(i, j) and updates the column, so only the new column i needs a
  // synchronisation before the next step reads it.
  for (int i = n - 1; i >= 0; i--) {
    l = i + 1;
    g = w[i];
    double col[9];
    FOR9(k) col[k] = (k >= i && k < m) ? A_(k, i) : 0.0;
    const double aii = A_(i, i);
    for (int j = l + lane; j < n; j += G) A_(i, j) = 0.0;
    if (g != 0.0) {
      g = 1.0 / g;
      const double iaii = 1.0 / aii;
      for (int j = l + lane; j < n; j += G) {
        double sj = 0.0;
        FOR9(k) if (k >= l && k < m) sj += col[k] * A_(k, j);
        const double fj = (sj * iaii) * g;
        FOR9(k) if (k >= i && k < m) A_(k, j) += fj * col[k];
      }
      GSYNC();  // every lane has read column i
      // A(k, i) * g, then + 1 on the diagonal: two roundings, as the
      // reference's separate statements make them
      FOR9(k) if (k >= i && k < m && ((k - i) & (G - 1)) == lane)
        A_(k, i) = k == i ? __dadd_rn(__dmul_rn(col[k], g), 1.0) : __dmul_rn(col[k], g);
    } else {
      GSYNC();
      FOR9(k) if (k >= i && k < m && ((k - i) & (G - 1)) == lane) A_(k, i) = k == i ? 1.0 : 0.0;
    }
    GSYNC();
  }
  // QR sweeps: each rotation touches the lane's own rows only, so the lanes
  // need no synchronisation until the end
  for (int k = n - 1; k >= 0; k--) {
    for (int its = 0; its < 50; its++) {
      int flag = 1;
      for (l = k; l >= 0; l--) {
        nm = l - 1;
        if ((fabs(rv1[l]) + anorm) == anorm) {
          flag = 0;
          break;
        }
        if (nm >= 0 && (fabs(w[nm]) + anorm) == anorm) break;
      }
      if (flag) {
        c = 0.0;
        s = 1.0;
        for (int i = l; i <= k; i++) {
          f = s * rv1[i];
          rv1[i] = c * rv1[i];
          if ((fabs(f) + anorm) == anorm) break;
          g = w[i];
          double ih;
          h = givens_radius<FAST>(f, g, ih);
          w[i] = h;
          c = g * ih;
          s = -f * ih;
          for (int jj = lane; jj < m; jj += G) {
            const double yy = A_(jj, nm), zz = A_(jj, i);
            A_(jj, nm) = yy * c + zz * s;
            A_(jj, i) = zz * c - yy * s;
          }
        }
      }
      z = w[k];
      if (l == k) {
        if (z < 0.0) w[k] = -z;
        break;
      }
      if (its == 49) hit = 1;
      x = w[l];
      nm = k - 1;
      y = w[nm];
      g = rv1[nm];
      h = rv1[k];
      f = ((y - z) * (y + z) + (g - h) * (g + h)) / (2.0 * h * y);
      g = pythag_d(f, 1.0);
      f = ((x - z) * (x + z) + h * (y / (f + (f >= 0.0 ? g : -g)) - h)) / x;
      c = s = 1.0;
      // each rotation is applied to the lane's rows one step late, beside
      // the next rotation's scalar chain, with the rows' column j + 1 carried
      // in registers (as in gr_svd_u)
      constexpr int R = (9 + G - 1) / G;  // rows per lane
      double cy[R];
#pragma unroll
      for (int r = 0; r < R; r++)
        if (lane + r * G < m) cy[r] = A_(lane + r * G, l);
      double pc = 0.0, ps = 0.0;
      double gi = rv1[l + 1], yi = w[l + 1];
      for (int j = l; j <= nm; j++) {
        const int i = j + 1;
        g = gi;
        y = yi;
        if (i < k) {
          gi = rv1[i + 1];
          yi = w[i + 1];
        }
        if (j > l) {
#pragma unroll
          for (int r = 0; r < R; r++)
            if (lane + r * G < m) {
              const int jj = lane + r * G;
              const double yy = cy[r], zz = A_(jj, j);
              A_(jj, j - 1) = yy * pc + zz * ps;
              cy[r] = zz * pc - yy * ps;
            }
        }
        h = s * g;
        g *= c;
        double iz;
        z = givens_radius<FAST>(f, h, iz);
        rv1[j] = z;
        chase_cs<FAST>(f, h, z, iz, c, s);
        f = x * c + g * s;
        g = g * c - x * s;
        h = y * s;
        y *= c;
        z = givens_radius<FAST>(f, h, iz);
        w[j] = z;
        if (z) {
          c = f * iz;
          s = h * iz;
        }
        f = c * g + s * y;
        x = c * y - s * g;
        pc = c;
        ps = s;
      }
#pragma unroll
      for (int r = 0; r < R; r++)
        if (lane + r * G < m) {
          const int jj = lane + r * G;
          const double yy = cy[r], zz = A_(jj, k);
          A_(jj, nm) = yy * pc + zz * ps;
          A_(jj, k) = zz * pc - yy * ps;
        }
      rv1[l] = 0.0;
      rv1[k] = f;
      w[k] = x;
    }
  }
  GSYNC();
  return hit;
#undef FOR9
#undef GSYNC
#undef A_
}

// gr_svd_u for a full 9x9 matrix held in registers (no parameter fixed, the
// common case).  Once the loops over the column i (Householder, left-hand
// accumulation) and over the block end k (QR sweeps) are unrolled, every index
// is a compile-time constant, so the 81 elements, w and rv1 stay in registers
// and the independent row and column updates of each step interleave.  The
// two per-matrix indices of the QR phase -- the start l of the unreduced block
// and the cancelled column l - 1 -- select among unrolled cases (predicated
// on j >= l, or one case per value of l).  The operations and their order are
// gr_svd_u's (SVD_TEMPLATE.h:84-344 without V).  A NaN matrix, for which no
// negligible entry is found, is left unrotated (the reference's loop would
// index below the matrix there).
template <bool FAST = false>
__device__ __forceinline__ int gr_svd_u9(double (&A)[9][9], double (&w)[9]) {
  constexpr int n = 9, m = 9;
  double rv1[9];
  double anorm = 0., g = 0., scale = 0.;
  int hit = 0;
#pragma unroll
  for (int i = 0; i < n; i++) {
    const int l = i + 1;
    rv1[i] = scale * g;
    double s = 0.0;
    g = scale = 0.0;
#pragma unroll
    for (int k = i; k < m; k++) scale += fabs(A[k][i]);
    if (scale) {
      const double is = 1.0 / scale;
#pragma unroll
      for (int k = i; k < m; k++) {
        const double t = A[k][i] * is;
        A[k][i] = t;
        s += t * t;
      }
      const double f = A[i][i];
      g = f >= 0 ? -sqrt(s) : sqrt(s);
      const double h = f * g - s;
      A[i][i] = f - g;
      const double ih = 1.0 / h;
#pragma unroll
      for (int j = l; j < n; j++) {
        double sj = 0.0;
#pragma unroll
        for (int k = i; k < m; k++) sj += A[k][i] * A[k][j];
        const double fj = sj * ih;
#pragma unroll
        for (int k = i; k < m; k++) A[k][j] += fj * A[k][i];
      }
#pragma unroll
      for (int k = i; k < m; k++) A[k][i] *= scale;
    }
    w[i] = scale * g;
    s = 0.0;
    g = scale = 0.0;
    if (i != n - 1) {
#pragma unroll
      for (int k = l; k < n; k++) scale += fabs(A[i][k]);
      if (scale) {
        const double is = 1.0 / scale;
#pragma unroll
        for (int k = l; k < n; k++) {
          const double t = A[i][k] * is;
          A[i][k] = t;
          s += t * t;
        }
        const double f = A[i][l];
        g = f >= 0 ? -sqrt(s) : sqrt(s);
        const double h = f * g - s;
        A[i][l] = f - g;
        const double ih = 1.0 / h;
#pragma unroll
        for (int k = l; k < n; k++) rv1[k] = A[i][k] * ih;
#pragma unroll
        for (int j = l; j < m; j++) {
          double sj = 0.0;
#pragma unroll
          for (int k = l; k < n; k++) sj += A[j][k] * A[i][k];
#pragma unroll
          for (int k = l; k < n; k++) A[j][k] += sj * rv1[k];
        }
#pragma unroll
        for (int k = l; k < n; k++) A[i][k] *= scale;
      }
    }
    const double t = fabs(w[i]) + fabs(rv1[i]);
    if (anorm < t) anorm = t;
  }
  // accumulation of the left-hand transformations into U
#pragma unroll
  for (int i = n - 1; i >= 0; i--) {
    const int l = i + 1;
    double gi = w[i];
#pragma unroll
    for (int j = l; j < n; j++) A[i][j] = 0.0;
    if (gi != 0.0) {
      gi = 1.0 / gi;
      const double iaii = 1.0 / A[i][i];
#pragma unroll
      for (int j = l; j < n; j++) {
        double sj = 0.0;
#pragma unroll
        for (int k = l; k < m; k++) sj += A[k][i] * A[k][j];
        const double fj = (sj * iaii) * gi;
#pragma unroll
        for (int k = i; k < m; k++) A[k][j] += fj * A[k][i];
      }
#pragma unroll
      for (int j = i; j < m; j++) A[j][i] *= gi;
    } else {
#pragma unroll
      for (int j = i; j < m; j++) A[j][i] = 0.0;
    }
    A[i][i] += 1.0;
  }
  // implicit-shift QR sweeps on the bidiagonal, block end k
#pragma unroll
  for (int k = n - 1; k >= 0; k--) {
    for (int its = 0; its < 50; its++) {
      // l: start of the unreduced block; cancel: w[l - 1] is negligible
      int l = 0;
      bool found = false, cancel = false;
#pragma unroll
      for (int ll = k; ll >= 0; ll--) {
        if (!found) {
          if ((fabs(rv1[ll]) + anorm) == anorm) {
            l = ll;
            found = true;
          } else if (ll >= 1 && (fabs(w[ll - 1]) + anorm) == anorm) {
            l = ll;
            found = true;
            cancel = true;
          }
        }
      }
      if (cancel) {
        double c = 0.0, s = 1.0;
#pragma unroll
        for (int lc = 1; lc <= k; lc++) {
          if (lc == l) {
            bool stop = false;
#pragma unroll
            for (int i = lc; i <= k; i++) {
              if (!stop) {
                const double f = s * rv1[i];
                rv1[i] = c * rv1[i];
                if ((fabs(f) + anorm) == anorm) {
                  stop = true;
                } else {
                  const double gg = w[i];
                  double ih;
                  const double h = givens_radius<FAST>(f, gg, ih);
                  w[i] = h;
                  c = gg * ih;
                  s = -f * ih;
#pragma unroll
                  for (int j = 0; j < m; j++) {
                    const double y = A[j][lc - 1], z = A[j][i];
                    A[j][lc - 1] = y * c + z * s;
                    A[j][i] = z * c - y * s;
                  }
                }
              }
            }
          }
        }
      }
      const double zk = w[k];
      if (l == k) {
        if (zk < 0.0) w[k] = -zk;
        break;
      }
      if (its == 49) hit = 1;
      double x = 0.0;
#pragma unroll
      for (int q = 0; q < k; q++)
        if (q == l) x = w[q];
      double y = w[k - 1];
      double gq = rv1[k - 1];
      double h = rv1[k];
      double z = zk;
      double f = ((y - z) * (y + z) + (gq - h) * (gq + h)) / (2.0 * h * y);
      gq = pythag_d(f, 1.0);
      f = ((x - z) * (x + z) + h * (y / (f + (f >= 0.0 ? gq : -gq)) - h)) / x;
      double c = 1.0, s = 1.0;
#pragma unroll
      for (int j = 0; j < k; j++) {
        if (j >= l) {
          const int i = j + 1;
          gq = rv1[i];
          y = w[i];
          h = s * gq;
          gq *= c;
          double iz;
          z = givens_radius<FAST>(f, h, iz);
          rv1[j] = z;
          chase_cs<FAST>(f, h, z, iz, c, s);
          f = x * c + gq * s;
          gq = gq * c - x * s;
          h = y * s;
          y *= c;
          z = givens_radius<FAST>(f, h, iz);
          w[j] = z;
          if (z) {
            c = f * iz;
            s = h * iz;
          }
          f = c * gq + s * y;
          x = c * y - s * gq;
#pragma unroll
          for (int jj = 0; jj < m; jj++) {
            const double yy = A[jj][j], zz = A[jj][i];
            A[jj][j] = yy * c + zz * s;
            A[jj][i] = zz * c - yy * s;
          }
        }
      }
#pragma unroll
      for (int q = 0; q < k; q++)
        if (q == l) rv1[q] = 0.0;
      rv1[k] = f;
      w[k] = x;
    }
  }
  return hit;
}

// x = V diag(1/w) U^T b, skipping w <= 1e-50 (svbksb, SVD_TEMPLATE.h:348-406).
__device__ __forceinline__ void gr_backsub(const double *u, const double *v, const double *w,
                                           const double *b, int n, double *x) {
  double t[9];
  for (int j = 0; j < n; j++) {
    double s = 0.0;
    if (w[j] > 1e-50) {
      for (int i = 0; i < n; i++) s += u[i * n + j] * b[i];
      s /= w[j];
    }
    t[j] = s;
  }
  for (int i = 0; i < n; i++) {
    double s = 0.0;
    for (int j = 0; j < n; j++) s += v[i * n + j] * t[j];
    x[i] = s;
  }
}

// SVD_solve_mem (LM_FIT.c:400-469): the SVD overwrites hess by U; singular
// values below w_max * thr are dropped, thr x5 from SVDthreshold until the
// step is inside +-0.5 or thr exceeds 2e-3, then the step is clamped.
__device__ __forceinline__ int svd_solve(double *hess, double *v, const double *g, int n,
                                         double thr, double *sol) {
  double w[9];
  const int hit = gr_svd(hess, n, w, v);
  double wmax = w[0];
  for (int i = 1; i < n; i++) wmax = wmax > w[i] ? wmax : w[i];
  while (true) {
    const double wthr = wmax * thr;
    for (int i = 0; i < n; i++)
      if (w[i] < wthr) w[i] = 0.;
    gr_backsub(hess, v, w, g, n, sol);
    bool inside = true;
    for (int i = 0; i < n; i++)
      if (sol[i] > 0.5 || sol[i] < -0.5) inside = false;
    if (inside) break;
    if (thr > 2e-3) {
      for (int i = 0; i < n; i++) sol[i] = sol[i] > 0.5 ? 0.5 : (sol[i] < -0.5 ? -0.5 : sol[i]);
      break;
    }
    thr *= 5.;
  }
  return hit;
}

// ---------------------------------------------------------------------------
// Restart draws: Philox4x32-10 (Salmon et al., SC'11) keyed by the plan's
// seed, counter (pixel, run, block); Box-Muller pairs -> 8 standard normals.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void philox10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    const uint32_t lo0 = 0xD2511F53u * c[0], hi0 = __umulhi(0xD2511F53u, c[0]);
    const uint32_t lo1 = 0xCD9E8D57u * c[2], hi1 = __umulhi(0xCD9E8D57u, c[2]);
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

__device__ inline void restart_draws(unsigned long long seed, long long pixel, int run,
                                     double z[8]) {
#pragma unroll
  for (int blk = 0; blk < 2; blk++) {
    uint32_t c[4] = {(uint32_t)((unsigned long long)pixel & 0xffffffffu),
                     (uint32_t)((unsigned long long)pixel >> 32), (uint32_t)run, (uint32_t)blk};
    philox10(c, (uint32_t)(seed & 0xffffffffu), (uint32_t)(seed >> 32));
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const double u1 = ((double)c[2 * h] + 0.5) * 2.3283064365386963e-10;
      const double u2 = ((double)c[2 * h + 1] + 0.5) * 2.3283064365386963e-10;
      const double r = sqrt(-2.0 * log(u1));
      double sn, cs;
      sincos(6.283185307179586 * u2, &sn, &cs);
      z[blk * 4 + 2 * h] = r * cs;
      z[blk * 4 + 2 * h + 1] = r * sn;
    }
  }
}

}  // namespace me

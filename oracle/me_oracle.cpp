// me_oracle.cpp -- CPU restatement of the reference's per-pixel Milne-Eddington
// inversion.  TEST INFRASTRUCTURE ONLY (the checker of the CUDA path; never
// linked into the product).
//
// Follows, function by function, the reference's files under Src/ (cited per
// function).  Floating-point expressions keep the reference's evaluation order
// and the same libm calls so that, on the same CPU, the oracle reproduces the
// reference bit for bit; that is what lets it be pinned against the reference
// on every pixel (the reference's LM flips to another trajectory on a one-ulp
// change of its inputs for about a quarter of the pixels of a configs-0 map).
// Build: oracle/Makefile (-ffp-contract=off).
#include "me_oracle.h"
#include "flop_count.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

namespace {

const double kPi = 3.14159265358979323846;      // Src/ME_SOLVER.c:46
const double kLightSpeed = 299792458.0;          // Src/ME_SOLVER.c:48
const double kSqrtPi = 1.77245385090551588191;   // Src/ME_SOLVER.c:128

// ---------------------------------------------------------------------------
// Faddeeva / Voigt.  Src/FADDEEVA.c
// ---------------------------------------------------------------------------

struct VoigtTables {  // STRUCT_FADDEEVA, Src/FADDEEVA.h; Faddeeva_init Src/FADDEEVA.c:406-436
  int nfigures = 6, row = 2, nmax = 50;
  double rmin0 = 0, log_rmin0 = 0, sqrt_log_rmin0 = 0, a = 0, aa = 0;
  double exp_a2n2[50];
  void init(int nfig) {
    nfigures = nfig;
    rmin0 = pow(10., -nfigures);
    a = M_PI / sqrt(-log(0.5 * rmin0));
    aa = a * a;
    log_rmin0 = -log(rmin0);
    sqrt_log_rmin0 = sqrt(log_rmin0);
    nmax = 50;
    row = nfigures > 4 ? nfigures - 4 : 0;
    exp_a2n2[0] = 1.;
    for (int n = 1; n < nmax; n++) exp_a2n2[n] = exp(-aa * n * n);
  }
};

// Dawson's integral, Rybicki's method as in Numerical Recipes (Src/FADDEEVA.c:29-79).
template <class R>
R dawson(R x) {
  const R A1 = 2.0 / 3.0, A2 = 0.4, A3 = 2.0 / 7.0, H = 0.4;
  R ax = fabs(x);
  if (ax < 0.2) {
    R x2 = x * x;
    return x * (1.0 - A1 * x2 * (1.0 - A2 * x2 * (1.0 - A3 * x2)));
  }
  R c[7];
  for (int i = 1; i <= 6; i++) {
    R t = (2.0 * i - 1.0) * H;
    c[i] = exp(-t * t);
  }
  int n0 = 2 * (int)round(ax / (2 * H));
  R xp = ax - n0 * H;
  R e1 = exp(2.0 * xp * H);
  R e2 = e1 * e1;
  R d1 = n0 + 1;
  R d2 = d1 - 2.0;
  R sum = 0.0;
  for (int i = 1; i <= 6; i++, d1 += 2.0, d2 -= 2.0, e1 *= e2)
    sum += c[i] * (e1 / d1 + 1.0 / (d2 * e1));
  R t = exp(-xp * xp);
  return 0.5641895835 * copysign(t, x) * sum;
}

// erfcx(a) = exp(a^2) erfc(a), with the large-argument asymptotic series
// (Src/FADDEEVA.c:83-108).
template <class R>
R erfcx_ref(R a) {
  if (a > 26.6) {
    R a2 = a * a;
    return ((((((162.421875 / a2 - 29.53125) / a2 + 6.5625) / a2 - 1.875) / a2 + 0.75) / a2 -
             0.5) / a2 + 1) / kSqrtPi / a;
  }
  return exp(a * a) * erfc(a);
}

// Hui, Armstrong & Wray (1978) 6-pole rational approximation (Src/FADDEEVA.c:112-163).
template <class R>
void voigt_hui6(R nu, R y, R *H, R *L) {
  static const R A[7] = {122.607931777104326, 214.382388694706425, 181.928533092181549,
                              93.155580458138441,  30.180142196210589,  5.912626209773153,
                              0.564189583562615};
  static const R B[7] = {122.60793177387535,  352.730625110963558, 457.334478783897737,
                              348.703917719495792, 170.354001821091472, 53.992906912940207,
                              10.479857114260399};
  const R zr = y, zi = -nu;
  R pr = A[6], pi = 0.0;
  R qr = B[6] + zr, qi = zi;
  for (int k = 5; k >= 0; k--) {
    R tr = pr * zr - pi * zi + A[k];
    R ti = pr * zi + pi * zr;
    pr = tr;
    pi = ti;
    tr = qr * zr - qi * zi + B[k];
    ti = qr * zi + qi * zr;
    qr = tr;
    qi = ti;
  }
  R den = qr * qr + qi * qi;
  *H = (pr * qr + pi * qi) / den;
  *L = (pi * qr - pr * qi) / den;
}

// Humlicek (1982) W4, four regions (Src/FADDEEVA.c:167-281).
template <class R>
void voigt_humlicek_w4(R nu, R y, R *H, R *L) {
  const R anu = fabs(nu);
  const R s = anu + y;
  const R tr = y, ti = -nu;
  if (s >= 15) {
    const R ur = tr * tr - ti * ti, ui = 2.0 * tr * ti;
    R dr = 0.5 + ur, di = ui;
    R den = dr * dr + di * di;
    *H = 0.56418958355 * (tr * dr + ti * di) / den;
    *L = 0.56418958355 * (ti * dr - tr * di) / den;
  } else if (s >= 5.5) {
    const R ur = tr * tr - ti * ti, ui = 2.0 * tr * ti;
    R nr = 1.4104739589 + 0.5641896 * ur;
    R ni = 0.5641896 * ui;
    R dr = 0.75 + 3.0 * ur + (ur * ur - ui * ui);
    R di = 3.0 * ui + 2.0 * ur * ui;
    R den = dr * dr + di * di;
    R qr = (nr * dr + ni * di) / den;
    R qi = (ni * dr - nr * di) / den;
    *H = tr * qr - ti * qi;
    *L = tr * qi + ti * qr;
  } else if (y >= 1.95 * anu - 0.176) {
    const R c[5] = {0.5642236, 3.778987, 11.96482, 20.20933, 16.4955};
    const R d[6] = {1.0, 6.699398, 21.69274, 39.27121, 38.82363, 16.4955};
    R nr = c[0], ni = 0, dr = d[0], di = 0;
    for (int k = 1; k < 5; k++) {
      R r = nr * tr - ni * ti + c[k];
      R i = nr * ti + ni * tr;
      nr = r;
      ni = i;
    }
    for (int k = 1; k < 6; k++) {
      R r = dr * tr - di * ti + d[k];
      R i = dr * ti + di * tr;
      dr = r;
      di = i;
    }
    R den = dr * dr + di * di;
    *H = (nr * dr + ni * di) / den;
    *L = (ni * dr - nr * di) / den;
  } else {
    const double c[7] = {0.5641900381, 1.320521697, 35.7668278,  219.0312964,
                         1540.786893,  3321.990492, 36183.30536};
    const R d[8] = {1,           1.841438936, 61.57036588, 364.2190727,
                         2186.181081, 9022.227659, 24322.84021, 32066.59372};
    const R ur = tr * tr - ti * ti, ui = 2.0 * tr * ti;
    R eu = exp(ur);
    R er = eu * cos(ui), ei = eu * sin(ui);
    R nr = c[0], ni = 0, dr = d[0], di = 0;
    for (int k = 1; k < 7; k++) {
      R r = -(nr * ur - ni * ui) + c[k];
      R i = -(nr * ui + ni * ur);
      nr = r;
      ni = i;
    }
    R r = nr * tr - ni * ti;
    R i = nr * ti + ni * tr;
    nr = r;
    ni = i;
    for (int k = 1; k < 8; k++) {
      r = -(dr * ur - di * ui) + d[k];
      i = -(dr * ui + di * ur);
      dr = r;
      di = i;
    }
    R den = dr * dr + di * di;
    *H = er - (nr * dr + ni * di) / den;
    *L = ei - (ni * dr - nr * di) / den;
  }
}

// Zaghloul & Ali (2011) ACM Algorithm 916 (Src/FADDEEVA.c:286-402).
template <class R>
void voigt_alg916(R nu, R y, R *H, R *L, const VoigtTables &f) {
  if (nu == 0) {
    *H = erfcx_ref(y);
    *L = 0;
    return;
  } else if (y == 0) {
    *H = exp(-nu * nu);
    *L = 2.0 / kSqrtPi * dawson(nu);
    return;
  }
  const R x = fabs(nu), ya = fabs(y);
  if (x + ya > 1e7) {
    if (x < ya) {
      R xs = x / ya;
      *H = 1. / kSqrtPi / (xs * xs + 1.);
      *L = xs / kSqrtPi / (xs * xs + 1.);
    } else {
      R ys = ya / x;
      *H = ys / kSqrtPi / (ys * ys + 1.);
      *L = 1. / kSqrtPi / (ys * ys + 1.);
    }
    return;
  }
  const R xx = x * x, yy = y * y, xy = x * y;
  const R xy2 = 2 * xy;
  const R sin_xy = sin(xy), sin_2xy = sin(xy2), cos_2xy = cos(xy2);
  const R exp_xx = exp(-xx), exp_2ax = exp(2 * f.a * x);
  const R k1 = exp_xx * erfcx_ref(y);

  const int nmax1 = (int)(sqrt(f.log_rmin0 - x * x) / f.a + 0.5);
  const int nmax2 = (int)((f.sqrt_log_rmin0 - x) / f.a + 0.5);
  int nmax = nmax1 > nmax2 ? nmax1 : nmax2;
  if (nmax >= f.nmax) nmax = f.nmax - 1;

  int nb = (int)(x / f.a + 0.5);
  int nf = nb + 1;
  const R dxf = f.a * nf - x;
  const R dxb = x - f.a * nb;
  int nmaxf = (int)((f.sqrt_log_rmin0 - dxf) / f.a);
  int nmaxb = (int)((f.sqrt_log_rmin0 - dxb) / f.a);
  if (nmaxf >= f.nmax) nmaxf = f.nmax - 1;
  if (nmaxb >= f.nmax) nmaxb = f.nmax - 1;
  const int nlo = (nb - nmaxb) > 1 ? (nb - nmaxb) : 1;

  R re = k1 * cos_2xy + 2 * f.a * x * sin_xy * exp_xx * sin_xy / xy / M_PI;
  R im = -k1 * sin_2xy + 2 * f.a * x * exp_xx * sin_2xy / xy2 / M_PI;
  R s1 = 0, s2 = 0, s3 = 0, s4 = 0, s5 = 0;

  R e1 = exp(-dxf * dxf);
  R e2 = exp(-2 * f.a * dxf);
  R ep = 1.;
  for (int n = nf; n <= nf + nmaxf; n++) {
    R t = e1 * f.exp_a2n2[n - nf] / (R(f.aa) * n * n + yy);
    s3 += t * ep;
    s5 += t * ep * f.a * n;
    ep *= e2;
  }
  e1 = exp(-dxb * dxb);
  e2 = exp(-2 * f.a * dxb);
  ep = 1.;
  for (int n = nb; n >= nlo; n--) {
    R t = e1 * f.exp_a2n2[nb - n] / (R(f.aa) * n * n + yy);
    s3 += t * ep;
    s5 += t * ep * f.a * n;
    ep *= e2;
  }
  re += f.a * y * s3 / M_PI;
  im += f.a * s5 / M_PI;
  if (x < f.sqrt_log_rmin0 || x < 10) {
    ep = 1.;
    for (int n = 1; n <= nmax; n++) {
      R t = exp_xx * f.exp_a2n2[n] / (R(f.aa) * n * n + yy);
      s1 += t;
      ep /= exp_2ax;
      s2 += t * ep;
      s4 += t * ep * f.a * n;
    }
    re += f.a * y * (-2 * cos_2xy * s1 + s2) / M_PI;
    im += f.a * (2 * y * sin_2xy * s1 - s4) / M_PI;
  }
  *H = re;
  *L = nu > 0 ? im : -im;
}

// Accuracy-selected w(z) (Zaghloul 2018 region thresholds), Src/FADDEEVA.c:440-590.
template <class R>
void voigt(R nu, R y, R *H, R *L, const VoigtTables &f) {
  if (nu == 0) {
    *H = erfcx_ref(y);
    *L = 0;
    return;
  } else if (y == 0) {
    *H = exp(-nu * nu);
    *L = 2.0 / kSqrtPi * dawson(nu);
    return;
  }
  // |z|^2 region boundaries per accuracy row (Src/FADDEEVA.c:471-477)
  static const R T[5][5] = {{1.6e4, 160.0, 107.0, 28.5, 3.5},
                                 {1.5e5, 510.0, 110.0, 39., -0.1},
                                 {1.451e6, 1.6e3, 180.0, 110.0, -0.1},
                                 {1.5e7, 5.01e3, 380.0, 115.0, 114.0},
                                 {1.3e8, 1.6e4, 810.0, 195.0, 116.0}};
  const R *t = T[f.row];
  const R zr = nu, zi = y;
  const R z2r = zr * zr - zi * zi;
  const R z2i = 2.0 * zr * zi;
  const R r2 = zr * zr + zi * zi;
  const R y2 = y * y;
  if (r2 >= t[0]) {
    R den = kSqrtPi * (zr * zr + zi * zi);
    *H = zi / den;
    *L = zr / den;
  } else if (r2 >= t[1]) {
    R wr = z2r - 0.5;
    R den = kSqrtPi * (wr * wr + z2i * z2i);
    *H = (-zi * wr + zr * z2i) / den;
    *L = (zr * wr + zi * z2i) / den;
  } else if (r2 >= t[2]) {
    R wr = z2r - 1.5;
    R pr = wr * zr - z2i * zi;
    R pi = wr * zi + z2i * zr;
    R den = kSqrtPi * (pr * pr + pi * pi);
    wr = z2r - 1.0;
    *H = (-z2i * pr + wr * pi) / den;
    *L = (wr * pr + z2i * pi) / den;
  } else if (r2 >= t[3]) {
    if (f.nfigures <= 4 && y2 < 6e-14) {
      voigt_humlicek_w4(nu, y, H, L);
      return;
    } else if (f.nfigures == 5 && r2 < 39 && y2 < 1e-9) {
      voigt_humlicek_w4(nu, y, H, L);
      return;
    }
    R wr = z2r - 2.5;
    R ar = -(wr * zi + z2i * zr);
    R ai = wr * zr - z2i * zi;
    wr = z2r - 3.;
    R br = wr * z2r - z2i * z2i + 0.75;
    R bi = (wr + z2r) * z2i;
    R den = kSqrtPi * (br * br + bi * bi);
    *H = (ar * br + ai * bi) / den;
    *L = (-ar * bi + ai * br) / den;
  } else if (r2 >= t[4]) {
    if (f.nfigures <= 4) {
      if (y2 < 0.026)
        voigt_humlicek_w4(nu, y, H, L);
      else
        voigt_hui6(nu, y, H, L);
      return;
    } else if (f.nfigures == 5) {
      if (y2 >= 0.27)
        voigt_hui6(nu, y, H, L);
      else if (y2 >= 1e-9)
        voigt_alg916(nu, y, H, L, f);
      else
        voigt_humlicek_w4(nu, y, H, L);
      return;
    } else if (f.nfigures == 6) {
      if (y2 >= 1)
        voigt_hui6(nu, y, H, L);
      else
        voigt_alg916(nu, y, H, L, f);
      return;
    }
    R wr = z2r - 4.5;
    R ar = -(wr + z2r) * z2i;
    R ai = wr * z2r - z2i * z2i + 2.;
    wr = z2r - 5.;
    R br = wr * z2r - z2i * z2i + 3.75;
    R bi = (wr + z2r) * z2i;
    R cr = br * zr - bi * zi;
    R ci = br * zi + bi * zr;
    R den = kSqrtPi * (cr * cr + ci * ci);
    *H = (ar * cr + ai * ci) / den;
    *L = (-ar * ci + ai * cr) / den;
  } else {
    if (f.nfigures <= 4)
      voigt_hui6(nu, y, H, L);
    else
      voigt_alg916(nu, y, H, L, f);
  }
}

// ---------------------------------------------------------------------------
// Restart draws.
// ---------------------------------------------------------------------------

// Park-Miller minimal standard with Bays-Durham shuffle (NR ran1) and the
// polar Box-Muller method: Src/RANDOM_NUMBER.c:65-174.
struct NrStream {
  int32_t idum = -1, iy = 0, iv[32];
  bool iset = true;
  double gset = 0;
  void seed(int s) {
    idum = -(int32_t)(s & 0x7FFFFFFF);
    iy = 0;
    iset = true;
  }
  double uniform() {
    const int IA = 16807, IM = 2147483647, IQ = 127773, IR = 2836;
    const int NDIV = (1 + (2147483647 - 1) / 32);
    const double AM = (1.0 / 2147483647), RNMX = (1.0 - 1.2e-7);
    int32_t k;
    if (idum <= 0 || !iy) {
      idum = (-idum < 1) ? 1 : -idum;
      for (int j = 32 + 7; j >= 0; j--) {
        k = idum / IQ;
        idum = IA * (idum - k * IQ) - IR * k;
        if (idum < 0) idum += IM;
        if (j < 32) iv[j] = idum;
      }
      iy = iv[0];
    }
    k = idum / IQ;
    idum = IA * (idum - k * IQ) - IR * k;
    if (idum < 0) idum += IM;
    int j = iy / NDIV;
    iy = iv[j];
    iv[j] = idum;
    double t = AM * iy;
    return (t > RNMX) ? RNMX : t;
  }
  double gauss() {
    if (iset) {
      double v1, v2, rsq;
      do {
        v1 = 2.0 * uniform() - 1.0;
        v2 = 2.0 * uniform() - 1.0;
        rsq = v1 * v1 + v2 * v2;
      } while (rsq >= 1.0 || rsq == 0.0);
      double fac = sqrt(-2.0 * log(rsq) / rsq);
      gset = v1 * fac;
      iset = false;
      return v2 * fac;
    }
    iset = true;
    return gset;
  }
};

// Philox4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11 "Parallel random numbers:
// as easy as 1, 2, 3").  The same function runs in the CUDA kernels.
void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

}  // namespace

extern "C" void meo_restart_draws(unsigned long long seed, long long pixel, int run,
                                  double *out) {
  for (int blk = 0; blk < 2; blk++) {
    uint32_t c[4] = {(uint32_t)((unsigned long long)pixel & 0xffffffffu),
                     (uint32_t)((unsigned long long)pixel >> 32), (uint32_t)run,
                     (uint32_t)blk};
    philox4x32_10(c, (uint32_t)(seed & 0xffffffffu), (uint32_t)(seed >> 32));
    for (int h = 0; h < 2; h++) {
      double u1 = ((double)c[2 * h] + 0.5) * 2.3283064365386963e-10;
      double u2 = ((double)c[2 * h + 1] + 0.5) * 2.3283064365386963e-10;
      double r = sqrt(-2.0 * log(u1));
      double th = 6.283185307179586 * u2;
      out[blk * 4 + 2 * h] = r * cos(th);
      out[blk * 4 + 2 * h + 1] = r * sin(th);
    }
  }
}

// ---------------------------------------------------------------------------
// Plan = INIT_INV's per-process state.
// ---------------------------------------------------------------------------
struct meo_plan {
  me_config cfg;
  int nw = 0, ncut = 0, ic = 0, i0 = 0, i1 = 0, npar = 9;
  double lambda0 = 0, bshift = 0;
  double limits[9][2];
  double step[9];
  double w2[4];
  VoigtTables vt;
  std::vector<double> lambda;
  // instrument filter (an extension; the reference has none): observed
  // wavelength i = sum_k sub_w[k] * synthesis at flambda[i * nsub + k]
  int nsub = 1;
  std::vector<double> sub_w, flambda;
  // per-process scratch of the reference's structures
  std::vector<double> syn, fit, fit_best, ivnoise, jac;
  // STRUCT_STK's syn/fit/fit_best pointers, swapped per accepted trial and per
  // saved run exactly as the reference does; they persist across pixels.
  double *syn_p = nullptr, *fit_p = nullptr, *fitbest_p = nullptr;
  // RNG stream (reference mode)
  NrStream nr;
  int nr_seed = 0;
  bool nr_seeded = false;
};

namespace {

// clamp (Src/ME_SOLVER.c:52-69)
inline double clampb(double x, const double *b) { return x < b[0] ? b[0] : (x > b[1] ? b[1] : x); }

// bounds_check (Src/ME_SOLVER.c:370-406): clamp B, v, Doppler, a, eta, S,
// beta; fold theta into [0, pi]; phi modulo pi.
void bounds(double *p, const double lim[9][2]) {
  const double two_pi = 2.0 * kPi;
  p[0] = clampb(p[0], lim[0]);
  double t = fmod(p[1], two_pi);
  if (t < 0) t += two_pi;
  if (t > kPi) t = two_pi - t;
  p[1] = t;
  for (int i = 3; i < 9; i++) p[i] = clampb(p[i], lim[i]);
  double ph = fmod(p[2], kPi);
  if (ph < 0.0) ph += kPi;
  p[2] = ph;
}

// Milne_Eddington_Single (Src/ME_SOLVER.c:101-366) on the grid lambda[nw].
// syn [4][nw]; jac [4][9][nw] scaled by step[] when deriv.
template <class R>
void synthesize_on(const meo_plan &P, const double *lambda, int nw, const double *mp, bool deriv,
                   const double *step, R *syn, R *jac) {
  const R p4 = mp[4], p5 = mp[5], p6 = mp[6], p7 = mp[7], p8 = mp[8];
  const R eta_half = 0.5 * p6;
  const R b0 = p7 * p8;
  const R b1 = p7 - b0;
  const R bsh_n = P.bshift / p4;
  const R lam_n = P.lambda0 / p4;
  const R sth = sin(mp[1]);
  const R cth = cos(mp[1]);
  const R sth2 = sth * sth;
  const R cth2p1 = cth * cth + 1;
  const R c2p = cos(2. * mp[2]);
  const R s2p = sin(2. * mp[2]);
  const R kq = eta_half * sth2 * c2p;   // ScSqCs2
  const R ku = eta_half * sth2 * s2p;   // ScSqSc2
  const R kt = eta_half * 2.0 * sth * cth;  // ScCsB2
  const R kv = eta_half * cth;          // CsB2
  const R shift_b = mp[0] * bsh_n;
  const R shift_v = 1e3 * (-1e3 * mp[3] / kLightSpeed * P.lambda0 - P.lambda0) / p4;
  R *sI = syn, *sQ = syn + nw, *sU = syn + 2 * nw, *sV = syn + 3 * nw;
  R *jI = jac, *jQ = jac ? jac + 9 * nw : nullptr, *jU = jac ? jac + 18 * nw : nullptr,
    *jV = jac ? jac + 27 * nw : nullptr;
  const R s7 = step[7], s8 = step[8];

  for (int iw = 0; iw < nw; iw++) {
    R phi[3], psi[3], dphi[3][6], dpsi[3][6];
    R shift_w = 1e3 * lambda[iw] / p4 + shift_v;
    for (int q = -1; q <= 1; q++) {
      int k = q + 1;
      R v = shift_w + q * shift_b;
      R H = 0, L = 0;
      voigt(v, p5, &H, &L, P.vt);
      phi[k] = H / kSqrtPi;
      psi[k] = L / kSqrtPi;
      if (deriv) {
        R dH = 2. * (-v * H + p5 * L) / kSqrtPi;
        R dL = -2. * (-1. / kSqrtPi + p5 * H + v * L) / kSqrtPi;
        dphi[k][0] = q * bsh_n * dH;
        dpsi[k][0] = q * bsh_n * dL;
        dphi[k][3] = -1e6 / kLightSpeed * lam_n * dH;
        dpsi[k][3] = -1e6 / kLightSpeed * lam_n * dL;
        dphi[k][4] = -v / p4 * dH;
        dpsi[k][4] = -v / p4 * dL;
        dphi[k][5] = -dL;
        dpsi[k][5] = dH;
      }
    }
    R eta[4], rho[4];
    R phis = 0.5 * (phi[0] + phi[2]);
    R phit = phi[1] - phis;
    R psit = psi[1] - 0.5 * (psi[0] + psi[2]);
    eta[0] = eta_half * (phi[1] * sth2 + phis * cth2p1);
    eta[1] = phit * kq;
    eta[2] = phit * ku;
    eta[3] = (phi[0] - phi[2]) * kv;
    rho[1] = psit * kq;
    rho[2] = psit * ku;
    rho[3] = (psi[0] - psi[2]) * kv;

    R a1 = 1 + eta[0];
    R a1s = a1 * a1;
    R e2 = eta[1] * eta[1] + eta[2] * eta[2] + eta[3] * eta[3];
    R r2 = rho[1] * rho[1] + rho[2] * rho[2] + rho[3] * rho[3];
    R er = eta[1] * rho[1] + eta[2] * rho[2] + eta[3] * rho[3];
    R del = (a1s * (a1s - e2 + r2) - er * er);
    R b1d = b1 / del;
    R c1 = (eta[3] * rho[2] - eta[2] * rho[3]);
    R c2 = (eta[1] * rho[3] - eta[3] * rho[1]);
    R c3 = (eta[2] * rho[1] - eta[1] * rho[2]);
    sI[iw] = b0 + b1d * (a1 * (a1s + r2));
    sQ[iw] = -b1d * (a1s * eta[1] + a1 * c1 + rho[1] * er);
    sU[iw] = -b1d * (a1s * eta[2] + a1 * c2 + rho[2] * er);
    sV[iw] = -b1d * (a1s * eta[3] + a1 * c3 + rho[3] * er);
    if (!deriv) continue;

    R de[4][7], dr[4][7];
    // d/dB
    R ps = 0.5 * (dphi[0][0] + dphi[2][0]);
    de[0][0] = eta_half * (dphi[1][0] * sth2 + ps * cth2p1);
    de[1][0] = (dphi[1][0] - ps);
    de[2][0] = de[1][0] * ku;
    de[1][0] *= kq;
    de[3][0] = (dphi[0][0] - dphi[2][0]) * kv;
    dr[1][0] = (dpsi[1][0] - 0.5 * (dpsi[0][0] + dpsi[2][0]));
    dr[2][0] = dr[1][0] * ku;
    dr[1][0] *= kq;
    dr[3][0] = (dpsi[0][0] - dpsi[2][0]) * kv;
    // d/dtheta
    de[0][1] = phit * kt;
    de[1][1] = de[0][1] * c2p;
    de[2][1] = de[0][1] * s2p;
    de[3][1] = eta_half * (phi[0] - phi[2]) * (-sth);
    dr[1][1] = psit * kt * c2p;
    dr[2][1] = psit * kt * s2p;
    dr[3][1] = eta_half * (psi[0] - psi[2]) * (-sth);
    // d/dphi
    de[0][2] = 0;
    de[1][2] = -2. * eta[2];
    de[2][2] = 2. * eta[1];
    de[3][2] = 0;
    dr[1][2] = -2. * rho[2];
    dr[2][2] = 2. * rho[1];
    dr[3][2] = 0;
    // d/dv, d/dDoppler, d/da
    for (int k = 3; k < 6; k++) {
      ps = 0.5 * (dphi[0][k] + dphi[2][k]);
      de[0][k] = eta_half * (dphi[1][k] * sth2 + ps * cth2p1);
      de[1][k] = dphi[1][k] - ps;
      de[2][k] = de[1][k] * ku;
      de[1][k] *= kq;
      de[3][k] = (dphi[0][k] - dphi[2][k]) * kv;
      dr[1][k] = dpsi[1][k] - 0.5 * (dpsi[0][k] + dpsi[2][k]);
      dr[2][k] = dr[1][k] * ku;
      dr[1][k] *= kq;
      dr[3][k] = (dpsi[0][k] - dpsi[2][k]) * kv;
    }
    // d/deta0
    de[0][6] = eta[0] / p6;
    for (int s = 1; s < 4; s++) {
      de[s][6] = eta[s] / p6;
      dr[s][6] = rho[s] / p6;
    }
    for (int k = 0; k < 7; k++) {
      R da1 = de[0][k];
      R de2 = 2.0 * eta[1] * de[1][k] + 2.0 * eta[2] * de[2][k] + 2.0 * eta[3] * de[3][k];
      R dr2 = 2.0 * rho[1] * dr[1][k] + 2.0 * rho[2] * dr[2][k] + 2.0 * rho[3] * dr[3][k];
      R der = de[1][k] * rho[1] + eta[1] * dr[1][k] + de[2][k] * rho[2] + eta[2] * dr[2][k] +
                   de[3][k] * rho[3] + eta[3] * dr[3][k];
      R ddel = 2 * a1 * da1 * (a1s - e2 + r2) + a1s * (2 * a1 * da1 - de2 + dr2) -
                    2.0 * er * der;
      R b1dd = b1d / del;
      jI[k * nw + iw] =
          (b1dd * (del * (da1 * (a1s + r2) + a1 * (2 * a1 * da1 + dr2)) - ddel * (a1 * (a1s + r2)))) *
          step[k];
      jQ[k * nw + iw] =
          (-b1dd * (del * (2 * a1 * da1 * eta[1] + a1s * de[1][k] + da1 * c1 +
                           a1 * (de[3][k] * rho[2] + eta[3] * dr[2][k] - de[2][k] * rho[3] -
                                 eta[2] * dr[3][k]) +
                           dr[1][k] * er + rho[1] * der) -
                    ddel * (a1s * eta[1] + a1 * (eta[3] * rho[2] - eta[2] * rho[3]) + rho[1] * er))) *
          step[k];
      jU[k * nw + iw] =
          (-b1dd * (del * (2 * a1 * da1 * eta[2] + a1s * de[2][k] + da1 * c2 +
                           a1 * (de[1][k] * rho[3] + eta[1] * dr[3][k] - de[3][k] * rho[1] -
                                 eta[3] * dr[1][k]) +
                           dr[2][k] * er + rho[2] * der) -
                    ddel * (a1s * eta[2] + a1 * (eta[1] * rho[3] - eta[3] * rho[1]) + rho[2] * er))) *
          step[k];
      jV[k * nw + iw] =
          (-b1dd * (del * (2 * a1 * da1 * eta[3] + a1s * de[3][k] + da1 * c3 +
                           a1 * (de[2][k] * rho[1] + eta[2] * dr[1][k] - de[1][k] * rho[2] -
                                 eta[1] * dr[2][k]) +
                           dr[3][k] * er + rho[3] * der) -
                    ddel * (a1s * eta[3] + a1 * (eta[2] * rho[1] - eta[1] * rho[2]) + rho[3] * er))) *
          step[k];
    }
    R T = (1 - p8) / del;
    jI[7 * nw + iw] = (p8 + T * (a1 * (a1s + r2))) * s7;
    jQ[7 * nw + iw] = (-T * (a1s * eta[1] + a1 * c1 + rho[1] * er)) * s7;
    jU[7 * nw + iw] = (-T * (a1s * eta[2] + a1 * c2 + rho[2] * er)) * s7;
    jV[7 * nw + iw] = (-T * (a1s * eta[3] + a1 * c3 + rho[3] * er)) * s7;
    T = p7 / del;
    jI[8 * nw + iw] = (p7 - T * (a1 * (a1s + r2))) * s8;
    jQ[8 * nw + iw] = (T * (a1s * eta[1] + a1 * c1 + rho[1] * er)) * s8;
    jU[8 * nw + iw] = (T * (a1s * eta[2] + a1 * c2 + rho[2] * er)) * s8;
    jV[8 * nw + iw] = (T * (a1s * eta[3] + a1 * c3 + rho[3] * er)) * s8;
  }
}

// The synthesis the inversion sees: Milne_Eddington_Single on the plan's
// grid, or, with an instrument filter (no reference counterpart), on the
// filter's sub-wavelengths followed by the weighted sum over each observed
// wavelength's sub-wavelengths (in order, from zero) of the profiles and of
// the Jacobian rows.
template <class R>
void synthesize(const meo_plan &P, const double *mp, bool deriv, const double *step, R *syn,
                R *jac) {
  if (P.nsub <= 1) {
    synthesize_on<R>(P, P.lambda.data(), P.nw, mp, deriv, step, syn, jac);
    return;
  }
  const int nl = P.nw, K = P.nsub, nf = nl * K;
  std::vector<R> fs((size_t)4 * nf), fj(deriv ? (size_t)36 * nf : 0);
  synthesize_on<R>(P, P.flambda.data(), nf, mp, deriv, step, fs.data(),
                   deriv ? fj.data() : nullptr);
  for (int row = 0; row < 4; row++)
    for (int i = 0; i < nl; i++) {
      R acc = 0;
      for (int k = 0; k < K; k++) acc += P.sub_w[k] * fs[(size_t)row * nf + i * K + k];
      syn[row * nl + i] = acc;
    }
  if (deriv)
    for (int row = 0; row < 36; row++)
      for (int i = 0; i < nl; i++) {
        R acc = 0;
        for (int k = 0; k < K; k++) acc += P.sub_w[k] * fj[(size_t)row * nf + i * K + k];
        jac[row * nl + i] = acc;
      }
}

// The Gaussian table of the `filter` keyword: `points` offsets uniform over
// +-1.5 FWHM [mA], weights exp(-d^2 / 2 sigma^2) normalised to sum 1.
void gaussian_filter(double fwhm, int points, std::vector<double> &off, std::vector<double> &w) {
  off.assign(points, 0.0);
  w.assign(points, 1.0);
  if (points <= 1) return;
  const double sigma = fwhm / (2.0 * sqrt(2.0 * log(2.0)));
  double sum = 0.0;
  for (int k = 0; k < points; k++) {
    off[k] = -1.5 * fwhm + 3.0 * fwhm * k / (points - 1);
    w[k] = exp(-off[k] * off[k] / (2.0 * sigma * sigma));
    sum += w[k];
  }
  for (int k = 0; k < points; k++) w[k] /= sum;
}

void set_filter(meo_plan *P, const double *off_mA, const double *w, int K) {
  P->nsub = K;
  P->sub_w.assign(w, w + K);
  P->flambda.resize((size_t)P->nw * K);
  for (int i = 0; i < P->nw; i++)
    for (int k = 0; k < K; k++) P->flambda[(size_t)i * K + k] = P->lambda[i] + off_mA[k] * 1e-3;
}

// Per-pixel state of the reference's STRUCT_STK / STRUCT_PARA / STRUCT_LM.
struct PixelState {
  double norm0 = 0, normp = 1;
  double guess[9];
  double lim7[2];
  double step[9];
};

// Init_Guess (Src/ME_SOLVER.c:445-676).  Returns 1 when mean(I) < Icriteria.
int init_guess(const meo_plan &P, const double *prof, PixelState &st) {
  const int nw = P.nw;
  const double *pI = prof, *pQ = prof + nw, *pU = prof + 2 * nw, *pV = prof + 3 * nw;
  const double *lam = P.lambda.data();
  const double lam0 = P.lambda0;
  double isum = 0., imin = 1e10, qsum = 0., usum = 0., vsum = 0.;
  double imax = 0, lmax = 0., vmax = 0., vmin = 0.;
  int i_imin = 0, i_vmax = 0, i_vmin = 0;
  std::vector<double> lp(nw, 0.0);
  for (int iw = 0; iw < nw; iw++) {
    if (imax < pI[iw]) imax = pI[iw];
    if (imin > pI[iw]) {
      i_imin = iw;
      imin = pI[iw];
    }
    isum += pI[iw];
    qsum += fabs(pQ[iw]);
    usum += fabs(pU[iw]);
    vsum += fabs(pV[iw]);
  }
  for (int iw = P.i0; iw <= P.i1; iw++) {
    lp[iw] = sqrt(pQ[iw] * pQ[iw] + pU[iw] * pU[iw]);
    if (lmax < lp[iw]) lmax = lp[iw];
    if (vmin > pV[iw]) {
      i_vmin = iw;
      vmin = pV[iw];
    } else if (vmax < pV[iw]) {
      i_vmax = iw;
      vmax = pV[iw];
    }
  }
  double imean = isum / nw;
  if (imean < P.cfg.icriteria) return 1;

  st.norm0 = 1e-2 * imean;
  st.norm0 *= st.norm0;
  st.normp = 1 + qsum * qsum / (isum * isum) * P.w2[1] + usum * usum / (isum * isum) * P.w2[2] +
             vsum * vsum / (isum * isum) * P.w2[3];

  lmax = 100 * lmax / imean;
  vmin = 100 * vmin / imean;
  vmax = 100 * vmax / imean;

  const bool ir_line = (lam0 > 15640 && lam0 < 15660);
  const double thr_v = ir_line ? 1.5 : 5.0;
  const double thr_l = ir_line ? 2.5 : 5.0;

  double blos = 0., bpos;
  double lv = 0.5 * (vmax - vmin);
  double factor = imin > 0.9 * imax ? 2. : 1.;
  if (lv > 0.1) {
    blos = 20 + P.cfg.vcoeffi * lv * factor;
    if (i_vmin < i_vmax) blos = -blos;
  }
  bpos = 100 + P.cfg.lcoeffi * lmax * factor;
  bpos = bpos < 2200 ? bpos : 2200;

  double *g = st.guess;
  double tmp = 0;
  g[3] = 0;
  if (lv > thr_v) {
    tmp = 0.5 * (lam[i_vmin] + lam[i_vmax]) - lam0;
    g[3] = tmp / lam0 * kLightSpeed / 1e3;
  } else {
    bool found = false;
    // The reference reads pI[i_imin-2 .. i_imin+2] without a range check; on
    // grids with nl < 10 (ncut < 2) that can fall outside the profile, where
    // this restatement treats the minimum test as failed.
    if (imin < 0.9 * imax && i_imin >= P.ncut && i_imin < nw - P.ncut && i_imin >= 2 &&
        i_imin + 2 <= nw - 1) {
      if (pI[i_imin - 1] < pI[i_imin - 2] && pI[i_imin] < pI[i_imin - 1] &&
          pI[i_imin] < pI[i_imin + 1] && pI[i_imin + 1] < pI[i_imin + 2]) {
        tmp = lam[i_imin] - lam0;
        found = true;
      }
    }
    if (!found) {
      double lsum = 0, wsum = 0.;
      int lo = (P.ic > 7) ? (P.ic - 7) : 0;
      int hi = (P.ic + 7 < nw) ? (P.ic + 7) : (nw - 1);
      for (int iw = lo; iw <= hi; iw++) {
        const double d = (imax - pI[iw]);
        lsum += lam[iw] * d;
        wsum += d;
      }
      tmp = lsum / wsum - lam0;
    }
    g[3] = tmp / lam0 * kLightSpeed / 1e3;
  }
  g[0] = sqrt(blos * blos + bpos * bpos);
  g[1] = acos(blos / g[0]);
  if (g[0] > 3000) g[0] = 3000;

  double wsum = 0., phi = 0.;
  for (int iw = P.i0; iw <= P.i1; iw++) {
    if (lp[iw] > thr_l) {
      double t = 0.5 * atan2(pU[iw], pQ[iw]);
      t = t > 0 ? t : kPi + t;
      phi += t * lp[iw];
      wsum += lp[iw];
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
  st.lim7[0] = imax * 0.6;
  st.lim7[1] = imax * 1.4;
  memcpy(st.step, P.step, sizeof(st.step));
  st.step[7] = imax * 0.1;
  double lim[9][2];
  memcpy(lim, P.limits, sizeof(lim));
  lim[7][0] = st.lim7[0];
  lim[7][1] = st.lim7[1];
  bounds(g, lim);
  return 0;
}

// Golub-Reinsch SVD (Householder bidiagonalisation, accumulation of V and U,
// implicit-shift QR on the bidiagonal), the Numerical Recipes svdcmp form the
// reference uses: Src/SVD_TEMPLATE.h:49-344.  a[m*n] row-major is replaced by
// U; w[n]; v[n*n].  Returns 1 if the QR sweep limit (50) was hit.
template <class R>
R pythag(R a, R b) {  // Src/SVD_TEMPLATE.h:49-80
  R aa = a > 0 ? a : -a;
  R ab = b > 0 ? b : -b;
  R mx = aa > ab ? aa : ab;
  if (mx == 0) return 0;
  if (mx < 1e150) return sqrt(a * a + b * b);
  R mn = aa > ab ? ab : aa;
  R r = mn / mx;
  return mx * sqrt(1.0 + r * r);
}

template <class R>
int gr_svd(R *a, int m, int n, R *w, R *v) {
#define A(i, j) a[(i) * n + (j)]
#define V(i, j) v[(i) * n + (j)]
  int l = 0, nm = 0;
  R anorm = 0., c, f, g = 0., h, s, scale = 0., x, y, z;
  R rv1[16];
  int hit_limit = 0;
  // Householder reduction to bidiagonal form
  for (int i = 0; i < n; i++) {
    l = i + 1;
    rv1[i] = scale * g;
    g = s = scale = 0.0;
    if (i < m) {
      for (int k = i; k < m; k++) scale += fabs(A(k, i));
      if (scale != 0.0) {
        for (int k = i; k < m; k++) {
          A(k, i) /= scale;
          s += A(k, i) * A(k, i);
        }
        f = A(i, i);
        g = f >= 0 ? -sqrt(s) : sqrt(s);
        h = f * g - s;
        A(i, i) = f - g;
        for (int j = l; j < n; j++) {
          s = 0.0;
          for (int k = i; k < m; k++) s += A(k, i) * A(k, j);
          f = s / h;
          for (int k = i; k < m; k++) A(k, j) += f * A(k, i);
        }
        for (int k = i; k < m; k++) A(k, i) *= scale;
      }
    }
    w[i] = scale * g;
    g = s = scale = 0.0;
    if (i < m && i != n - 1) {
      for (int k = l; k < n; k++) scale += fabs(A(i, k));
      if (scale != 0.0) {
        for (int k = l; k < n; k++) {
          A(i, k) /= scale;
          s += A(i, k) * A(i, k);
        }
        f = A(i, l);
        g = f >= 0 ? -sqrt(s) : sqrt(s);
        h = f * g - s;
        A(i, l) = f - g;
        for (int k = l; k < n; k++) rv1[k] = A(i, k) / h;
        for (int j = l; j < m; j++) {
          s = 0.0;
          for (int k = l; k < n; k++) s += A(j, k) * A(i, k);
          for (int k = l; k < n; k++) A(j, k) += s * rv1[k];
        }
        for (int k = l; k < n; k++) A(i, k) *= scale;
      }
    }
    R t = fabs(w[i]) + fabs(rv1[i]);
    if (anorm < t) anorm = t;
  }
  // accumulate right-hand transformations
  for (int i = n - 1; i >= 0; i--) {
    if (i < n - 1) {
      if (g != 0.0) {
        for (int j = l; j < n; j++) V(j, i) = (A(i, j) / A(i, l)) / g;
        for (int j = l; j < n; j++) {
          s = 0.0;
          for (int k = l; k < n; k++) s += A(i, k) * V(k, j);
          for (int k = l; k < n; k++) V(k, j) += s * V(k, i);
        }
      }
      for (int j = l; j < n; j++) V(i, j) = V(j, i) = 0.0;
    }
    V(i, i) = 1.0;
    g = rv1[i];
    l = i;
  }
  // accumulate left-hand transformations
  for (int i = (m <= n ? m : n) - 1; i >= 0; i--) {
    l = i + 1;
    g = w[i];
    for (int j = l; j < n; j++) A(i, j) = 0.0;
    if (g != 0.0) {
      g = 1.0 / g;
      for (int j = l; j < n; j++) {
        s = 0.0;
        for (int k = l; k < m; k++) s += A(k, i) * A(k, j);
        f = (s / A(i, i)) * g;
        for (int k = i; k < m; k++) A(k, j) += f * A(k, i);
      }
      for (int j = i; j < m; j++) A(j, i) *= g;
    } else {
      for (int j = i; j < m; j++) A(j, i) = 0.0;
    }
    A(i, i) += 1.0;
  }
  // diagonalise the bidiagonal form
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
          h = pythag(f, g);
          w[i] = h;
          h = 1.0 / h;
          c = g * h;
          s = -f * h;
          for (int j = 0; j < m; j++) {
            y = A(j, nm);
            z = A(j, i);
            A(j, nm) = y * c + z * s;
            A(j, i) = z * c - y * s;
          }
        }
      }
      z = w[k];
      if (l == k) {
        if (z < 0.0) {
          w[k] = -z;
          for (int j = 0; j < n; j++) V(j, k) = -V(j, k);
        }
        break;
      }
      if (its == 50 - 1) hit_limit = 1;  // the reference exits here (Src/SVD_TEMPLATE.h:283-286)
      x = w[l];
      nm = k - 1;
      y = w[nm];
      g = rv1[nm];
      h = rv1[k];
      f = ((y - z) * (y + z) + (g - h) * (g + h)) / (2.0 * h * y);
      g = pythag(f, R(1.0));
      R sg = f >= 0.0 ? g : -g;
      f = ((x - z) * (x + z) + h * (y / (f + sg) - h)) / x;
      c = s = 1.0;
      for (int j = l; j <= nm; j++) {
        int i = j + 1;
        g = rv1[i];
        y = w[i];
        h = s * g;
        g *= c;
        z = pythag(f, h);
        rv1[j] = z;
        c = f / z;
        s = h / z;
        f = x * c + g * s;
        g = g * c - x * s;
        h = y * s;
        y *= c;
        for (int jj = 0; jj < n; jj++) {
          x = V(jj, j);
          z = V(jj, i);
          V(jj, j) = x * c + z * s;
          V(jj, i) = z * c - x * s;
        }
        z = pythag(f, h);
        w[j] = z;
        if (z != 0.0) {
          z = 1.0 / z;
          c = f * z;
          s = h * z;
        }
        f = c * g + s * y;
        x = c * y - s * g;
        for (int jj = 0; jj < m; jj++) {
          y = A(jj, j);
          z = A(jj, i);
          A(jj, j) = y * c + z * s;
          A(jj, i) = z * c - y * s;
        }
      }
      rv1[l] = 0.0;
      rv1[k] = f;
      w[k] = x;
    }
  }
  return hit_limit;
#undef A
#undef V
}

// svbksb (Src/SVD_TEMPLATE.h:348-406): x = V diag(1/w) U^T b, w <= 1e-50 skipped.
template <class R>
void gr_backsub(const R *u, const R *v, const R *w, const R *b, int n, R *x) {
  R t[16];
  for (int j = 0; j < n; j++) {
    R s = 0.0;
    if (w[j] > 1e-50) {
      for (int i = 0; i < n; i++) s += u[i * n + j] * b[i];
      s /= w[j];
    }
    t[j] = s;
  }
  for (int i = 0; i < n; i++) {
    R s = 0.0;
    for (int j = 0; j < n; j++) s += v[i * n + j] * t[j];
    x[i] = s;
  }
}

// One pixel's LM machinery: STRUCT_LM + the buffers of STRUCT_STK.
struct LmState {
  int npar;
  double hess[81], vmat[81], w[9], jvec[9], sol[9];
  double damp, ratio, chisq, penalty;
  double *syn, *fit, *fit_best;  // swapped pointers, as the reference
  double par_a[9], par_b[9], par_c[9];
  double *par, *par_best, *par_tmp;
  double chisq_run, chisq_best;
  long long c_runs, c_iter, c_trials, c_acc, c_syn, c_jac, c_maxtrial;
};

}  // namespace

// ---------------------------------------------------------------------------
// extern "C" API
// ---------------------------------------------------------------------------

extern "C" int meo_plan_create(const me_config *cfg, const double *lambda, int nl,
                               meo_plan **out) {
  if (!cfg || !lambda || !out || nl < 4 || nl > ME_MAX_NL) return ME_ERR_ARG;
  meo_plan *P = new meo_plan();
  P->cfg = *cfg;
  P->nw = nl;
  P->lambda.assign(lambda, lambda + nl);
  // INIT_INV (Src/INV_INIT.c:121-177)
  P->lambda0 = cfg->line_lambda0[0];
  P->bshift = 4.6686e-10 * cfg->line_geff[0] * cfg->line_lambda0[0] * cfg->line_lambda0[0];
  P->npar = 0;
  for (int i = 0; i < 9; i++) {
    if (!cfg->fixed[i]) P->npar++;
    P->limits[i][0] = cfg->bounds[i][0];
    P->limits[i][1] = cfg->bounds[i][1];
    P->step[i] = cfg->step[i];
  }
  P->ncut = nl / 5;
  const double c = 299792458.0;
  double t = (lambda[P->ncut] - P->lambda0) * c / 1e3;
  if (P->limits[3][0] < t) P->limits[3][0] = t;
  t = (lambda[nl - 1 - P->ncut] - P->lambda0) * c / 1e3;
  if (P->limits[3][1] > t) P->limits[3][1] = t;
  // ic: the last index iw < nl-1 with lambda[iw] < lambda0 (the reference's
  // boolean arithmetic, Src/INV_INIT.c:150-156); 0 when there is none (the
  // reference leaves Stk->ic at its zero initialisation).
  P->ic = 0;
  for (int iw = 0; iw < nl - 1; iw++) {
    double t1 = P->lambda0 > lambda[iw];
    double t2 = lambda[iw + 1] * P->lambda0;
    if (t1 > 0 && t2 > 0) P->ic = t1 < t2 ? iw : iw + 1;
  }
  int r1 = 2, r2 = 2;
  if (P->ic - P->ncut >= 2) r1 = P->ic - P->ncut;
  if (nl - 1 - P->ncut - P->ic >= 2) r2 = nl - 1 - P->ncut - P->ic;
  int range = r1 > r2 ? r1 : r2;
  P->i0 = P->ic - range;
  if (P->i0 < 0) {
    P->i0 = 0;
    range = P->ic - P->i0;
  }
  P->i1 = P->ic + range;
  if (P->i1 > nl - 1) {
    P->i1 = nl - 1;
    range = P->i1 - P->ic;
    P->i0 = P->ic - range;
  }
  for (int s = 0; s < 4; s++) P->w2[s] = cfg->weights[s] * cfg->weights[s];
  P->vt.init(cfg->nfigures);
  P->syn.assign(4 * nl, 0.0);
  P->fit.assign(4 * nl, 0.0);
  P->fit_best.assign(4 * nl, 0.0);
  P->ivnoise.assign(4 * nl, 0.0);
  P->jac.assign(36 * nl, 0.0);
  P->syn_p = P->syn.data();
  P->fit_p = P->fit.data();
  P->fitbest_p = P->fit_best.data();
  if (cfg->filter_fwhm > 0 && cfg->filter_points > 1) {
    std::vector<double> off, w;
    gaussian_filter(cfg->filter_fwhm, cfg->filter_points, off, w);
    set_filter(P, off.data(), w.data(), cfg->filter_points);
  }
  *out = P;
  return ME_OK;
}

extern "C" int meo_plan_set_filter(meo_plan *p, const double *offsets_mA, const double *weights,
                                   int k) {
  if (!p || k < 1 || k > ME_MAX_FILTER || (k > 1 && (!offsets_mA || !weights))) return ME_ERR_ARG;
  if (k == 1) {
    p->nsub = 1;
    p->sub_w.clear();
    p->flambda.clear();
    return ME_OK;
  }
  set_filter(p, offsets_mA, weights, k);
  return ME_OK;
}

extern "C" void meo_plan_destroy(meo_plan *p) { delete p; }

extern "C" int meo_plan_facts(const meo_plan *p, me_plan_facts *o) {
  if (!p || !o) return ME_ERR_ARG;
  o->nl = p->nw;
  o->ncut = p->ncut;
  o->ic = p->ic;
  o->i0 = p->i0;
  o->i1 = p->i1;
  o->npar = p->npar;
  o->bshift = p->bshift;
  memcpy(o->limits, p->limits, sizeof(o->limits));
  o->fadd_a = p->vt.a;
  return ME_OK;
}

namespace {

struct PixelCtx {
  const meo_plan *P;
  const double *prof;
  PixelState st;
  double lim[9][2];
  LmState *lm;
  std::vector<double> *jac, *ivn;
};

// Loss_Function (Src/LM_FIT.c:89-120).
double loss(const PixelCtx &C, const double *syn) {
  const int n4 = 4 * C.P->nw;
  double chisq = 0;
  for (int i = 0; i < n4; i++) {
    double d = syn[i] - C.prof[i];
    chisq += d * d * (*C.ivn)[i];
  }
  chisq /= (4. * C.P->nw);
  return chisq;
}

// Hessian_Compute (Src/LM_FIT.c:240-350): H = J^T W J and g = -J^T W r over the
// free parameters.
void normal_equations(const PixelCtx &C, const double *syn, double *H, double *g) {
  const meo_plan &P = *C.P;
  const int nw = P.nw;
  const double *iv = C.ivn->data();
  const double *J = C.jac->data();
  const int n = C.lm->npar;
  int ip = 0;
  for (int ii = 0; ii < 9; ii++) {
    if (P.cfg.fixed[ii]) continue;
    int jp = ip;
    for (int jj = ii; jj < 9; jj++) {
      if (P.cfg.fixed[jj]) continue;
      double s = 0;
      for (int iw = 0; iw < nw; iw++) {
        s += iv[iw] * J[ii * nw + iw] * J[jj * nw + iw];
        s += iv[nw + iw] * J[9 * nw + ii * nw + iw] * J[9 * nw + jj * nw + iw];
        s += iv[2 * nw + iw] * J[18 * nw + ii * nw + iw] * J[18 * nw + jj * nw + iw];
        s += iv[3 * nw + iw] * J[27 * nw + ii * nw + iw] * J[27 * nw + jj * nw + iw];
      }
      H[jp * n + ip] = s;
      H[ip * n + jp] = s;
      jp++;
    }
    double s = 0;
    for (int iw = 0; iw < nw; iw++) {
      s -= iv[iw] * J[ii * nw + iw] * (syn[iw] - C.prof[iw]);
      s -= iv[nw + iw] * J[9 * nw + ii * nw + iw] * (syn[nw + iw] - C.prof[nw + iw]);
      s -= iv[2 * nw + iw] * J[18 * nw + ii * nw + iw] * (syn[2 * nw + iw] - C.prof[2 * nw + iw]);
      s -= iv[3 * nw + iw] * J[27 * nw + ii * nw + iw] * (syn[3 * nw + iw] - C.prof[3 * nw + iw]);
    }
    g[ip] = s;
    ip++;
  }
}

// Get_Regul (Src/LM_FIT.c:354-396).
void regularise(const PixelCtx &C, const double *par, bool with_matrix) {
  const me_config &cfg = C.P->cfg;
  LmState &L = *C.lm;
  int ip = -1;
  L.penalty = 0.0;
  for (int ii = 0; ii < 9; ii++) {
    if (cfg.fixed[ii]) continue;
    ip++;
    if (!cfg.regul[ii]) continue;
    double r = par[ii] - cfg.regul_value[ii];
    L.penalty += r * r * cfg.regul_weight[ii];
    if (with_matrix) {
      double rj = 1. * r * cfg.regul_weight[ii];
      double rh = 1. * 1. * cfg.regul_weight[ii];
      L.jvec[ip] -= rj * L.ratio;
      L.hess[ip * L.npar + ip] += rh * L.ratio;
    }
  }
}

// SVD_solve_mem (Src/LM_FIT.c:400-469): SVD of the (undamped) normal matrix in
// place, truncation ladder from SVDthreshold x5 until |step| <= 0.5 or the
// threshold passes 2e-3, then clamp.
void svd_solve(const PixelCtx &C) {
  LmState &L = *C.lm;
  const int n = L.npar;
  const double maxstep = 0.5;
  double thr = C.P->cfg.svd_threshold;
  gr_svd(L.hess, n, n, L.w, L.vmat);
  double wmax = L.w[0];
  for (int i = 1; i < n; i++) wmax = wmax > L.w[i] ? wmax : L.w[i];
  while (1) {
    double wthr = wmax * thr;
    for (int i = 0; i < n; i++)
      if (L.w[i] < wthr) L.w[i] = 0.;
    gr_backsub(L.hess, L.vmat, L.w, L.jvec, n, L.sol);
    bool inside = true;
    for (int i = 0; i < n; i++) {
      if (L.sol[i] > maxstep || L.sol[i] < -maxstep) {
        inside = false;
        break;
      }
    }
    if (inside) break;
    if (thr > 2e-3) {
      for (int i = 0; i < n; i++) {
        if (L.sol[i] > maxstep)
          L.sol[i] = maxstep;
        else if (L.sol[i] < -maxstep)
          L.sol[i] = -maxstep;
      }
      break;
    }
    thr *= 5.;
  }
}

// Par_update (Src/LM_FIT.c:205-236).
void apply_step(const PixelCtx &C, double *par) {
  int ip = 0;
  for (int ii = 0; ii < 9; ii++) {
    if (C.P->cfg.fixed[ii]) continue;
    par[ii] += C.lm->sol[ip] * C.st.step[ii];
    ip++;
  }
}

// Trial_Synthesis (Src/LM_FIT.c:473-527).  The damped copy the reference
// builds (Src/LM_FIT.c:498-507) is never read, so it is not built here.
double trial(PixelCtx &C) {
  LmState &L = *C.lm;
  svd_solve(C);
  for (int i = 0; i < 9; i++) L.par_tmp[i] = L.par[i];
  apply_step(C, L.par_tmp);
  bounds(L.par_tmp, C.lim);
  synthesize<double>(*C.P, L.par_tmp, false, C.st.step, L.syn, nullptr);
  L.c_syn++;
  L.chisq = loss(C, L.syn);
  if (C.P->cfg.regul_any) regularise(C, L.par_tmp, false);
  return L.chisq;
}

// LM_FIT (Src/LM_FIT.c:531-661).  Returns the iteration index it stopped at.
int lm_fit(PixelCtx &C) {
  LmState &L = *C.lm;
  const me_config &cfg = C.P->cfg;
  synthesize(*C.P, L.par, true, C.st.step, L.syn, C.jac->data());
  L.c_jac++;
  const double limit = 0.1;
  L.ratio = 1.0;
  double chisq = loss(C, L.syn);
  if (cfg.regul_any) {
    regularise(C, L.par, false);
    if (L.penalty > limit * L.chisq) L.ratio = limit * chisq / L.penalty;
  }
  const double damp0 = L.damp;
  bool accepted = false;
  double chisq_new = 0;
  int it;
  for (it = 0; it < cfg.num_iter; it++) {
    accepted = false;
    normal_equations(C, L.syn, L.hess, L.jvec);
    if (cfg.regul_any) regularise(C, L.par, true);
    L.c_iter++;
    long long k = 0;
    do {
      chisq_new = trial(C);
      L.c_trials++;
      k++;
      if (chisq_new < chisq) {
        if (cfg.regul_any) {
          if (L.penalty > limit * L.chisq) L.ratio = limit * chisq / L.penalty;
        }
        accepted = true;
        std::swap(L.par, L.par_tmp);
        std::swap(L.syn, L.fit);
        synthesize(*C.P, L.par, true, C.st.step, L.syn, C.jac->data());
        L.c_jac++;
        L.c_acc++;
        // Lambda_propose (Src/LM_FIT.c:140-143)
        L.damp /= cfg.lambda_accept;
        if (L.damp < cfg.lambda_limits[0]) L.damp = cfg.lambda_limits[0];
      } else {
        accepted = false;
        // Lambda_propose (Src/LM_FIT.c:145-150)
        L.damp *= cfg.lambda_reject;
        if (L.damp > cfg.lambda_limits[1]) break;
      }
    } while (!accepted);
    if (k > L.c_maxtrial) L.c_maxtrial = k;
    L.damp = damp0;
    if (accepted) {
      if (((chisq - chisq_new) / chisq) < cfg.convg_criteria) {
        chisq = chisq_new;
        break;
      }
      chisq = chisq_new;
    } else {
      break;
    }
  }
  L.chisq_run = chisq / C.st.normp;
  return it;
}

// Random_Jump (Src/LM_FIT.c:157-201).
void restart_point(PixelCtx &C, int irun, int rng_mode, long long pixel, meo_plan *P) {
  LmState &L = *C.lm;
  double *m = L.par;
  const double *best = L.par_best;
  const double *g = C.st.guess;
  if (irun < 4) {
    for (int i = 0; i < 9; i++) m[i] = best[i];
    m[2] = g[2] + kPi / 4. * irun;
  } else {
    double z[8];
    if (rng_mode == MEO_RNG_NR) {
      for (int k = 0; k < 8; k++) z[k] = P->nr.gauss();
    } else {
      meo_restart_draws(P->cfg.rng_seed, pixel, irun, z);
    }
    m[0] = g[0] * (1 + 0.6 * z[0]);
    m[1] = g[1] + kPi / 8. * z[1];
    m[2] = g[2] + kPi / 4. * (irun + 0.3 * z[2]);
    m[3] = g[3] + 5. * z[3];
    m[4] = best[4] * (1 + 0.2 * z[4]);
    m[5] = g[5] + 0.1 * z[5];
    m[6] = g[6] + 5 * z[6];
    m[7] = best[7];
    m[8] = g[8] + 0.1 * z[7];
  }
  bounds(m, C.lim);
}

}  // namespace

extern "C" int meo_invert(meo_plan *P, const double *prof, long npix, long pixel_offset,
                          double *res, double *fit, int rng_mode, int nr_seed,
                          double *carry_chisq, long long *counters) {
  if (!P || !prof || !res || npix < 0) return ME_ERR_ARG;
  const me_config &cfg = P->cfg;
  const int nw = P->nw;
  const int n4 = 4 * nw;
  if (rng_mode == MEO_RNG_NR && (!P->nr_seeded || P->nr_seed != nr_seed)) {
    P->nr.seed(nr_seed);
    P->nr_seed = nr_seed;
    P->nr_seeded = true;
  }
  LmState L;
  memset(&L, 0, sizeof(L));
  L.npar = P->npar;
  L.chisq = carry_chisq ? *carry_chisq : 0.0;
  L.syn = P->syn_p;
  L.fit = P->fit_p;
  L.fit_best = P->fitbest_p;
  L.par = L.par_a;
  L.par_best = L.par_b;
  L.par_tmp = L.par_c;
  for (long ip = 0; ip < npix; ip++) {
    const double *pp = prof + ip * n4;
    double *r = res + ip * 10;
    L.c_runs = L.c_iter = L.c_trials = L.c_acc = L.c_syn = L.c_jac = L.c_maxtrial = 0;
    // INVERSION_MULTI gate (Src/LM_FIT.c:776-785)
    double imean = 0.0;
    for (int iw = 0; iw < nw; iw++) imean += pp[iw];
    imean /= nw;
    bool valid = !(isnan(imean) || imean < cfg.icriteria);
    int final_run = -1;
    if (valid) {
      PixelCtx C;
      C.P = P;
      C.prof = pp;
      C.lm = &L;
      C.jac = &P->jac;
      C.ivn = &P->ivnoise;
      // INVERSION (Src/LM_FIT.c:665-742)
      if (init_guess(*P, pp, C.st)) {
        valid = false;
      } else {
        memcpy(C.lim, P->limits, sizeof(C.lim));
        C.lim[7][0] = C.st.lim7[0];
        C.lim[7][1] = C.st.lim7[1];
        for (int i = 0; i < 9; i++) L.par[i] = C.st.guess[i];
        L.damp = cfg.damp;
        // Noise_Init (Src/ME_SOLVER.c:410-441)
        const double inv_n0 = 1. / C.st.norm0;
        for (int s = 0; s < 4; s++) {
          double v = P->w2[s] * inv_n0;
          for (int iw = 0; iw < nw; iw++) P->ivnoise[s * nw + iw] = v;
        }
        int irun;
        for (irun = 0; irun < cfg.num_run * 4; irun++) {
          if (irun > 0) restart_point(C, irun, rng_mode, pixel_offset + ip, P);
          lm_fit(C);
          L.c_runs++;
          bool save = false;
          if (L.chisq_run < cfg.chisq_criteria) {
            save = true;
          } else if (irun == 0) {
            save = true;
          } else if (L.chisq_run < L.chisq_best) {
            save = true;
          }
          if (save) {  // sav_par (Src/LM_FIT.c:62-85)
            std::swap(L.par, L.par_best);
            std::swap(L.fit, L.fit_best);
            L.chisq_best = L.chisq_run;
          }
          if (L.chisq_run < cfg.chisq_criteria) {
            if (irun >= 4 || irun == cfg.num_run * 4) break;
          }
          if (irun >= cfg.num_run * 2) {
            if (L.chisq_best < cfg.chisq_criteria * 2) break;
          }
        }
        final_run = irun;
        if (L.par_best[1] > kPi) L.par_best[1] -= kPi;
        if (cfg.hmi_ref) {
          L.par_best[2] += 0.5 * kPi;
          if (L.par_best[2] > kPi) L.par_best[2] -= kPi;
        }
        if (irun == 0) valid = false;  // INVERSION returned 0 (Src/LM_FIT.c:788)
      }
    }
    if (valid) {
      for (int i = 0; i < 9; i++) r[i] = L.par_best[i];
      r[9] = L.chisq_best;
      if (fit) memcpy(fit + ip * n4, L.fit_best, sizeof(double) * n4);
    } else {
      memset(r, 0, sizeof(double) * 10);
      if (fit) memset(fit + ip * n4, 0, sizeof(double) * n4);
    }
    if (counters) {
      long long *c = counters + ip * 8;
      c[0] = L.c_runs;
      c[1] = L.c_iter;
      c[2] = L.c_trials;
      c[3] = L.c_acc;
      c[4] = L.c_syn;
      c[5] = L.c_jac;
      c[6] = L.c_maxtrial;
      c[7] = final_run;
    }
  }
  P->syn_p = L.syn;
  P->fit_p = L.fit;
  P->fitbest_p = L.fit_best;
  if (carry_chisq) *carry_chisq = L.chisq;
  return ME_OK;
}

extern "C" int meo_synth(meo_plan *P, const double *par, int deriv, double step7, double *syn,
                         double *jac) {
  if (!P || !par || !syn) return ME_ERR_ARG;
  double step[9];
  memcpy(step, P->step, sizeof(step));
  step[7] = step7;
  std::vector<double> J(deriv ? 36 * P->nw : 0);
  synthesize<double>(*P, par, deriv != 0, step, syn, deriv ? J.data() : nullptr);
  if (deriv && jac) memcpy(jac, J.data(), sizeof(double) * J.size());
  return ME_OK;
}

extern "C" int meo_faddeeva(int nfigures, const double *nu, const double *y, long n, double *H,
                            double *L) {
  VoigtTables t;
  t.init(nfigures);
  for (long i = 0; i < n; i++) voigt(nu[i], y[i], &H[i], &L[i], t);
  return ME_OK;
}

extern "C" int meo_svd(double *a, int n, double *w, double *v) {
  if (n < 1 || n > 16) return ME_ERR_ARG;
  return gr_svd(a, n, n, w, v);
}

extern "C" int meo_svbksb(const double *u, const double *v, const double *w, const double *b,
                          int n, double *x) {
  if (n < 1 || n > 16) return ME_ERR_ARG;
  gr_backsub(u, v, w, b, n, x);
  return ME_OK;
}

extern "C" int meo_init_guess(meo_plan *P, const double *prof, double *guess, double *extra) {
  PixelState st;
  int r = init_guess(*P, prof, st);
  if (r == 0) {
    memcpy(guess, st.guess, sizeof(st.guess));
    extra[0] = st.norm0;
    extra[1] = st.normp;
    extra[2] = st.lim7[0];
    extra[3] = st.lim7[1];
    extra[4] = st.step[7];
  }
  return r;
}

extern "C" int meo_normal_equations(meo_plan *P, const double *prof, const double *par,
                                    double step7, double norm0, double *H, double *g,
                                    double *chisq) {
  LmState L;
  memset(&L, 0, sizeof(L));
  L.npar = P->npar;
  PixelCtx C;
  C.P = P;
  C.prof = prof;
  C.lm = &L;
  C.jac = &P->jac;
  C.ivn = &P->ivnoise;
  memcpy(C.st.step, P->step, sizeof(C.st.step));
  C.st.step[7] = step7;
  C.st.norm0 = norm0;
  const double inv_n0 = 1. / norm0;
  for (int s = 0; s < 4; s++)
    for (int iw = 0; iw < P->nw; iw++) P->ivnoise[s * P->nw + iw] = P->w2[s] * inv_n0;
  std::vector<double> syn(4 * P->nw);
  synthesize(*P, par, true, C.st.step, syn.data(), P->jac.data());
  normal_equations(C, syn.data(), H, g);
  *chisq = loss(C, syn.data());
  return ME_OK;
}

thread_local FlopTally g_tally;

namespace {
void tally_out(double *c) {
  c[0] = (double)g_tally.add;
  c[1] = (double)g_tally.mul;
  c[2] = (double)g_tally.div;
  c[3] = (double)g_tally.sqrt_;
  c[4] = (double)g_tally.exp_;
  c[5] = (double)g_tally.trig;
  c[6] = (double)g_tally.special;
  c[7] = (double)g_tally.cmp;
}
}  // namespace

// Operation counts of one synthesis (all nl wavelengths) of the reference's
// algorithm at `par`: counts[8] = add/sub, mul, div, sqrt, exp/log,
// sin/cos, erfc, compares.
extern "C" int meo_count_synth(meo_plan *P, const double *par, int deriv, double *counts) {
  if (!P || !par || !counts) return ME_ERR_ARG;
  std::vector<Cnt> syn(4 * P->nw), jac(deriv ? 36 * P->nw : 0);
  double step[9];
  memcpy(step, P->step, sizeof(step));
  g_tally = FlopTally();
  synthesize<Cnt>(*P, par, deriv != 0, step, syn.data(), deriv ? jac.data() : nullptr);
  tally_out(counts);
  return ME_OK;
}

// Operation counts of one SVD_solve_mem (Golub-Reinsch SVD + truncation
// ladder + back-substitutions) on the n x n matrix a with right-hand side g.
extern "C" int meo_count_svd_solve(const double *a, const double *g, int n, double thr,
                                   double *counts) {
  if (!a || !g || !counts || n < 1 || n > 16) return ME_ERR_ARG;
  std::vector<Cnt> A(a, a + n * n), V(n * n), W(n), G(g, g + n), X(n);
  g_tally = FlopTally();
  gr_svd<Cnt>(A.data(), n, n, W.data(), V.data());
  Cnt wmax = W[0];
  for (int i = 1; i < n; i++) wmax = wmax > W[i] ? wmax : W[i];
  Cnt t = thr;
  while (true) {
    Cnt wthr = wmax * t;
    for (int i = 0; i < n; i++)
      if (W[i] < wthr) W[i] = 0.;
    gr_backsub<Cnt>(A.data(), V.data(), W.data(), G.data(), n, X.data());
    bool inside = true;
    for (int i = 0; i < n; i++)
      if (X[i] > 0.5 || X[i] < -0.5) inside = false;
    if (inside || t > 2e-3) break;
    t *= 5.;
  }
  tally_out(counts);
  return ME_OK;
}

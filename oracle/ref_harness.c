/* Test-infrastructure harness around the reference's own C inversion core.
 *
 * This file is part of the oracle (test infrastructure only).  It is compiled
 * together with the UNMODIFIED reference sources (Src/ME_SOLVER.c, Src/LM_FIT.c,
 * Src/FADDEEVA.c, Src/SVD.c, Src/INV_INIT.c, Src/RINPUT.c, Src/RANDOM_NUMBER.c,
 * Src/LOG_ERROR.c, Src/STR.c, Src/ALLOCATION.c) by oracle/Makefile into
 * oracle/_ref/libmeref.so.  Nothing of the reference is copied here: the
 * harness only fills the reference's own structures the way Src/ME_INV.c:64-134
 * does for a single-process run and then calls the reference's entry points.
 *
 * Entry points (all return 0 on success):
 *   meref_setup     RDINPUT (Src/RINPUT.c:361) + INIT_INV (Src/INV_INIT.c:86)
 *                   with a caller-supplied wavelength grid, then replaces the
 *                   time-seeded RNG state (Src/RANDOM_NUMBER.c:44) by a fixed seed.
 *   meref_invert    INVERSION_MULTI (Src/LM_FIT.c:746) over a caller buffer.
 *   meref_synth     Milne_Eddington_Single (Src/ME_SOLVER.c:101).
 *   meref_faddeeva  Faddeeva (Src/FADDEEVA.c:440) for a given Nfigures.
 *   meref_svd       svdcmp_double (Src/SVD_TEMPLATE.h:84).
 *   meref_svbksb    svbksb_double (Src/SVD_TEMPLATE.h:348).
 *   meref_init_guess Init_Guess (Src/ME_SOLVER.c:445).
 *   meref_bounds    bounds_check (Src/ME_SOLVER.c:370).
 *   meref_rng_gauss RNG_GAUSS (Src/RANDOM_NUMBER.c:137) from the fixed seed.
 *   meref_get/set_lm_chisq  the LM->chisq value carried between pixels.
 *   meref_reseed    the RNG state of meref_setup for another seed, carried
 *                   LM->chisq zeroed (a fresh map in the same process).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "RINPUT.h"
#include "INV_INIT.h"
#include "LM_FIT.h"
#include "ME_SOLVER.h"
#include "FADDEEVA.h"
#include "SVD.h"
#include "RANDOM_NUMBER.h"

static STRUCT_INPUT g_input;
static STRUCT_STK g_stk;
static STRUCT_LM g_lm;
static STRUCT_PARA g_para;
static STRUCT_SUBSET g_subset;
static STRUCT_MPI g_mpi;
static int g_ready = 0;
static long g_nbuf = 0;

/* Reads the control file with the reference's parser, sets up the inversion
 * for `nl` wavelengths and a batch of at most `npix_max` pixels, and seeds the
 * reference's Park-Miller/Bays-Durham RNG with `seed` (idum = -seed, iy = 0,
 * iset = true: the state RNG_INIT leaves behind, Src/RANDOM_NUMBER.c:55-57).
 * RDINPUT appends to ./log_00000 (Src/RINPUT.c:381-384); `logdir` (may be
 * NULL) is the directory that file is created in. */
int meref_setup(const char *ctl_path, const double *lambda, int nl,
                long npix_max, int seed, const char *logdir) {
  char cwd[4096];
  if (!ctl_path || !lambda || nl < 8 || npix_max < 1) return -1;
  if (g_ready) return -2; /* one setup per process: INIT_INV has no teardown here */
  memset(&g_input, 0, sizeof(g_input));
  memset(&g_stk, 0, sizeof(g_stk));
  memset(&g_lm, 0, sizeof(g_lm));
  memset(&g_para, 0, sizeof(g_para));
  memset(&g_subset, 0, sizeof(g_subset));
  memset(&g_mpi, 0, sizeof(g_mpi));
  g_mpi.rank = 0;
  g_mpi.size = 1;

  if (!getcwd(cwd, sizeof(cwd))) return -3;
  if (logdir && chdir(logdir) != 0) return -4;
  RDINPUT(ctl_path, &g_input, &g_mpi);
  LOG_FINALIZE();
  if (logdir && chdir(cwd) != 0) return -5;

  g_stk.nw = nl;
  g_stk.Lambda = (double *)malloc(sizeof(double) * nl);
  memcpy(g_stk.Lambda, lambda, sizeof(double) * nl);

  /* The pixel box is one row of npix_max pixels, read in one chunk. */
  g_input.nx = (int)npix_max;
  g_input.ny = 1;
  g_input.sol_box[0][0] = 0;
  g_input.sol_box[0][1] = (int)npix_max - 1;
  g_input.sol_box[1][0] = 0;
  g_input.sol_box[1][1] = 0;
  g_input.nProf = (int)npix_max;
  g_input.cache_prof = false;

  INIT_INV(&g_input, &g_stk, &g_lm, &g_para, &g_mpi, &g_subset);
  g_nbuf = npix_max;

  g_lm.RNG.idum = -(int32_t)(seed & 0x7FFFFFFF);
  g_lm.RNG.iy = 0;
  g_lm.RNG.iset = true;
  g_ready = 1;
  return 0;
}

int meref_invert(const double *prof, long npix, double *res, double *fit) {
  if (!g_ready) return -1;
  if (npix < 1 || npix > g_nbuf) return -2;
  const long n = 4L * g_stk.nw;
  memcpy(g_input.profbuff, prof, sizeof(double) * n * npix);
  g_subset.nProf = (int)npix;
  INVERSION_MULTI(&g_input, &g_stk, &g_para, &g_lm, &g_subset);
  memcpy(res, g_input.resbuff, sizeof(double) * 10 * npix);
  if (fit) {
    if (!g_input.output_fit) return -3;
    memcpy(fit, g_input.fitbuff, sizeof(double) * n * npix);
  }
  return 0;
}

/* Per-wavelength grid facts INIT_INV derived (Src/INV_INIT.c:144-177) and the
 * limits after its v_los clip: ints[0..4] = ncut, ic, i0, i1, npar;
 * limits[18] = Para->Limits. */
int meref_plan_facts(int *ints, double *limits) {
  if (!g_ready) return -1;
  ints[0] = g_stk.ncut;
  ints[1] = g_stk.ic;
  ints[2] = g_stk.i0;
  ints[3] = g_stk.i1;
  ints[4] = g_para.npar;
  for (int i = 0; i < 9; i++) {
    limits[2 * i] = g_para.Limits[i][0];
    limits[2 * i + 1] = g_para.Limits[i][1];
  }
  return 0;
}

/* Puts the RNG back in the state meref_setup leaves for `seed` and zeroes the
 * LM chi^2 carried from pixel to pixel, so that a process set up once can
 * invert a map afresh with another restart stream. */
int meref_reseed(int seed) {
  if (!g_ready) return -1;
  g_lm.RNG.idum = -(int32_t)(seed & 0x7FFFFFFF);
  g_lm.RNG.iy = 0;
  g_lm.RNG.iset = true;
  g_lm.chisq = 0;
  return 0;
}

#ifdef ME_WITH_SHIM
/* The same buffers and structures through the GPU adapter that replaces
 * INVERSION_MULTI (milne-eddington_b200/shim/me_inversion_multi.c), for the
 * test that runs both on one set-up.  Built into _ref/libmeshim.so only. */
#include "me_inversion_multi.h"

int meref_invert_shim(const double *prof, long npix, double *res, double *fit,
                      int precision) {
  if (!g_ready) return -1;
  if (npix < 1 || npix > g_nbuf) return -2;
  const long n = 4L * g_stk.nw;
  memcpy(g_input.profbuff, prof, sizeof(double) * n * npix);
  g_subset.nProf = (int)npix;
  me_inversion_multi_set_precision(precision);
  const int st = me_inversion_multi(&g_input, &g_stk, &g_para, &g_lm, &g_subset);
  if (st != 0) return st;
  memcpy(res, g_input.resbuff, sizeof(double) * 10 * npix);
  if (fit) {
    if (!g_input.output_fit) return -3;
    memcpy(fit, g_input.fitbuff, sizeof(double) * n * npix);
  }
  return 0;
}

/* me_config of the parsed control file, as the adapter builds it. */
int meref_shim_config(me_config *cfg) {
  if (!g_ready) return -1;
  return me_inversion_multi_config(&g_input, &g_stk, &g_para, &g_lm, cfg);
}
#endif

double meref_get_lm_chisq(void) { return g_lm.chisq; }
void meref_set_lm_chisq(double v) { g_lm.chisq = v; }

/* Milne_Eddington_Single with the set-up line, steps and Faddeeva state.
 * step7 overrides Para->step[7] (Init_Guess sets it to 0.1*Imax per pixel). */
int meref_synth(const double *par, int deriv, double step7, double *syn,
                double *jac) {
  if (!g_ready) return -1;
  double p[9];
  memcpy(p, par, sizeof(p));
  double saved = g_para.step[7];
  g_para.step[7] = step7;
  Milne_Eddington_Single(p, &g_stk, &g_para, deriv ? true : false);
  g_para.step[7] = saved;
  const int nw = g_stk.nw;
  memcpy(syn, g_stk.syn, sizeof(double) * 4 * nw);
  if (deriv && jac) memcpy(jac, g_stk.Jacobian, sizeof(double) * 36 * nw);
  return 0;
}

int meref_faddeeva(int nfigures, const double *nu, const double *y, long n,
                   double *H, double *L) {
  STRUCT_FADDEEVA f;
  memset(&f, 0, sizeof(f));
  f.nfigures = nfigures;
  Faddeeva_init(&f);
  for (long i = 0; i < n; i++) Faddeeva(nu[i], y[i], &H[i], &L[i], &f);
  free(f.Expa2n2);
  return 0;
}

/* a[n*n] row-major in, U out (in place); w[n]; v[n*n]. */
int meref_svd(double *a, int n, double *w, double *v) {
  STRUCT_MATRIX am = MATRIX(0, n - 1, 0, n - 1, enum_dbl, false);
  STRUCT_MATRIX vm = MATRIX(0, n - 1, 0, n - 1, enum_dbl, false);
  memcpy(am.data, a, sizeof(double) * n * n);
  svdcmp_double(&am, w, &vm);
  memcpy(a, am.data, sizeof(double) * n * n);
  memcpy(v, vm.data, sizeof(double) * n * n);
  FREE_MATRIX(am);
  FREE_MATRIX(vm);
  return 0;
}

int meref_svbksb(const double *u, const double *v, const double *w,
                 const double *b, int n, double *x) {
  STRUCT_MATRIX am = MATRIX(0, n - 1, 0, n - 1, enum_dbl, false);
  STRUCT_MATRIX vm = MATRIX(0, n - 1, 0, n - 1, enum_dbl, false);
  memcpy(am.data, u, sizeof(double) * n * n);
  memcpy(vm.data, v, sizeof(double) * n * n);
  svbksb_double(&am, &vm, w, b, x);
  FREE_MATRIX(am);
  FREE_MATRIX(vm);
  return 0;
}

/* Init_Guess on one profile.  out9 = Par_Guess after bounds_check;
 * extra[0..4] = norm0, normp, Limits[7][0], Limits[7][1], step[7];
 * returns Init_Guess's status (1 = below Icriteria). */
int meref_init_guess(const double *prof, double *out9, double *extra) {
  if (!g_ready) return -1;
  double *save_prof = g_stk.prof;
  double saved_l70 = g_para.Limits[7][0], saved_l71 = g_para.Limits[7][1];
  double saved_s7 = g_para.step[7];
  g_stk.prof = (double *)prof;
  int st = Init_Guess(&g_stk, &g_para);
  if (st == 0) {
    memcpy(out9, g_para.Par_Guess, sizeof(double) * 9);
    extra[0] = g_stk.norm0;
    extra[1] = g_stk.normp;
    extra[2] = g_para.Limits[7][0];
    extra[3] = g_para.Limits[7][1];
    extra[4] = g_para.step[7];
  }
  g_stk.prof = save_prof;
  g_para.Limits[7][0] = saved_l70;
  g_para.Limits[7][1] = saved_l71;
  g_para.step[7] = saved_s7;
  return st;
}

int meref_bounds(double *par9, const double *limits7) {
  if (!g_ready) return -1;
  double s0 = g_para.Limits[7][0], s1 = g_para.Limits[7][1];
  if (limits7) {
    g_para.Limits[7][0] = limits7[0];
    g_para.Limits[7][1] = limits7[1];
  }
  bounds_check(par9, &g_para);
  g_para.Limits[7][0] = s0;
  g_para.Limits[7][1] = s1;
  return 0;
}

/* n Gaussian deviates from a fresh NR stream seeded with `seed`. */
int meref_rng_gauss(int seed, long n, double *out) {
  STRUCT_RNGState st;
  memset(&st, 0, sizeof(st));
  st.idum = -(int32_t)(seed & 0x7FFFFFFF);
  st.iy = 0;
  st.iset = true;
  for (long i = 0; i < n; i++) out[i] = RNG_GAUSS(&st);
  return 0;
}

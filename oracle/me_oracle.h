/* me_oracle.h -- CPU restatement of the reference's per-pixel ME inversion.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle the CUDA path is checked
 * against; only tests/, __graft_entry__.smoke() and bench.py's CPU legs may
 * load it.  It is never part of the product path.
 *
 * The restatement keeps the reference's floating-point evaluation order, so on
 * the same CPU/libm it reproduces the reference bit for bit (the reference's LM
 * is sensitive to the last bit of its inputs, so anything less would not pin
 * it).  Each function cites the reference file:line it follows.
 */
#ifndef ME_ORACLE_H
#define ME_ORACLE_H

#include "../include/me_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* draws of the random restarts (irun >= 4, Src/LM_FIT.c:185-196) */
#define MEO_RNG_COUNTER 0  /* per-(pixel, run) Philox4x32-10 draws, as the CUDA path */
#define MEO_RNG_NR 1       /* one sequential NR ran1 + polar Box-Muller stream, as the reference */

typedef struct meo_plan meo_plan;

int meo_plan_create(const me_config *cfg, const double *lambda, int nl, meo_plan **out);
/* Instrument filter (an extension; the reference has none): observed
 * wavelength i becomes sum_k weights[k] * synthesis(lambda_i + offsets_mA[k] / 1e3),
 * for the profiles and the Jacobian; k = 1 removes it.  The `filter` keyword
 * sets the Gaussian table (offsets uniform over +-1.5 FWHM). */
int meo_plan_set_filter(meo_plan *p, const double *offsets_mA, const double *weights, int k);
void meo_plan_destroy(meo_plan *p);
int meo_plan_facts(const meo_plan *p, me_plan_facts *out);

/* INVERSION_MULTI over npix pixels.  pixel_offset = global index of prof[0]
 * (keys the counter RNG); rng_mode MEO_RNG_*; nr_seed seeds the NR stream
 * (state kept in the plan across calls once seeded, reseeded when nr_seed
 * changes); carry_chisq in/out = LM->chisq between pixels; counters may be
 * NULL, else [npix][8] = runs, iterations, trials, accepted, syntheses,
 * jacobians, max trial index in any iteration, final irun. */
int meo_invert(meo_plan *p, const double *prof, long npix, long pixel_offset,
               double *res, double *fit, int rng_mode, int nr_seed,
               double *carry_chisq, long long *counters);

int meo_synth(meo_plan *p, const double *par, int deriv, double step7, double *syn,
              double *jac);
int meo_faddeeva(int nfigures, const double *nu, const double *y, long n, double *H,
                 double *L);
int meo_svd(double *a, int n, double *w, double *v);
int meo_svbksb(const double *u, const double *v, const double *w, const double *b,
               int n, double *x);
/* returns Init_Guess's status; guess[9]; extra[5] as me_init_guess */
int meo_init_guess(meo_plan *p, const double *prof, double *guess, double *extra);
/* normal equations at `par` for one pixel: H[npar*npar], g[npar], chisq
 * (Hessian_Compute + Loss_Function with Noise_Init's weights from norm0) */
int meo_normal_equations(meo_plan *p, const double *prof, const double *par,
                         double step7, double norm0, double *H, double *g,
                         double *chisq);
/* Algorithmic operation counts (a counting scalar type through the same
 * templated code): counts[8] = add/sub, mul, div, sqrt, exp/log, sin/cos,
 * erfc, compares for one synthesis at par (all nl wavelengths) and for one
 * SVD solve (SVD + truncation ladder) of a with right-hand side g. */
int meo_count_synth(meo_plan *p, const double *par, int deriv, double *counts);
int meo_count_svd_solve(const double *a, const double *g, int n, double thr, double *counts);
/* the project's counter-based standard normal draws: out[8] for (pixel, run) */
void meo_restart_draws(unsigned long long seed, long long pixel, int run, double *out);

#ifdef __cplusplus
}
#endif

#endif

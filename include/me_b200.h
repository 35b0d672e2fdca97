/* me_b200.h -- C ABI of the B200 Milne-Eddington Stokes inversion library.
 *
 * Drop-in replacement for the per-pixel inversion of the reference
 * (HaoLi-70/Milne-Eddington).  Every entry point names the reference function it
 * replaces.  Conventions:
 *   - status 0 = OK, negative = error (see me_strerror); nothing aborts;
 *   - the caller owns host buffers, a plan owns its device memory and stream;
 *   - one plan per host thread (a plan is not thread-safe);
 *   - parameter order and units are the reference's Par[0..8]
 *     (Src/ME_SOLVER.c:121-122): B [G], theta_B [rad], phi_B [rad], v_los [km/s],
 *     Doppler width [mA], damping a, eta0, S0+S1, beta = S0/(S0+S1);
 *   - profiles are pixel-major [pixel][I,Q,U,V][lambda] doubles and results
 *     [pixel][10] doubles (9 parameters then chi^2, zeros for skipped pixels),
 *     exactly the reference's profbuff/resbuff layout (Src/LM_FIT.c:767-808).
 */
#ifndef ME_B200_H
#define ME_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ME_MAX_LINES 20   /* Src/RINPUT.h:15 NUM_LINES */
#define ME_PATH_LEN 512   /* Src/STR.h:15 Max_Line_Length */
#define ME_MAX_NL 512     /* largest wavelength grid a plan accepts */
#define ME_MAX_FILTER 63  /* most sub-wavelengths of an instrument filter */

/* status codes */
#define ME_OK 0
#define ME_ERR_ARG -1        /* bad argument (null pointer, size out of range) */
#define ME_ERR_CONFIG -2     /* control file missing keyword / malformed value */
#define ME_ERR_IO -3         /* file could not be opened / read / written */
#define ME_ERR_CUDA -4       /* CUDA runtime error */
#define ME_ERR_NODEVICE -5   /* no CUDA device: the library has no CPU fallback */
#define ME_ERR_TIMEOUT -6    /* device work exceeded its iteration budget */
#define ME_ERR_NOMEM -7      /* allocation failed */
#define ME_ERR_FORMAT -8     /* unsupported file format (FITS) */

/* precision of the synthesis / Jacobian / normal equations on the device.
 * The 9x9 SVD solve and the chi^2 accept test are FP64 in both modes. */
#define ME_PREC_FP32 0
#define ME_PREC_FP64 1

/* Parsed control file.  Field meanings and defaults are the reference's
 * keyword table (Src/RINPUT.c:400-458) after Get_Keys' unit handling
 * (Src/RINPUT.c:48-357): Bounds_Btheta / Bounds_Bphi and the theta/phi
 * regularisation targets are stored in radians (x pi). */
typedef struct me_config {
  int nline;                          /* `lines` repeats; only line 0 is used (Src/ME_SOLVER.c:131) */
  double line_lambda0[ME_MAX_LINES];  /* [A] */
  double line_geff[ME_MAX_LINES];
  int verbose;                        /* verbose            (default 1)    */
  int num_iter;                       /* num_iter           (60)           */
  int num_run;                        /* num_run            (4)            */
  double convg_criteria;              /* convg_criteria     (1e-3)         */
  double chisq_criteria;              /* chisq_criteria     (1.0)          */
  char data_path[ME_PATH_LEN];        /* data_path          (required)     */
  char wavelength_path[ME_PATH_LEN];  /* wavelength_path    (required)     */
  double weights[4];                  /* weights            (1,1,1,1)      */
  int sol_box[4];                     /* sol_box x0,x1,y0,y1 (-1,-1,-1,-1) */
  int output_fit;                     /* output_fit         (NO)           */
  char cache_path[ME_PATH_LEN];       /* cache_path         (./cache)      */
  char result_path[ME_PATH_LEN];      /* result_path        (./res.fits)   */
  char fit_path[ME_PATH_LEN];         /* fit_path           (./fit.fits)   */
  double damp;                        /* damp               (1e-3)         */
  double lambda_accept;               /* lambda_accept      (5.0)          */
  double lambda_reject;               /* lambda_reject      (5.0)          */
  double lambda_limits[2];            /* lambda_limits      (1e-5, 1e3)    */
  double bounds[9][2];                /* Bounds_*           (see table)    */
  int fixed[9];                       /* *_fixed            (NO)           */
  int regul[9];                       /* *_Regularization   (theta: YES)   */
  double regul_value[9];
  double regul_weight[9];
  int regul_any;                      /* any regul[] set (Input->Regul)    */
  double vcoeffi;                     /* VCoeffi            (100)          */
  double lcoeffi;                     /* LCoeffi            (250)          */
  double icriteria;                   /* Icriteria          (100)          */
  double svd_threshold;               /* SVDthreshold       (1e-6)         */
  int hmi_ref;                        /* HMI_REF            (No)           */
  int cache_prof;                     /* Cache_prof         (No)           */
  int nthreads;                       /* Nthreads           (4, unused)    */
  int nfigures;                       /* Nfigures           (6)            */
  double step[9];                     /* Step    (1000,2,2,2,20,0.3,30,1e5,0.3) */
  int nprofiles;                      /* nprofiles          (20)           */
  int cache_inv;                      /* Cache_inv          (No)           */
  /* --- keywords of this library (not in the reference) --- */
  int precision;                      /* precision = FP32 | FP64 (FP32)    */
  unsigned long long rng_seed;        /* rng_seed (0): key of the per-(pixel, run) draws */
  int lines_seen;                     /* bookkeeping: `lines` present      */
  int data_path_seen, wavelength_path_seen;
  /* filter = FWHM [mA], points (0 = none): each observed wavelength is the
   * Gaussian-weighted mean of the synthesis over `points` offsets spanning
   * +-1.5 FWHM (an instrument filter; not in the reference) */
  double filter_fwhm;
  int filter_points;
} me_config;

/* Facts INIT_INV derives from the grid (Src/INV_INIT.c:121-177). */
typedef struct me_plan_facts {
  int nl, ncut, ic, i0, i1, npar;
  double bshift;           /* 4.6686e-10 * g * lambda0^2 [mA/G] */
  double limits[9][2];     /* after INIT_INV's v_los clip       */
  double fadd_a;           /* Alg-916 spacing a for Nfigures    */
} me_plan_facts;

/* Counters of one me_invert_batch call (device-side event counts). */
typedef struct me_stats {
  long long pixels;        /* pixels in the batch                          */
  long long valid;         /* pixels inverted (not skipped by the I gate)  */
  long long runs;          /* LM_FIT runs (restarts included)              */
  long long iterations;    /* LM iterations                                */
  long long trials;        /* trial steps = SVD solves                     */
  long long accepted;      /* accepted trials                              */
  long long syntheses;     /* forward syntheses (trials)                   */
  long long jacobians;     /* syntheses with Jacobian + normal equations   */
  long long wavelengths;   /* wavelength points synthesised (both kinds)   */
  long long redo_pixels;   /* pixels re-run to honour the carried LM chi^2 */
  long long launches;      /* inversion kernel launches made by the call     */
  long long rounds;        /* LM rounds (one trial step per pixel in flight) */
  double kernel_ms;        /* device time of the inversion kernel(s)       */
  double h2d_ms, d2h_ms;   /* host<->device copy time (host entry point)   */
  double init_ms;          /* device time of the learned initialiser        */
  long long learned_done;  /* pixels that ended after the learned start     */
  /* with me_plan_set_profiling(plan, 1): device time per kernel (CUDA events
   * around every launch) and the trial steps / syntheses with Jacobian that
   * the tail kernel did; zeros otherwise */
  double jac_ms, svd_ms, trial_ms, tail_ms;
  long long tail_trials, tail_jacobians;
} me_stats;

typedef struct me_plan me_plan;

const char *me_version(void);
const char *me_strerror(int status);
/* Message of the last failure on the calling thread ("" if none). */
const char *me_last_error(void);

/* Defaults of every keyword.  Replaces the default table of RDINPUT
 * (Src/RINPUT.c:400-458). */
int me_config_init(me_config *cfg);

/* Reads a control file (`key = value`, comments `#`/`!`/`*`, inline `!`) with
 * the reference's keyword semantics.  Replaces RDINPUT + Get_Keys
 * (Src/RINPUT.c:361-563, 48-357).  Unlike the reference it does not check that
 * data_path / wavelength_path exist (the FITS entry points do), and reports
 * malformed values as ME_ERR_CONFIG instead of exiting.  `errbuf` (may be
 * NULL) receives a one-line message. */
int me_config_parse(const char *ctl_path, me_config *cfg, char *errbuf, size_t errlen);
int me_config_parse_text(const char *text, me_config *cfg, char *errbuf, size_t errlen);

/* Builds a plan for one wavelength grid on CUDA device `device`: line
 * constants, ncut/ic/i0/i1, v_los clip, Faddeeva constants, device buffers.
 * Replaces INIT_INV (Src/INV_INIT.c:86-289).  Returns ME_ERR_NODEVICE when no
 * GPU is visible (there is no CPU path). */
int me_plan_create(const me_config *cfg, const double *lambda, int nl, int device,
                   me_plan **out);
void me_plan_destroy(me_plan *plan);
int me_plan_get_facts(const me_plan *plan, me_plan_facts *out);

/* The reference carries LM->chisq (the chi^2 of the last trial step) from one
 * pixel to the next inside a process and uses it in the first regularisation
 * ratio test of the next pixel (Src/LM_FIT.c:555-559).  A plan carries it the
 * same way across pixels and batches; it starts at 0 (STRUCT_LM LM = {0},
 * Src/ME_INV.c:91).  These read / reset it. */
double me_plan_get_carry_chisq(const me_plan *plan);
void me_plan_set_carry_chisq(me_plan *plan, double chisq);

/* Instrument filter (no reference counterpart): each observed wavelength
 * lambda_i becomes sum_q weights[q] * synthesis(lambda_i + offsets_mA[q] / 1e3)
 * for the profiles and the Jacobian, everywhere the plan synthesises (the
 * inversion, me_synthesize*, the fit profiles, initialiser training).  k = 1
 * removes it; k <= ME_MAX_FILTER.  The control keyword `filter = FWHM, points`
 * sets a Gaussian table at plan creation.  me_invert_batch_device_noalloc does
 * not take filtered control files. */
int me_plan_set_filter(me_plan *plan, const double *offsets_mA, const double *weights, int k);

/* Persistent-grid size (CTAs) of the inversion kernel; set_grid overrides the
 * occupancy-derived default (used by the autotuner and the benchmarks). */
int me_plan_grid(const me_plan *plan);
void me_plan_set_grid(me_plan *plan, int grid);

/* Number of pixels a plan keeps in flight on the device (0 = default,
 * 131072); each holds ~1.6 KB of LM state in HBM. */
int me_plan_window(const me_plan *plan);
void me_plan_set_window(me_plan *plan, int window);

/* Pixels in flight at or below which, once every pixel of a batch has been
 * taken from the queue, the remaining ones are run to the end one warp per
 * pixel (their synthesis spread over the lanes) instead of one LM step per
 * launch round: the same arithmetic up to the compiler's contraction of
 * multiply-adds, and a much shorter tail.  -1 (default): half a wave of the
 * tail kernel's warps on this device (~900 on a B200); 0: rounds only. */
int me_plan_tail_slots(const me_plan *plan);
/* Once every pixel of a batch has been taken from the queue, the LM rounds
 * give each pixel still in flight a group of lanes (2, 4, ... up to this
 * power of two, enough to fill about one wave of the Jacobian kernel) that
 * splits its synthesis and SVD; 1 keeps one thread per pixel.  Default 32.
 * Results agree with one thread per pixel to rounding. */
int me_plan_max_group(const me_plan *plan);
void me_plan_set_max_group(me_plan *plan, int lanes);
/* Lanes per 9x9 SVD in the LM rounds that still feed from the queue (1, 2, 4
 * or 8); more lanes cut the decomposition's latency, fewer keep more of them
 * in flight.  Default 1. */
int me_plan_svd_lanes(const me_plan *plan);
/* With all nine parameters free, the SVD solves can keep their 9x9 matrix in
 * registers, one thread per pixel: 0 (default) = shared memory everywhere;
 * 1 = registers in the one-thread-per-pixel rounds; 2 = registers also in the
 * lane-split rounds after the queue drains (in place of the lanes' shared
 * SVD).  Same operations in the same order (results agree to rounding: the
 * compiler fuses multiply-adds differently); the register form has no
 * shared-memory round trips, the shared-memory form a smaller code.  Which is
 * faster depends on the batch (me_plan_autotune tries them). */
int me_plan_svd_registers(const me_plan *plan);
void me_plan_set_svd_registers(me_plan *plan, int mode);
/* The LM rounds between two checks of the queue go to the GPU as one CUDA
 * graph, captured once per batch for each lane-group size (default on; off:
 * one launch per kernel).  Profiling (me_plan_set_profiling) launches
 * directly. */
void me_plan_set_graphs(me_plan *plan, int on);
/* The SVD solves of trials after a rejection run on a second stream beside
 * the Jacobian kernel of the same round (they concern other pixels; default
 * on).  Profiling launches serially. */
void me_plan_set_overlap(me_plan *plan, int on);

/* With a learned start (an initialiser attached), the queue takes the pixels
 * in descending order of the misfit of their start -- the chi^2 of the run -1
 * parameters on about 16 of the grid's wavelengths, in quarter-octave
 * buckets, ties in pixel order -- so that the pixels likely to need many
 * iterations and restarts start early instead of running on alone at the end
 * of the batch.  0 restores pixel order.  Default on.  A pixel's steps are the
 * same in any order; which kernel runs each of them depends on when it is
 * queued, so results agree with pixel order to rounding.  The time of the
 * misfit and the sort is part of the stats' init_ms. */
void me_plan_set_queue_order(me_plan *plan, int on);

/* The stable counting sort behind the queue order, for testing: order [n]
 * receives the indices of keys [n] (each < 128) by ascending key, equal keys
 * in index order; host buffers, run on CUDA device `device`. */
int me_order_by_key(int device, const unsigned char *keys, long n, long long *order);
void me_plan_set_svd_lanes(me_plan *plan, int lanes);
/* Records CUDA events around every inversion launch and reports per-kernel
 * device time in me_stats (off by default; costs a little host time). */
void me_plan_set_profiling(me_plan *plan, int on);
void me_plan_set_tail_slots(me_plan *plan, int slots);
/* The rounds after the queue drains: each pixel in flight gets the most lanes
 * (a power of two, at most max_group) for which pixels x lanes stay within
 * group_fill (1..8) half waves of the Jacobian kernel -- more lanes cut each
 * round's latency, fewer keep each round's work compact -- and the host checks
 * the pixels in flight every poll_rounds rounds (even, 2..64), which is how
 * often the lanes adapt and when the tail kernel can take over.  Defaults 4
 * (two waves) and 4. */
void me_plan_set_drain(me_plan *plan, int group_fill, int poll_rounds);
void me_plan_get_drain(const me_plan *plan, int *group_fill, int *poll_rounds);

/* The host's checks of the queue during the plan's last batch, one record per
 * check: host time since the batch's rounds began (ms; the check waits for
 * the rounds launched before it, so this is when they ended), LM rounds so
 * far, queue position, pixels in flight and lanes per pixel of the rounds
 * before it (1 = one thread per pixel; 0 marks the tail kernel's launch,
 * -1 the end of the batch's first pass).  Writes at most cap records to out
 * (may be NULL) and returns how many the batch made. */
typedef struct me_poll_record {
  double ms;
  long long rounds, next;
  int busy, group;
} me_poll_record;
int me_plan_poll_trace(const me_plan *plan, me_poll_record *out, int cap);

/* Per-pixel counters of the plan's last batch: [npix][4] = LM runs,
 * iterations (syntheses with Jacobian), trial steps, accepted steps; zeros
 * for skipped pixels.  npix at most the last batch's. */
int me_plan_last_counters(const me_plan *plan, unsigned int *counters, long npix);

/* Variant of the one-thread-per-pixel Jacobian and trial kernels (default
 * 0): 0 = 128 pixels per CTA, the wavelength
 * grid read through the L1 cache, the FP32 Faddeeva (Alg-916) series terms
 * 1 / (a^2 n^2 + y^2) from a per-synthesis table in shared memory; 1 = 64 and 2 = 256 pixels per CTA; 3 = the grid
 * staged in shared memory per CTA; 4 = no table, each term's correctly
 * rounded reciprocal computed where it is used; 5 = the Jacobian kernel's
 * normal-equation sums in shared memory, 3 CTAs of 128 per SM (FP32 plans;
 * FP64 plans run 0).  All run the same arithmetic; each variant is compiled
 * on its own, so results agree to rounding. */
int me_plan_kernel_variant(const me_plan *plan);
void me_plan_set_kernel_variant(me_plan *plan, int variant);

/* How an FP32 plan's syntheses evaluate the Faddeeva function w(z) (Voigt and
 * Faraday-Voigt profiles): 0 = the reference's |z| regions with their rational
 * approximations and Alg-916 (Faddeeva, Src/FADDEEVA.c:440-590) in FP32;
 * 1 (default) = Weideman's 16-term rational series (SIAM J. Numer. Anal. 31,
 * 1994), one formula for every z with Im z >= 0, within 6e-7 of w in FP32, with
 * no branch -- a different method at least as accurate as mode 0 in FP32, so
 * results agree with mode 0 to that accuracy, not bit for bit.  FP64 plans
 * always use 0, the reference's method. */
int me_plan_faddeeva(const me_plan *plan);
void me_plan_set_faddeeva(me_plan *plan, int mode);
/* How an FP32 plan's 9x9 SVD solves form the Givens rotations of their QR
 * sweeps: 1 (default) = the radius z = sqrt(a^2 + b^2) and its reciprocal from
 * one reciprocal square root (each within two ulps of the correctly rounded
 * values; a third of the dependent latency of a square root and a division);
 * 0 = the reference's pythag and division (SVD_TEMPLATE.h).  The SVD and the
 * chi^2 stay FP64; results agree with mode 0 to rounding.  FP64 plans always
 * use 0, so they stay bit-exact with the reference's arithmetic. */
int me_plan_givens(const me_plan *plan);
void me_plan_set_givens(me_plan *plan, int mode);
/* 1: the one-thread-per-pixel Jacobian and trial kernels read each pixel's
 * observed profile from a slot-major copy made when the pixel enters a slot
 * (4 nl doubles per slot in flight), so that a warp's reads are coalesced;
 * 0 (default): from the pixel's rows of the map.  Same values, same results.
 * The copy pays when pixels take many trials (the plain LM: 7 % faster per
 * batch) and costs a little when most end after a learned start. */
void me_plan_set_slot_profiles(me_plan *plan, int on);
/* The coefficients c_0..c_15 and the scale L of that series, for checking. */
void me_weideman16(float *coef, float *L);
/* w(nu + i a) by that series in FP32 on the device: H = Re w, L = Im w. */
int me_faddeeva_weideman(const double *nu, const double *a, long n, double *H, double *L,
                         int device);

/* Autotuner: times me_invert_batch_device on the caller's batch (device
 * profiles d_prof [npix][4][nl], ideally of the size and kind the plan will
 * invert) for candidate values of the plan's runtime knobs -- pixels in
 * flight (window), lanes per pixel after the queue drains (max_group), the
 * tail kernel's threshold (tail_slots), lanes per SVD (svd_lanes), the
 * kernel variant (pixels per CTA, grid staging, Faddeeva series reciprocals;
 * me_plan_set_kernel_variant), where the SVD keeps its matrix
 * (me_plan_set_svd_registers), the lanes and check interval after the
 * queue drains (me_plan_set_drain), the FP32 Faddeeva evaluation
 * (me_plan_set_faddeeva) and the slot-major profile copy
 * (me_plan_set_slot_profiles) -- one knob at a time, keeping each
 * improvement, and leaves the best setting on the plan.  The carried LM chi^2 is restored afterwards.  out (may be NULL)
 * receives the choice, its time and the number of timed runs. */
typedef struct me_tune_result {
  int window, max_group, tail_slots, svd_lanes;
  double ms;    /* device time of the batch with the chosen setting */
  int trials;   /* batches timed */
  int kernel_variant, svd_registers;  /* me_plan_set_kernel_variant / _svd_registers */
  int group_fill, drain_poll;         /* me_plan_set_drain */
  int faddeeva;                       /* me_plan_set_faddeeva */
  int slot_profiles;                  /* me_plan_set_slot_profiles */
} me_tune_result;
int me_plan_autotune(me_plan *plan, const double *d_prof, long npix, void *stream,
                     me_tune_result *out);

/* Inverts npix pixels.  prof: host [npix][4][nl]; res: host [npix][10];
 * fit: host [npix][4][nl] or NULL (best-fit profiles, zeros when skipped);
 * stats may be NULL.  Replaces INVERSION_MULTI (Src/LM_FIT.c:746-811). */
int me_invert_batch(me_plan *plan, const double *prof, long npix, double *res,
                    double *fit, me_stats *stats);

/* With `prof` in page-locked host memory (cudaHostAlloc / cudaHostRegister)
 * and at least 131072 pixels, me_invert_batch copies the map in chunks of about
 * an eighth and starts inverting the first chunk while the others are on
 * their way; with a learned start each chunk's guesses and queue order
 * (sorted within the chunk) are made as it lands, and once the last chunk
 * has landed the part of the queue not yet taken is re-sorted into the global
 * order.  Results agree with the whole-map copy to rounding (the order in
 * which pixels meet the kernels changes).  1 (default): on; 2: on, without
 * the global re-sort; 0: copy the map whole first. */
void me_plan_set_feed(me_plan *plan, int mode);

/* Same on device buffers (d_prof, d_res, d_fit device pointers; d_fit may be
 * NULL); work is ordered on `stream` (a cudaStream_t, NULL = the plan's). */
int me_invert_batch_device(me_plan *plan, const double *d_prof, long npix,
                           double *d_res, double *d_fit, void *stream,
                           me_stats *stats);

/* Forward Stokes synthesis for npix parameter vectors par [npix][9] into
 * prof [npix][4][nl] (host buffers).  Replaces Milne_Eddington_Single with
 * Deriv=false (Src/ME_SOLVER.c:101-366). */
int me_synthesize(me_plan *plan, const double *par, long npix, double *prof);

/* Forward synthesis on device buffers d_par [npix][9] -> d_prof [npix][4][nl],
 * ordered on `stream` (NULL = the plan's stream, waited for). */
int me_synthesize_device(me_plan *plan, const double *d_par, long npix, double *d_prof,
                         void *stream);

/* Synthesis with the step-scaled analytic Jacobian (Deriv=true).  jac is
 * [npix][4][9][nl] (the reference's Stk->Jacobian layout, Src/ME_SOLVER.c:169-177);
 * step7 is the S step (Init_Guess sets 0.1*I_max per pixel). */
int me_synthesize_jacobian(me_plan *plan, const double *par, long npix, double step7,
                           double *prof, double *jac);

/* Voigt H and Faraday-Voigt L for n (nu, a) pairs at accuracy Nfigures, on
 * the device, in the given precision (ME_PREC_*).  Replaces Faddeeva
 * (Src/FADDEEVA.c:440-590). */
int me_faddeeva(int nfigures, int precision, const double *nu, const double *a, long n,
                double *H, double *L, int device);

/* Golub-Reinsch SVD of nmat n x n matrices (n <= 9) in FP64 on the device:
 * a = u * diag(w) * v^T.  Replaces svdcmp_double (Src/SVD_TEMPLATE.h:84-344). */
int me_svd(const double *a, long nmat, int n, double *u, double *w, double *v, int device);

/* The same decomposition as the inversion's trial-step solve runs it: U and w
 * only (the operations on V left out; SVD_solve_mem, Src/LM_FIT.c:400-469,
 * through svdcmp_double, Src/SVD_TEMPLATE.h:84-344), with `lanes` lanes per
 * matrix (1, 2, 4, 8, 16 or 32: one thread, the lane-split rounds, the tail
 * kernel) and the Givens rotations' radius from the reference's pythag and a
 * division (fast = 0, FP64 plans) or from one reciprocal square root
 * (fast = 1, FP32 plans).  u and w as me_svd's.  Returns the number of
 * matrices whose QR sweeps hit the 50-sweep limit in *limit_hits (may be
 * NULL). */
int me_svd_u(const double *a, long nmat, int n, int lanes, int fast, double *u, double *w,
             int *limit_hits, int device);

/* Device-buffer variants (work ordered on `stream`, a cudaStream_t; NULL =
 * the default stream, waited for before returning). */
int me_svd_device(const double *d_a, long nmat, int n, double *d_u, double *d_w, double *d_v,
                  void *stream);
int me_svd_u_device(const double *d_a, long nmat, int n, int lanes, int fast, double *d_u,
                    double *d_w, void *stream);
int me_synthesize_jacobian_device(me_plan *plan, const double *d_par, long npix, double step7,
                                  double *d_prof, double *d_jac, void *stream);

/* me_invert_batch_device without any device allocation.  No counterpart in
 * the reference: an addition of this library, for callers that cannot
 * allocate device memory while they invert -- data-reduction pipelines and
 * frameworks that reserve the GPU's memory for their own pool when they start
 * (an allocation of ours would fail or take memory their pool counts on), and
 * real-time loops at the instrument, where cudaMalloc / cudaFree can
 * synchronise the device and stall the loop.  It takes the control file and
 * the wavelength grid (host arrays) instead of a plan and runs the same round
 * kernels as me_invert_batch_device.
 *
 * All of its scratch lives in one static device array of fixed size (about
 * 12.4 MB, held on every GPU the library is loaded on until the process
 * exits): at most ME_NOALLOC_MAX_PIXELS pixels per call, ME_NOALLOC_SLOTS of
 * them in flight; a larger npix is rejected with ME_ERR_ARG -- invert large
 * maps in chunks, passing *carry_chisq (the LM chi^2 carried from pixel to
 * pixel, 0 at the start of a map) from one call to the next.  Control files
 * with an instrument filter are rejected (ME_ERR_CONFIG).  d_prof
 * [npix][4][nl] and d_res [npix][10] are device buffers of the caller; the
 * work is ordered on `stream` (a cudaStream_t, NULL = legacy default stream)
 * and complete when the call returns.  Rounds beyond the LM step bound end
 * the call with ME_ERR_TIMEOUT.
 *
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) and the kernels' occupancy with that device current;
 * make that first call before any stream capture.  Every call on a device
 * shares the one array, which keeps the previous call's contents (the call
 * clears what must start at zero): calls that overlap on the GPU -- from two
 * host threads or two streams at once -- race and must be serialised by the
 * caller. */
#define ME_NOALLOC_MAX_PIXELS 65536
#define ME_NOALLOC_SLOTS 8192
int me_invert_batch_device_noalloc(const me_config *cfg, const double *lambda, int nl,
                                   const double *d_prof, long npix, double *d_res,
                                   double *carry_chisq, void *stream);

/* Initial guess for npix profiles: guess [npix][9]; extra [npix][5] =
 * norm0, normp, S lower limit, S upper limit, S step; status [npix] (0 ok,
 * 1 below Icriteria).  Replaces Init_Guess (Src/ME_SOLVER.c:445-676). */
int me_init_guess(me_plan *plan, const double *prof, long npix, double *guess,
                  double *extra, int *status);

/* ---------------------------------------------------------------------------
 * Learned initialiser (no reference counterpart).
 *
 * A multilayer perceptron, 4 nl features (I / I_max - 1, 10 Q / I_max,
 * 10 U / I_max, 10 V / I_max, standardised) -> 256 -> 256 -> 256 GELU -> 10
 * outputs (B, cos theta, sin 2 phi, cos 2 phi, v, Doppler width, damping,
 * eta0, beta, S / I_max), on BF16 tensor-core GEMMs with FP32 accumulation,
 * trained with Adam on profiles that the plan's FP32 forward model synthesises
 * on the device from seeded parameter draws plus Gaussian noise.
 *
 * With an initialiser attached to a plan, every pixel first gets one LM run
 * (LM_FIT, Src/LM_FIT.c:531-660) from the network's guess; a pixel whose run
 * meets chisq_criteria ends there, the others go on with the reference's run
 * schedule (INVERSION, Src/LM_FIT.c:701-733) from Init_Guess, and the best
 * run is kept.  Without one (the default) the plan is the reference's
 * algorithm.
 * ------------------------------------------------------------------------- */
typedef struct me_mlp me_mlp;

/* Training set and optimiser.  Parameters are drawn uniformly in each range
 * (cos theta uniform, v normal with sigma v_sigma, S fixed), synthesised on
 * the plan's grid and line, and given noise of standard deviation `noise`
 * (in units of the continuum). */
typedef struct me_mlp_train_params {
  long long samples;            /* training profiles (>= batch)           */
  int epochs;                   /* passes over them                        */
  int batch;                    /* rows per Adam step (multiple of 256)    */
  double lr;                    /* Adam step size                          */
  unsigned long long seed;      /* key of the parameter and noise draws    */
  double b_range[2];            /* field strength [G]                      */
  double cos_theta_range[2];    /* cosine of the inclination               */
  double phi_range[2];          /* azimuth [rad]                           */
  double v_sigma;               /* line-of-sight velocity sigma [km/s]     */
  double doppler_range[2];      /* Doppler width [mA]                      */
  double damping_range[2];      /* damping                                 */
  double eta_range[2];          /* line-to-continuum absorption eta0       */
  double s;                     /* source function S0 (continuum units)    */
  double beta_range[2];         /* source function gradient ratio          */
  double noise;                 /* Gaussian noise sigma                    */
  int gemm;                     /* GEMM kernel, ME_GEMM_TCGEN05 (default)  */
                                /* or ME_GEMM_MMA_SYNC (defined below)     */
  /* an optional second population: with probability mix_weight a sample
   * draws B and eta0 from these ranges instead of b_range / eta_range
   * (0, the default: one population) */
  double mix_weight;
  double mix_b_range[2];
  double mix_eta_range[2];
} me_mlp_train_params;

/* The defaults: the parameter distributions of the Fe I 15648.5 A maps
 * (B ~ U(0, 3000) G, cos theta ~ U(-1, 1), phi ~ U(0, pi), v ~ N(0, 1.5) km/s,
 * Doppler width ~ U(150, 350) mA, a ~ U(0.1, 0.8), eta0 ~ U(2, 30), S0 = 1,
 * beta ~ U(0.1, 0.6), noise 1e-3, one population); 2^22 samples, 16 epochs,
 * batch 4096, lr 1e-3, tcgen05 GEMMs. */
int me_mlp_train_params_default(me_mlp_train_params *tp);

/* Trains a new initialiser for the plan's line and grid on the plan's device.
 * final_loss (may be NULL) receives the mean squared error of the standardised
 * outputs over the last epoch. */
int me_mlp_train(me_plan *plan, const me_mlp_train_params *tp, me_mlp **out,
                 double *final_loss);
void me_mlp_destroy(me_mlp *mlp);

/* Binary file of the weights and the standardisation; load places the model
 * on CUDA device `device`. */
int me_mlp_save(const me_mlp *mlp, const char *path);
int me_mlp_load(const char *path, int device, me_mlp **out);

/* Network guess par [npix][9] (the reference's units) for profiles prof
 * [npix][4][nl]: host buffers, or device buffers ordered on `stream`. */
int me_mlp_predict(me_mlp *mlp, const double *prof, long npix, double *par);
int me_mlp_predict_device(me_mlp *mlp, const double *d_prof, long npix, double *d_par,
                          void *stream);

/* Attaches an initialiser to a plan (NULL detaches).  The plan does not own
 * it; its grid size must match the plan's. */
int me_plan_set_initializer(me_plan *plan, me_mlp *mlp);

/* Layer sizes and parameters, for checking the training arithmetic.  nl: the
 * grid size; nin_pad: input width (4 nl rounded up to 32, zero weights past
 * 4 nl); the output layer has 32 rows of which the first 10 are used.
 * Parameters are flattened layer by layer as W [dout][din] then b [dout] (FP32
 * master copies). */
int me_mlp_shape(const me_mlp *mlp, int *nl, int *nin_pad, long long *nparams);
int me_mlp_get_params(const me_mlp *mlp, float *params);
int me_mlp_set_params(me_mlp *mlp, const float *params);

/* Loss and gradient of one batch: x [rows][nin_pad] standardised features,
 * t [rows][10] standardised targets (host FP32; rows a multiple of 256).
 * loss = mean over rows and the 10 outputs of (y - t)^2; grad has the layout
 * of the parameters.  No optimiser step is taken. */
int me_mlp_loss_grad(me_mlp *mlp, const float *x, const float *t, int rows, double *loss,
                     float *grad);

/* The initialiser's GEMM kernel.  ME_GEMM_TCGEN05 (the default): TMA loads
 * of 128-byte-swizzled BF16 tiles, tcgen05.mma with the FP32 accumulator in
 * tensor memory, tcgen05.ld epilogue.  ME_GEMM_MMA_SYNC: warp-level
 * mma.sync m16n8k16, kept for comparison.  Shapes the tcgen05 kernel does
 * not take (N % 16 != 0, a split-K share not a multiple of 64) run on the
 * mma.sync kernel whatever is set. */
#define ME_GEMM_TCGEN05 0
#define ME_GEMM_MMA_SYNC 1
int me_mlp_set_gemm(me_mlp *mlp, int path);
/* GEMM launches of each kernel since the initialiser was made. */
int me_mlp_gemm_launches(const me_mlp *mlp, long long *tcgen05, long long *mma_sync);

/* One GEMM of the initialiser's kernels, for testing them: with A [m][r] and
 * Bt [n][r] row-major BF16 bit patterns (host), z [m][n] = A Bt^T + bias
 * (bias [n] or NULL) and y [m][n] = GELU(z) if gelu else z, FP32 host
 * buffers (z may be NULL).  split > 1 divides the reduction over that many
 * CTAs that add into y with atomics (bias NULL, gelu 0, z NULL).  r % 32 ==
 * 0 and r % (32 split) == 0.  Runs on CUDA device `device`; *ran (may be
 * NULL) receives the kernel that ran. */
int me_gemm_bf16(int device, int path, const uint16_t *a, const uint16_t *bt, int m, int n,
                 int r, int split, const float *bias, int gelu, float *z, float *y, int *ran);

/* ---------------------------------------------------------------------------
 * FITS primary-HDU I/O, the subset of cfitsio the reference's driver uses
 * (Src/IO.c:120-742): dimensions and BITPIX, reads of doubles from an element
 * offset with BSCALE / BZERO applied (fits_read_pix with TDOUBLE), creation of
 * a zero-filled BITPIX -64 image (fits_create_img), writes of doubles at an
 * element offset (fits_write_pix).  Element offsets count in the FITS order
 * (NAXIS1 fastest).  CPU only.
 * ------------------------------------------------------------------------- */
int me_fits_image_info(const char *path, int *bitpix, int *naxis, long naxes[8]);
int me_fits_read(const char *path, long first, long n, double *out);
int me_fits_create(const char *path, int naxis, const long *naxes);
int me_fits_write(const char *path, long first, long n, const double *v);

/* ---------------------------------------------------------------------------
 * The driver: the reference's MEINV program around INVERSION_MULTI
 * (Src/ME_INV.c:64-295 with rWavelength, rProfile, rProfilesll, PixelMV,
 * CACHE_INIT, WRITE_RESULT of Src/IO.c and INIT_INV's chunking,
 * Src/INV_INIT.c:207-250).  It reads data_path / wavelength_path, inverts the
 * pixels of sol_box in chunks of nprofiles (all at once with Cache_prof),
 * writes result_path [10][nx'][ny'] and, with output_fit, fit_path
 * [nw][4][nx'][ny'], and with Cache_inv keeps the reference's checkpoint file
 * (cache_path) and skips the chunks it marks done.  Consecutive chunks are
 * inverted together (batch_pixels per GPU call); several GPUs take batches in
 * turn (batch b on device b mod N) in place of the MPI farm.
 * ------------------------------------------------------------------------- */
typedef struct me_run_options {
  int ndevices;            /* plans, one per entry of devices (default 1)           */
  const int *devices;      /* CUDA device of each plan (NULL: 0, 1, ...)            */
  long batch_pixels;       /* pixels per GPU call, in whole chunks (131072)         */
  int max_group;           /* me_plan_set_max_group for every plan (-1: default)    */
  int tail_slots;          /* me_plan_set_tail_slots for every plan (-2: default)   */
  long stop_after_chunks;  /* stop once this many chunks are done (0: run to the
                              end); an interrupted run, for checkpoint tests        */
  me_mlp *initializer;     /* learned initialiser for every plan (NULL: none)       */
} me_run_options;

typedef struct me_run_report {
  long nx, ny, nw;         /* data cube                                      */
  long counts;             /* pixels of sol_box                              */
  long chunk_pixels;       /* nProf                                          */
  long nchunks;            /* chunks of sol_box                              */
  long chunks_done;        /* chunks inverted by this run                    */
  long chunks_skipped;     /* chunks the checkpoint file marked done         */
  long pixels_inverted;    /* pixels inverted by this run                    */
  double seconds;          /* wall time of the run                           */
} me_run_report;

int me_run_options_default(me_run_options *opt);
/* opt and report may be NULL. */
int me_run(const char *ctl_path, const me_run_options *opt, me_run_report *report);
int me_run_config(const me_config *cfg, const me_run_options *opt, me_run_report *report);

#ifdef __cplusplus
}
#endif

#endif /* ME_B200_H */

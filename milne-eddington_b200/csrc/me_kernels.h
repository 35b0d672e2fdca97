// me_kernels.h -- launch interface between the host plan (me_api.cu) and the
// CUDA kernels (me_invert.cuh, me_units.cu).
#pragma once

#include <cuda_runtime.h>

#include "../../include/me_b200.h"
#include "me_device.cuh"

namespace me {

constexpr int kBlock = 128;
// minimum resident CTAs per SM jac_kernel is compiled for (its register cap)
#ifndef ME_JAC_MINB
#define ME_JAC_MINB 2
#endif
constexpr int kSvdBlock = 64;  // threads of svd_kernel; each holds its matrix in shared memory
// Variants of the one-thread-per-slot Jacobian and trial kernels, chosen per
// plan (DevPlan::kvar, me_plan_set_kernel_variant, the autotuner):
//   0  128 pixels per CTA, grid through the L1 cache, FP32 reciprocal table
//   1   64 pixels per CTA     2  256 pixels per CTA
//   3  the wavelength grid staged in shared memory (up to kMaxStage points)
//   4  no reciprocal table: each Alg-916 series term's correctly rounded
//      reciprocal computed in place (the table holds the same values)
//   5  the Jacobian kernel's normal-equation sums in shared memory, 3 CTAs
//      of 128 per SM (the trial kernel as 0; FP32 synthesis only, FP64 plans
//      run variant 0)
// All give the same arithmetic.
constexpr int kKernelVariants = 6;
constexpr int kMaxStage = 1024;
constexpr int kSvdSmem = (81 + 18) * kSvdBlock * 8;
// learned initialiser inference: rows per chunk, kernel launches per chunk
constexpr int kMlpPredChunk = 65536;
constexpr int kMlpPredLaunches = 6;
// error status of the initialiser's tensor-core GEMMs since the last call
// (a bounded wait that expired); synchronises the device (me_mlp.cu)
int mlp_gemm_status(me_mlp *m);

// Life cycle of an inversion slot (one pixel in flight).
enum SlotStateCode : int {
  SL_EMPTY = 0,      // waiting for a pixel from the queue
  SL_JAC_START = 1,  // first synthesis of an LM run (LM_FIT set-up)
  SL_JAC_NEXT = 2,   // synthesis at newly accepted parameters (next iteration)
  SL_TRIAL = 3,      // normal equations ready: trial steps
  SL_RUN_END = 4,    // run ended without a trial step (num_iter <= 0)
  SL_DONE = 5,       // queue exhausted
  SL_WAIT = 6,       // holds a queue position whose pixel has not arrived yet
                     // (S.pix = the position; InvertArgs::avail)
};

// Per-slot scalars, stored [SC_COUNT][W].
enum SlotScalar : int {
  SC_CHISQ = 0,    // the LM's current chi^2 (Chisq in LM_FIT)
  SC_LMCHISQ,      // LM->chisq: chi^2 of the last trial step, carried
  SC_RATIO,        // LM->ratio (regularisation scaling)
  SC_DAMP,         // LM->Damp
  SC_BEST,         // Para->Chisq_Best
  SC_NORMP,        // Stk->normp
  SC_ISN,          // 1 / sqrt(Stk->norm0)
  SC_STEP7,        // Para->step[7] of this pixel
  SC_L70, SC_L71,  // Para->Limits[7] of this pixel
  SC_COUNT
};

// Device state of the in-flight pixels, structure of arrays over W slots so
// that consecutive threads touch consecutive addresses.
struct Slots {
  int W;
  long long *pix;            // [W]
  int *state, *run, *it;     // [W]
  unsigned int *cnt;         // [4][W] runs, iterations, trials, accepted
  unsigned char *had_trial;  // [W]
  double *sc;                // [SC_COUNT][W]
  double *guess, *par, *pbest, *jvec;  // [9][W]
  double *hess;              // [81][W]: normal matrix, then the SVD's U factor
  double *ptmp;              // [9][W]: trial parameters of this round
  int *tk;                   // [W]: index of the trial step within the LM iteration (1 = first)
  int *jlist;                // [2][W] slots needing a synthesis with Jacobian
  int *jcount;               // [2]
  int *rlist;                // [2][W] slots going on to another trial after a rejected one
  int *rcount;               // [2]
  int *busy;                 // slots holding a pixel
  // [4 nl][W]: the observed profile of each slot's pixel, slot-major, copied
  // at refill so that the one-thread-per-slot kernels read it coalesced
  // (null: they read the pixel's rows of the input map)
  double *obs;
};

// An upper bound on the LM steps (syntheses with Jacobian + trial steps) of
// one pixel: every run ends after num_iter accepted steps, each preceded by
// at most the trials that take the damping from damp past lambda_limits[1]
// (lambda_reject >= 1.5 and finite limits are checked on the host).
__host__ __device__ inline long long slot_step_cap(const DevPlan &P) {
  double tpi = ceil(log(P.lam_lim[1] / P.damp) / log(P.lam_reject)) + 2.0;
  if (!(tpi >= 2.0)) tpi = 2.0;
  if (tpi > 1e4) tpi = 1e4;
  const double runs = 4.0 * P.nruns + 1.0;
  return (long long)(runs * (P.niter * (tpi + 1.0) + 2.0) + 16.0);
}

// One batch (all device pointers).
struct InvertArgs {
  const double *prof;          // [npix][4][nl]
  double *res;                 // [npix][10]
  double *fit;                 // [npix][4][nl] or null
  double *fitpar;              // [npix][9] best parameters before the post-folds (with fit)
  unsigned char *flags;        // [npix] bit0 inverted, bit1 made a trial step
  double *penalty0;            // [npix] regularisation penalty at the first guess
  double *lastchi;             // [npix] chi^2 of the pixel's last trial step
  unsigned int *counters;      // [npix][4] runs, iterations, trials, accepted
  unsigned long long *totals;  // [8] valid, runs, iterations, trials, accepted, jacobians,
                               // svd limit hits, pixels done after a learned start
  unsigned long long *next;    // queue position (zeroed before the batch)
  const long long *list;       // pixel indices to process (null = 0..count-1)
  long long count;             // number of queue items
  const double *stale;         // [npix] carried LM chi^2 per pixel (null = carry/first_pixel)
  double carry;                // carried LM chi^2 for pixel first_pixel
  long long first_pixel;
  const double *init_par;      // [npix][9] learned starting parameters (an extra first
                               // run, run -1), or null for the reference's schedule
  // queue positions below *avail can be taken (their profiles, and with a
  // learned start their guesses and order, are on the device); the host
  // raises it while it copies the map in.  null: the whole queue is there.
  const unsigned long long *avail;
};

// Plan constants from a control file and a wavelength grid (me_api.cu);
// returns an ME_* status, P.lambda / P.dlambda left null.
int build_devplan(const struct me_config *cfg, const double *lambda, int nl, DevPlan &P);

// Records `msg` as the calling thread's me_last_error(); returns `code`.
int record_error(int code, const char *msg);

// CTAs for a full device: which = 0 jac_kernel, 1 trial_kernel, 2 svd_kernel,
// 3 finish_kernel
int round_grid(int precision, int which, int device);
// The tail kernel: runs every slot still in flight to completion, one warp
// per slot (slots taken through *cursor, zeroed by the caller).  Only when the
// queue is exhausted (it does not refill).
cudaError_t launch_finish(int precision, const DevPlan &P, const InvertArgs &A, const Slots &S,
                          int *cursor, int grid, cudaStream_t st);
// One round: jac_kernel, svd (first trials), svd (later trials),
// trial_kernel.  grids: jac, trial, svd CTAs.  ev (nullable): 5 events
// recorded before, between and after the four launches (per-kernel device
// time when profiling).  svd_lanes: lanes per matrix of the SVD launches
// (1: svd_kernel; 2, 4, 8: svd_grp_kernel).
// Overlap (nullable): the later-trial SVD launch runs on ov->aux, forked from
// st before the Jacobian kernel and joined before the trial kernel (the two
// lists hold disjoint slots).
struct Overlap {
  cudaStream_t aux;
  cudaEvent_t fork, join;
};
cudaError_t launch_round(int precision, const DevPlan &P, const InvertArgs &A, const Slots &S,
                         int parity, const int grids[3], cudaStream_t st,
                         cudaEvent_t *ev = nullptr, int svd_lanes = 1,
                         const Overlap *ov = nullptr);
// A round with G lanes per slot (G = 2, 4, 8, 16, 32): for when the queue is
// empty and the slots in flight are too few to fill the device one thread
// each.  The trial kernel runs over the round's lists and does not refill.
cudaError_t launch_round_grp(int precision, int G, const DevPlan &P, const InvertArgs &A,
                             const Slots &S, int parity, const int grids[3], cudaStream_t st,
                             cudaEvent_t *ev = nullptr, const Overlap *ov = nullptr);
// Best-fit profiles after a batch: synthesis at fitpar for the inverted
// pixels (flags bit 0), zeros for the skipped ones.
cudaError_t launch_fit(int precision, const DevPlan &P, const double *d_fitpar,
                       const unsigned char *d_flags, long long npix, double *d_fit,
                       cudaStream_t st);
cudaError_t launch_synth(int precision, const DevPlan &P, const double *d_par, long long npix,
                         double step7, double *d_prof, double *d_jac, cudaStream_t st);
cudaError_t launch_voigt(int precision, const DevPlan &P, const double *d_nu, const double *d_a,
                         long long n, double *d_H, double *d_L, cudaStream_t st);
cudaError_t launch_svd(const double *d_a, long long nmat, int n, double *d_u, double *d_w,
                       double *d_v, int *d_hits, cudaStream_t st);
// The trial-step solve's U-only decomposition (no V) with `lanes` lanes per
// matrix (1, 2, 4, 8, 16, 32) and the Givens rotations' form (fast: from one
// reciprocal square root, as FP32 plans run it).
cudaError_t launch_svd_u(const double *d_a, long long nmat, int n, int lanes, int fast,
                         double *d_u, double *d_w, int *d_hits, cudaStream_t st);
cudaError_t launch_init_guess(const DevPlan &P, const double *d_prof, long long npix,
                              double *d_guess, double *d_extra, int *d_status, cudaStream_t st);
// Queue order of a learned start: pixels by descending misfit of their run -1
// parameters (kOrderBuckets quarter-octave buckets of chi^2, stable), into
// d_order [npix] as base + the index into d_prof.  d_key: npix bytes; d_hist:
// kOrderBuckets * kOrderBlocks ints.
constexpr int kOrderBuckets = 128;
constexpr int kOrderBlocks = 1024;
cudaError_t launch_start_order(int precision, const DevPlan &P, const double *d_prof,
                               const double *d_init, long long npix, unsigned char *d_key,
                               int *d_hist, long long *d_order, cudaStream_t st,
                               long long base = 0);
// queue positions [first, first + n) of d_list re-sorted by the per-pixel
// keys d_key (stable); d_tkey (n bytes), d_tval, d_perm (n each): scratch
cudaError_t launch_resort_tail(long long *d_list, long long first, long long n,
                               const unsigned char *d_key, unsigned char *d_tkey,
                               long long *d_tval, int *d_hist, long long *d_perm,
                               cudaStream_t st);
// the stable counting sort alone (keys < kOrderBuckets)
cudaError_t launch_order_by_key(const unsigned char *d_key, long long n, int *d_hist,
                                long long *d_order, cudaStream_t st, long long base = 0);

}  // namespace me

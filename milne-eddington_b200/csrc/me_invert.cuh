// me_invert.cuh -- the inversion hot path: one LM "round" is two kernels.
//
// Every pixel in flight owns a slot whose state lives in HBM (struct Slots).
// A round advances every slot by exactly one LM trial step:
//
//   jac_kernel    over the compacted list of slots that need the synthesis
//                 with Jacobian (a run start or an accepted step): the
//                 Milne-Eddington synthesis + analytic Jacobian fused with the
//                 weighted normal equations (Milne_Eddington_Single(Deriv) +
//                 Hessian_Compute + Get_Regul, Src/ME_SOLVER.c:101-366,
//                 Src/LM_FIT.c:240-396, 549-586);
//   trial_kernel  over all slots: one trial step (Trial_Synthesis,
//                 Src/LM_FIT.c:473-527: SVD solve, parameter update, forward
//                 synthesis, chi^2), the accept / reject / convergence logic
//                 (Src/LM_FIT.c:588-646), the end-of-run restart policy
//                 (INVERSION, Src/LM_FIT.c:701-733) and, when a pixel is done,
//                 its result and the refill of the slot from the queue.
//
// Slots that accept a step append themselves to the next round's Jacobian
// list, so that work runs at full SIMD width instead of in a divergent subset
// of a warp; finished pixels leave and new ones enter without a host round
// trip.  Instantiated per synthesis precision by me_invert_f32.cu / _f64.cu.
#pragma once

#include <cuda_runtime.h>

#include "me_device.cuh"
#include "me_kernels.h"

namespace me {
namespace detail {

// Synthesis with Jacobian fused with the weighted normal equations.
// sw[s] = weight_s / sqrt(norm0): sum (J sw)(J sw) = J^T W J with
// W = weight^2 / norm0 (Noise_Init, Src/ME_SOLVER.c:410-441).  H45 = upper
// triangle of the full 9x9 (row-major, i <= j), g9 = -J^T W r; returns
// sum (r sw)^2 / (4 nl) accumulated in FP64.  The observed value of Stokes s
// at wavelength iw is prof[(s nl + iw) pstr]: pstr 1 for a pixel's rows of the
// input map, W for a slot's column of the slot-major copy (Slots::obs).
template <class T, bool FILT>
__device__ __forceinline__ double deriv_pass(const DevPlan &P, VoigtK<T> &K, T *rden,
                                             const double *par, const double *step,
                                             const double *prof, const double sw[4], double *H45,
                                             double *g9, const T *sgrid = nullptr, int pstr = 1) {
  SynthCall<T> c;
  synth_setup<T>(c, par, P, step);
  c.grid = sgrid;
  voigt_prepare<T>(K, c.p5, rden, blockDim.x);
  T h[45], g[9];
#pragma unroll
  for (int i = 0; i < 45; i++) h[i] = T(0);
#pragma unroll
  for (int i = 0; i < 9; i++) g[i] = T(0);
  double chi = 0.0;
  const int nl = P.nl;
  const T tsw[4] = {T(sw[0]), T(sw[1]), T(sw[2]), T(sw[3])};
#pragma unroll 1
  for (int iw = 0; iw < nl; iw++) {
    T syn[4], J[4][9];
    channel_point<T, true, FILT>(c, P, K, tsw, iw, syn, J);
    T r[4];
#pragma unroll
    for (int s = 0; s < 4; s++) {
      const double rd = ((double)syn[s] - __ldg(prof + (size_t)(s * nl + iw) * pstr)) * sw[s];
      chi += rd * rd;
      r[s] = T(rd);
    }
    int idx = 0;
#pragma unroll
    for (int i = 0; i < 9; i++) {
#pragma unroll
      for (int j = i; j < 9; j++) {
        h[idx] += J[0][i] * J[0][j] + J[1][i] * J[1][j] + J[2][i] * J[2][j] + J[3][i] * J[3][j];
        idx++;
      }
      g[i] -= J[0][i] * r[0] + J[1][i] * r[1] + J[2][i] * r[2] + J[3][i] * r[3];
    }
  }
#pragma unroll
  for (int i = 0; i < 45; i++) H45[i] = (double)h[i];
#pragma unroll
  for (int i = 0; i < 9; i++) g9[i] = (double)g[i];
  return chi / (4.0 * nl);
}

// deriv_pass with the 45 + 9 sums of the normal equations in shared memory
// (acc[k * BLOCK], this thread's column) instead of registers: the same
// additions in the same order, fewer live registers across the wavelength
// loop (the kernel then fits more CTAs per SM).
template <class T, bool FILT, int BLOCK>
__device__ __forceinline__ double deriv_pass_sacc(const DevPlan &P, VoigtK<T> &K, T *rden,
                                                  const double *par, const double *step,
                                                  const double *prof, const double sw[4],
                                                  double *H45, double *g9, const T *sgrid,
                                                  T *acc, int pstr = 1) {
  SynthCall<T> c;
  synth_setup<T>(c, par, P, step);
  c.grid = sgrid;
  voigt_prepare<T>(K, c.p5, rden, blockDim.x);
#pragma unroll
  for (int i = 0; i < 54; i++) acc[i * BLOCK] = T(0);
  double chi = 0.0;
  const int nl = P.nl;
  const T tsw[4] = {T(sw[0]), T(sw[1]), T(sw[2]), T(sw[3])};
#pragma unroll 1
  for (int iw = 0; iw < nl; iw++) {
    T syn[4], J[4][9];
    channel_point<T, true, FILT>(c, P, K, tsw, iw, syn, J);
    T r[4];
#pragma unroll
    for (int s = 0; s < 4; s++) {
      const double rd = ((double)syn[s] - __ldg(prof + (size_t)(s * nl + iw) * pstr)) * sw[s];
      chi += rd * rd;
      r[s] = T(rd);
    }
    int idx = 0;
#pragma unroll
    for (int i = 0; i < 9; i++) {
#pragma unroll
      for (int j = i; j < 9; j++) {
        acc[idx * BLOCK] += J[0][i] * J[0][j] + J[1][i] * J[1][j] + J[2][i] * J[2][j] +
                            J[3][i] * J[3][j];
        idx++;
      }
      acc[(45 + i) * BLOCK] -= J[0][i] * r[0] + J[1][i] * r[1] + J[2][i] * r[2] + J[3][i] * r[3];
    }
  }
#pragma unroll
  for (int i = 0; i < 45; i++) H45[i] = (double)acc[i * BLOCK];
#pragma unroll
  for (int i = 0; i < 9; i++) g9[i] = (double)acc[(45 + i) * BLOCK];
  return chi / (4.0 * nl);
}

// Forward synthesis + chi^2 (Trial_Synthesis's synthesis and Loss_Function);
// residuals and their squares in FP64.  fit (nullable) receives the profile.
template <class T, bool FILT>
__device__ __forceinline__ double forward_pass(const DevPlan &P, VoigtK<T> &K, T *rden,
                                            const double *par, const double *step,
                                            const double *prof, const double sw[4],
                                            double *fit, const T *sgrid = nullptr, int pstr = 1) {
  SynthCall<T> c;
  synth_setup<T>(c, par, P, step);
  c.grid = sgrid;
  voigt_prepare<T>(K, c.p5, rden, blockDim.x);
  const T ones[4] = {T(1), T(1), T(1), T(1)};
  double chi = 0.0;
  const int nl = P.nl;
#pragma unroll 1
  for (int iw = 0; iw < nl; iw++) {
    T syn[4];
    channel_point<T, false, FILT>(c, P, K, ones, iw, syn, nullptr);
#pragma unroll
    for (int s = 0; s < 4; s++) {
      if (prof) {
        const double rd = ((double)syn[s] - __ldg(prof + (size_t)(s * nl + iw) * pstr)) * sw[s];
        chi += rd * rd;
      }
      if (fit) fit[s * nl + iw] = (double)syn[s];
    }
  }
  return chi / (4.0 * nl);
}

// Get_Regul's penalty (Src/LM_FIT.c:354-396).
__device__ __forceinline__ double penalty_of(const DevPlan &P, const double *par) {
  double pen = 0.0;
#pragma unroll
  for (int i = 0; i < 9; i++) {
    if (P.fixed[i] || !P.regul[i]) continue;
    const double r = par[i] - P.regul_value[i];
    pen += r * r * P.regul_weight[i];
  }
  return pen;
}

__device__ __forceinline__ void append_jac(const Slots &S, int parity_next, int s) {
  const int k = atomicAdd(S.jcount + parity_next, 1);
  S.jlist[parity_next * S.W + k] = s;
}
__device__ __forceinline__ void append_rej(const Slots &S, int parity_next, int s) {
  const int k = atomicAdd(S.rcount + parity_next, 1);
  S.rlist[parity_next * S.W + k] = s;
}

__device__ __forceinline__ void store9_px(double *a, long long pix, const double *v) {
#pragma unroll
  for (int i = 0; i < 9; i++) a[(size_t)pix * 9 + i] = v[i];
}
__device__ __forceinline__ void load9(const double *a, int W, int s, double *v) {
#pragma unroll
  for (int i = 0; i < 9; i++) v[i] = a[(size_t)i * W + s];
}
__device__ __forceinline__ void store9(double *a, int W, int s, const double *v) {
#pragma unroll
  for (int i = 0; i < 9; i++) a[(size_t)i * W + s] = v[i];
}

// Takes pixels from the queue until one is valid (INVERSION_MULTI's gate and
// Init_Guess, Src/LM_FIT.c:776-789) and sets the slot up for its first run.
// Skipped pixels get zeros.  Returns kRefilled, kExhausted when the queue is
// exhausted, or kWaiting when the queue position drawn is not on the device
// yet (A.avail): the slot then keeps the position (SL_WAIT, S.pix = the
// position) and calls again with it (held) in a later round.
enum RefillResult : int { kExhausted = 0, kRefilled = 1, kWaiting = 2 };

static __device__ int refill(const DevPlan &P, const InvertArgs &A, const Slots &S, int s,
                             unsigned long long &t_valid, long long held = -1) {
  const int nl = P.nl;
  const int W = S.W;
  while (true) {
    unsigned long long k;
    if (held >= 0) {
      k = (unsigned long long)held;
      held = -1;
    } else {
      k = atomicAdd(A.next, 1ULL);
      if (k >= (unsigned long long)A.count) return kExhausted;
    }
    if (A.avail && k >= *(volatile const unsigned long long *)A.avail) {
      S.pix[s] = (long long)k;
      S.state[s] = SL_WAIT;
      return kWaiting;
    }
    // with a feed (A.avail) the list and the guesses were written while this
    // kernel may run: read them past the L1 cache
    const long long pix = A.list ? (A.avail ? __ldcg(A.list + k) : A.list[k]) : (long long)k;
    const double *pp = A.prof + (size_t)pix * 4 * nl;
    PixelInit pin;
    const int bad = init_guess(pp, P, pin, true);
    if (bad || P.nruns <= 0) {
#pragma unroll
      for (int i = 0; i < 10; i++) A.res[(size_t)pix * 10 + i] = 0.0;
      if (A.fit)
        for (int i = 0; i < 4 * nl; i++) A.fit[(size_t)pix * 4 * nl + i] = 0.0;
      if (A.flags) A.flags[pix] = 0;
      continue;
    }
    t_valid++;
    S.pix[s] = pix;
    S.it[s] = 0;
    if (S.obs)
      for (int i = 0; i < 4 * nl; i++) S.obs[(size_t)i * W + s] = pp[i];
    store9(S.guess, W, s, pin.guess);
    if (A.init_par) {
      // learned start: the free parameters from the initialiser, folded into
      // the bounds; the fixed ones keep Init_Guess's values
      double q[9];
#pragma unroll
      for (int i = 0; i < 9; i++) {
        const double v = A.avail ? __ldcg(A.init_par + (size_t)pix * 9 + i)
                                 : A.init_par[(size_t)pix * 9 + i];
        q[i] = (P.fixed[i] || !isfinite(v)) ? pin.guess[i] : v;
      }
      bounds_fold(q, P, pin.l70, pin.l71);
      store9(S.par, W, s, q);
      S.run[s] = -1;
      if (A.penalty0) A.penalty0[pix] = P.regul_any ? penalty_of(P, q) : 0.0;
    } else {
      store9(S.par, W, s, pin.guess);
      S.run[s] = 0;
      if (A.penalty0) A.penalty0[pix] = P.regul_any ? penalty_of(P, pin.guess) : 0.0;
    }
    double *sc = S.sc;
    sc[SC_LMCHISQ * W + s] =
        A.stale ? A.stale[pix] : (pix == A.first_pixel ? A.carry : INFINITY);
    sc[SC_RATIO * W + s] = 1.0;
    sc[SC_BEST * W + s] = 0.0;
    sc[SC_NORMP * W + s] = pin.normp;
    sc[SC_ISN * W + s] = 1.0 / sqrt(pin.norm0);
    sc[SC_STEP7 * W + s] = pin.step7;
    sc[SC_L70 * W + s] = pin.l70;
    sc[SC_L71 * W + s] = pin.l71;
#pragma unroll
    for (int i = 0; i < 4; i++) S.cnt[i * W + s] = 0;
    S.had_trial[s] = 0;
    S.state[s] = SL_JAC_START;
    return kRefilled;
  }
}

// Counts a kernel accumulates per thread and adds to the batch totals once.
struct Tally {
  unsigned long long valid = 0, runs = 0, iter = 0, trials = 0, acc = 0, learned = 0, jac = 0,
                     svdlim = 0;
  int busy_delta = 0;
  __device__ void flush(const InvertArgs &A, const Slots &S) const {
    if (busy_delta) atomicAdd(S.busy, busy_delta);
    if (!A.totals) return;
    if (valid) atomicAdd(A.totals + 0, valid);
    if (runs) atomicAdd(A.totals + 1, runs);
    if (iter) atomicAdd(A.totals + 2, iter);
    if (trials) atomicAdd(A.totals + 3, trials);
    if (acc) atomicAdd(A.totals + 4, acc);
    if (jac) atomicAdd(A.totals + 5, jac);
    if (svdlim) atomicAdd(A.totals + 6, svdlim);
    if (learned) atomicAdd(A.totals + 7, learned);
  }
};

// The slot's per-pixel constants of a synthesis: step (with the pixel's S
// step) and the Stokes weights / sqrt(norm0).
__device__ __forceinline__ void slot_weights(const DevPlan &P, const Slots &S, int s,
                                             double step[9], double sw[4]) {
  const int W = S.W;
#pragma unroll
  for (int k = 0; k < 9; k++) step[k] = P.step[k];
  step[7] = S.sc[SC_STEP7 * W + s];
  const double isn = S.sc[SC_ISN * W + s];
#pragma unroll
  for (int k = 0; k < 4; k++) sw[k] = P.weights[k] * isn;
}

// After the synthesis with Jacobian at the slot's parameters: the LM_FIT
// set-up on a run start (Src/LM_FIT.c:549-566), the free-parameter block of the
// normal matrix with Get_Regul's diagonal and gradient terms
// (Hessian_Compute + Get_Regul, Src/LM_FIT.c:240-396), and the move to the
// first trial (or the run's end when num_iter <= 0).  One thread per slot.
// UNROLL: the loops below over all nine parameters with compile-time indices
// (the sums stay in registers: the FP32 kernels); otherwise over the free
// parameters through P.free_idx (the sums in local memory: the FP64 kernels,
// whose 54 double sums would not fit in registers beside the loop state).
template <bool UNROLL = false>
__device__ __forceinline__ void jac_store(const DevPlan &P, const Slots &S, int s,
                                          const double *par, double chi0, const double *H45,
                                          const double *g9) {
  const int W = S.W;
  const int n = P.npar;
  double ratio = S.sc[SC_RATIO * W + s];
  if (S.state[s] == SL_JAC_START) {
    S.sc[SC_CHISQ * W + s] = chi0;
    ratio = 1.0;
    if (P.regul_any) {
      const double pen = penalty_of(P, par);
      if (pen > 0.1 * S.sc[SC_LMCHISQ * W + s]) ratio = 0.1 * chi0 / pen;
    }
    S.sc[SC_RATIO * W + s] = ratio;
    S.it[s] = 0;
    if (P.niter <= 0) {
      S.state[s] = SL_RUN_END;
      return;
    }
  }
  if constexpr (!UNROLL) {
    double g[9];
    for (int a = 0; a < n; a++) {
      const int ia = P.free_idx[a];
      for (int b = a; b < n; b++) {
        const int ib = P.free_idx[b];
        double h = H45[ia * 9 - ia * (ia + 1) / 2 + ib];
        if (a == b && P.regul_any && P.regul[ia]) h += P.regul_weight[ia] * ratio;
        S.hess[(size_t)(a * n + b) * W + s] = h;
        S.hess[(size_t)(b * n + a) * W + s] = h;
      }
      g[a] = g9[ia];
      if (P.regul_any && P.regul[ia])
        g[a] -= (par[ia] - P.regul_value[ia]) * P.regul_weight[ia] * ratio;
    }
    for (int a = 0; a < n; a++) S.jvec[(size_t)a * W + s] = g[a];
    S.cnt[1 * W + s]++;
    S.sc[SC_DAMP * W + s] = P.damp;
    S.tk[s] = 1;
    S.state[s] = SL_TRIAL;
    return;
  }
  // all nine parameters with compile-time indices into H45 / g9, skipping
  // the fixed ones; a and b count the free parameters before ia and ib
  int a = 0;
#pragma unroll
  for (int ia = 0; ia < 9; ia++) {
    if (P.fixed[ia]) continue;
    int b = a;
#pragma unroll
    for (int ib = ia; ib < 9; ib++) {
      if (P.fixed[ib]) continue;
      double h = H45[ia * 9 - ia * (ia + 1) / 2 + ib];
      if (ib == ia && P.regul_any && P.regul[ia]) h += P.regul_weight[ia] * ratio;
      S.hess[(size_t)(a * n + b) * W + s] = h;
      S.hess[(size_t)(b * n + a) * W + s] = h;
      b++;
    }
    double gv = g9[ia];
    if (P.regul_any && P.regul[ia]) gv -= (par[ia] - P.regul_value[ia]) * P.regul_weight[ia] * ratio;
    S.jvec[(size_t)a * W + s] = gv;
    a++;
  }
  S.cnt[1 * W + s]++;
  S.sc[SC_DAMP * W + s] = P.damp;
  S.tk[s] = 1;
  S.state[s] = SL_TRIAL;
}

// The SVD solve of one trial step (SVD_solve_mem, Src/LM_FIT.c:400-469) and
// its trial parameters (Par_update + bounds_check, Src/LM_FIT.c:511-516).
//
// The reference decomposes, at the first trial of an LM iteration, the
// normal matrix H, and at every later trial the U factor the previous trial's
// SVD left in its place.  Two exact identities let this skip V:
//   * H is symmetric positive semi-definite, so its SVD has V = U and the
//     truncated solve V W+ U^T g equals U W+ U^T g;
//   * a U factor is orthogonal: its singular values are all 1 (nothing is
//     truncated at any rung of the threshold ladder) and V W^-1 U^T g is
//     U_prev^T g, clamped to +-0.5 as the ladder's last rung does.
// So trial 1 runs the U-only decomposition of H and the ladder; trial k >= 2
// uses the stored factor directly, and the decomposition that the reference
// ran at trial k-1 (whose U only trial k+1 needs) is run here at trial k >= 3,
// i.e. only when the iteration really goes on.
//
// G = 1: one thread, its matrix a column of shared memory (stride STR), w
// and rv1 likewise.  G > 1: a group of G lanes (`mask`), the matrix
// row-major in the group's shared memory, w and rv1 private to each lane (the
// decomposition is gr_svd_u_grp, the rest runs redundantly in every lane and
// lane 0 stores).  Returns the number of decompositions that hit the 50-sweep
// limit.
template <int STR, int G>
__device__ __forceinline__ int solve_slot(const DevPlan &P, const Slots &S, int s, double *a,
                                          double *w, double *rv1, int lane, unsigned mask) {
  constexpr bool WARP = G > 1;
  const int W = S.W;
  const int n = P.npar;
  int hits = 0;
  int tk = S.tk[s];
  if (WARP) tk = __shfl_sync(mask, tk, 0, G);
  double g[9], x[9];
  for (int k = 0; k < n; k++) g[k] = S.jvec[(size_t)k * W + s];
  for (int k = WARP ? lane : 0; k < n * n; k += G) a[k * STR] = S.hess[(size_t)k * W + s];
  if (WARP) __syncwarp(mask);
  auto decompose = [&]() {
    if constexpr (WARP)
      return P.fastg ? gr_svd_u_grp<G, true>(a, n, w, lane, mask)
                     : gr_svd_u_grp<G, false>(a, n, w, lane, mask);
    else
      return P.fastg ? gr_svd_u<STR, true>(a, n, w, rv1) : gr_svd_u<STR, false>(a, n, w, rv1);
  };
  if (tk == 1) {
    hits += decompose();
    double wmax = w[0];
    for (int i = 1; i < n; i++) wmax = fmax(wmax, w[i * (WARP ? 1 : STR)]);
    double thr = P.svd_thr;
    double ug[9];  // U^T g
    for (int j = 0; j < n; j++) {
      double acc = 0.0;
      for (int i = 0; i < n; i++) acc += a[(i * n + j) * STR] * g[i];
      ug[j] = acc;
    }
    while (true) {
      const double wthr = wmax * thr;
      double tj[9];
      for (int j = 0; j < n; j++) {
        double &wr = w[j * (WARP ? 1 : STR)];
        double wj = wr;
        if (wj < wthr) {
          wj = 0.0;
          wr = 0.0;
        }
        tj[j] = wj > 1e-50 ? ug[j] / wj : 0.0;
      }
      bool inside = true;
      for (int i = 0; i < n; i++) {
        double acc = 0.0;
        for (int j = 0; j < n; j++) acc += a[(i * n + j) * STR] * tj[j];
        x[i] = acc;
        if (acc > 0.5 || acc < -0.5) inside = false;
      }
      if (inside) break;
      if (thr > 2e-3) {
        for (int i = 0; i < n; i++) x[i] = x[i] > 0.5 ? 0.5 : (x[i] < -0.5 ? -0.5 : x[i]);
        break;
      }
      thr *= 5.;
    }
  } else {
    if (tk >= 3) hits += decompose();
    for (int j = 0; j < n; j++) {
      double acc = 0.0;
      for (int i = 0; i < n; i++) acc += a[(i * n + j) * STR] * g[i];
      x[j] = acc > 0.5 ? 0.5 : (acc < -0.5 ? -0.5 : acc);
    }
  }
  if (tk != 2)
    for (int k = WARP ? lane : 0; k < n * n; k += G) S.hess[(size_t)k * W + s] = a[k * STR];
  if (!WARP || lane == 0) {
    double ptmp[9], step_ia;
    load9(S.par, W, s, ptmp);
    for (int q = 0; q < n; q++) {
      const int ia = P.free_idx[q];
      step_ia = ia == 7 ? S.sc[SC_STEP7 * W + s] : P.step[ia];
      ptmp[ia] += x[q] * step_ia;
    }
    bounds_fold(ptmp, P, S.sc[SC_L70 * W + s], S.sc[SC_L71 * W + s]);
    store9(S.ptmp, W, s, ptmp);
  }
  if (WARP) __syncwarp(mask);
  return hits;
}

// solve_slot for a plan with all nine parameters free, one thread per slot,
// the matrix in registers (gr_svd_u9): the same trial steps and ladder.
// Trial 1 decomposes H; trial 2 uses the factor trial 1 stored; trial
// k >= 3 decomposes the factor trial k - 1 left (see solve_slot).
__device__ __forceinline__ void trial_params9(const DevPlan &P, const Slots &S, int s,
                                              const double x[9]) {
  const int W = S.W;
  double ptmp[9];
  load9(S.par, W, s, ptmp);
#pragma unroll
  for (int q = 0; q < 9; q++) ptmp[q] += x[q] * (q == 7 ? S.sc[SC_STEP7 * W + s] : P.step[q]);
  bounds_fold(ptmp, P, S.sc[SC_L70 * W + s], S.sc[SC_L71 * W + s]);
  store9(S.ptmp, W, s, ptmp);
}

template <bool FAST>
__device__ __forceinline__ int solve_slot9(const DevPlan &P, const Slots &S, int s) {
  const int W = S.W;
  const int tk = S.tk[s];
  double x[9];
  if (tk == 2) {  // U^T g with the stored factor, clamped
    double g[9];
#pragma unroll
    for (int k = 0; k < 9; k++) g[k] = S.jvec[(size_t)k * W + s];
#pragma unroll
    for (int j = 0; j < 9; j++) {
      double acc = 0.0;
#pragma unroll
      for (int i = 0; i < 9; i++) acc += S.hess[(size_t)(i * 9 + j) * W + s] * g[i];
      x[j] = acc > 0.5 ? 0.5 : (acc < -0.5 ? -0.5 : acc);
    }
    trial_params9(P, S, s, x);
    return 0;
  }
  double A[9][9], w[9];
#pragma unroll
  for (int r = 0; r < 9; r++)
#pragma unroll
    for (int c = 0; c < 9; c++) A[r][c] = S.hess[(size_t)(r * 9 + c) * W + s];
  const int hits = gr_svd_u9<FAST>(A, w);
#pragma unroll
  for (int r = 0; r < 9; r++)
#pragma unroll
    for (int c = 0; c < 9; c++) S.hess[(size_t)(r * 9 + c) * W + s] = A[r][c];
  double ug[9];  // U^T g
  {
    double g[9];
#pragma unroll
    for (int k = 0; k < 9; k++) g[k] = S.jvec[(size_t)k * W + s];
#pragma unroll
    for (int j = 0; j < 9; j++) {
      double acc = 0.0;
#pragma unroll
      for (int i = 0; i < 9; i++) acc += A[i][j] * g[i];
      ug[j] = acc;
    }
  }
  if (tk == 1) {
    double wmax = w[0];
#pragma unroll
    for (int i = 1; i < 9; i++) wmax = fmax(wmax, w[i]);
    double thr = P.svd_thr;
    while (true) {
      const double wthr = wmax * thr;
      double tj[9];
#pragma unroll
      for (int j = 0; j < 9; j++) {
        double wj = w[j];
        if (wj < wthr) {
          wj = 0.0;
          w[j] = 0.0;
        }
        tj[j] = wj > 1e-50 ? ug[j] / wj : 0.0;
      }
      bool inside = true;
#pragma unroll
      for (int i = 0; i < 9; i++) {
        double acc = 0.0;
#pragma unroll
        for (int j = 0; j < 9; j++) acc += A[i][j] * tj[j];
        x[i] = acc;
        if (acc > 0.5 || acc < -0.5) inside = false;
      }
      if (inside) break;
      if (thr > 2e-3) {
#pragma unroll
        for (int i = 0; i < 9; i++) x[i] = x[i] > 0.5 ? 0.5 : (x[i] < -0.5 ? -0.5 : x[i]);
        break;
      }
      thr *= 5.;
    }
  } else {
#pragma unroll
    for (int j = 0; j < 9; j++) x[j] = ug[j] > 0.5 ? 0.5 : (ug[j] < -0.5 ? -0.5 : ug[j]);
  }
  trial_params9(P, S, s, x);
  return hits;
}

// After a trial synthesis (chi_new, when the slot is in SL_TRIAL) or at a run
// that ended without one (SL_RUN_END): the accept / reject / convergence logic
// (Src/LM_FIT.c:588-646), the end-of-run restart policy (INVERSION,
// Src/LM_FIT.c:701-733) and, when the pixel is done, its result.  ROUNDS: the
// slot goes on the next round's lists and a finished slot takes the next
// pixel from the queue; otherwise (the tail kernel) it only changes state.
// One thread per slot.
template <bool ROUNDS>
__device__ __forceinline__ void trial_transition(const DevPlan &P, const InvertArgs &A,
                                                 const Slots &S, int s, int st, double chi_new,
                                                 int next_parity, Tally &t) {
  const int W = S.W;
  bool end_run = (st == SL_RUN_END);
  double par[9];
  load9(S.par, W, s, par);
  double *sc = S.sc;
  double chisq = sc[SC_CHISQ * W + s];
  double ratio = sc[SC_RATIO * W + s];
  double lmchisq = sc[SC_LMCHISQ * W + s];
  const long long pix = S.pix[s];
  const double l70 = sc[SC_L70 * W + s], l71 = sc[SC_L71 * W + s];

  if (!end_run) {
    // --------- Trial_Synthesis (Src/LM_FIT.c:473-527) ---------
    double ptmp[9];
    load9(S.ptmp, W, s, ptmp);
    lmchisq = chi_new;
    S.had_trial[s] = 1;
    S.cnt[2 * W + s]++;
    t.trials++;
    const double penalty = P.regul_any ? penalty_of(P, ptmp) : 0.0;
    if (chi_new < chisq) {  // accept (Src/LM_FIT.c:591-615)
      if (P.regul_any && penalty > 0.1 * lmchisq) ratio = 0.1 * chisq / penalty;
#pragma unroll
      for (int i = 0; i < 9; i++) par[i] = ptmp[i];
      store9(S.par, W, s, par);
      S.cnt[3 * W + s]++;
      t.acc++;
      const bool conv = ((chisq - chi_new) / chisq) < P.convg;
      chisq = chi_new;
      const int it = S.it[s] + 1;
      S.it[s] = it;
      if (conv || it >= P.niter) {
        end_run = true;
      } else {
        S.state[s] = SL_JAC_NEXT;
        if (ROUNDS) append_jac(S, next_parity, s);
      }
    } else {  // reject: grow the damping; past its limit the run ends
      const double damp = sc[SC_DAMP * W + s] * P.lam_reject;
      sc[SC_DAMP * W + s] = damp;
      if (damp > P.lam_lim[1]) {
        end_run = true;
      } else {  // another trial, on the SVD's U factor (solve_slot)
        S.tk[s]++;
        if (ROUNDS) append_rej(S, next_parity, s);
      }
    }
    sc[SC_CHISQ * W + s] = chisq;
    sc[SC_RATIO * W + s] = ratio;
    sc[SC_LMCHISQ * W + s] = lmchisq;
  }

  if (end_run) {
    // ---------------- end of one LM_FIT run (INVERSION) ----------------
    const double chisq_run = chisq / sc[SC_NORMP * W + s];
    int run = S.run[s];
    S.cnt[0 * W + s]++;
    t.runs++;
    double pbest[9];
    double best = sc[SC_BEST * W + s];
    const int first_run = A.init_par ? -1 : 0;
    if (chisq_run < P.chisq_crit || run == first_run || chisq_run < best) {
#pragma unroll
      for (int i = 0; i < 9; i++) pbest[i] = par[i];
      store9(S.pbest, W, s, pbest);
      best = chisq_run;
      sc[SC_BEST * W + s] = best;
    } else {
      load9(S.pbest, W, s, pbest);
    }
    bool stop = false;
    // a learned start that meets chisq_criteria ends the pixel; otherwise
    // the reference's schedule follows from run 0, keeping the best
    if (run < 0 && chisq_run < P.chisq_crit) {
      stop = true;
      t.learned++;
    }
    if (chisq_run < P.chisq_crit && (run >= 4 || run == P.nruns * 4)) stop = true;
    if (run >= P.nruns * 2 && best < P.chisq_crit * 2) stop = true;
    run++;
    S.run[s] = run;
    if (!stop && run < P.nruns * 4) {
      // Random_Jump (Src/LM_FIT.c:157-201)
      double g[9];
      load9(S.guess, W, s, g);
      if (run == 0) {  // after a learned start: the reference's first run
#pragma unroll
        for (int i = 0; i < 9; i++) par[i] = g[i];
      } else if (run < 4) {
#pragma unroll
        for (int i = 0; i < 9; i++) par[i] = pbest[i];
        par[2] = g[2] + kPi / 4. * run;
      } else {
        double z[8];
        restart_draws(P.seed, pix, run, z);
        par[0] = g[0] * (1 + 0.6 * z[0]);
        par[1] = g[1] + kPi / 8. * z[1];
        par[2] = g[2] + kPi / 4. * (run + 0.3 * z[2]);
        par[3] = g[3] + 5. * z[3];
        par[4] = pbest[4] * (1 + 0.2 * z[4]);
        par[5] = g[5] + 0.1 * z[5];
        par[6] = g[6] + 5 * z[6];
        par[7] = pbest[7];
        par[8] = g[8] + 0.1 * z[7];
      }
      if (run > 0) bounds_fold(par, P, l70, l71);
      store9(S.par, W, s, par);
      S.state[s] = SL_JAC_START;
      if (ROUNDS) append_jac(S, next_parity, s);
    } else {
      // pixel done: best-fit profile, theta fold, HMI_REF, result
      // (Src/LM_FIT.c:727-733, 791-799)
      if (A.fitpar) store9_px(A.fitpar, pix, pbest);  // profiles: launch_fit after the batch
      if (pbest[1] > kPi) pbest[1] -= kPi;
      if (P.hmi_ref) {
        pbest[2] += 0.5 * kPi;
        if (pbest[2] > kPi) pbest[2] -= kPi;
      }
      double *r = A.res + (size_t)pix * 10;
#pragma unroll
      for (int i = 0; i < 9; i++) r[i] = pbest[i];
      r[9] = best;
      if (A.flags) A.flags[pix] = 1 | (S.had_trial[s] ? 2 : 0);
      if (A.lastchi) A.lastchi[pix] = sc[SC_LMCHISQ * W + s];
      if (A.counters) {
        uint4 c4 = make_uint4(S.cnt[0 * W + s], S.cnt[1 * W + s], S.cnt[2 * W + s],
                              S.cnt[3 * W + s]);
        reinterpret_cast<uint4 *>(A.counters)[pix] = c4;
      }
      t.iter += S.cnt[1 * W + s];
      const int got = ROUNDS ? refill(P, A, S, s, t.valid) : kExhausted;
      if (got == kRefilled) {
        append_jac(S, next_parity, s);
      } else if (got == kExhausted) {
        S.state[s] = SL_DONE;
        t.busy_delta--;
      }  // kWaiting: the slot holds a queue position (still busy)
    }
  }
}

}  // namespace detail

using namespace detail;

// ---------------------------------------------------------------------------
// Synthesis with Jacobian + normal equations for the slots of jlist[parity].
// ---------------------------------------------------------------------------
// Kernel variants (pixels per CTA BLOCK, the grid staged in shared memory,
// the reciprocal table): the same arithmetic, bit for bit.
template <class T, bool STAGE>
__device__ __forceinline__ const T *stage_grid(const DevPlan &P, T *s_grid) {
  if (!STAGE) return nullptr;
  const int m = P.nl * P.nsub;
  if (m > kMaxStage) return nullptr;
  for (int i = threadIdx.x; i < m; i += blockDim.x) s_grid[i] = grid_value<T>(P, i);
  return s_grid;  // (voigt_block_setup's barrier follows)
}

// SACC: the normal-equation sums in shared memory (deriv_pass_sacc), compiled
// for 3 CTAs of 128 per SM instead of 2
template <class T, bool FILT, int BLOCK, bool STAGE, bool TABLE, bool SACC = false>
__global__ void __launch_bounds__(BLOCK, SACC ? 3 : ME_JAC_MINB * kBlock / BLOCK)
    jac_kernel(const __grid_constant__ DevPlan P, const __grid_constant__ InvertArgs A,
               const __grid_constant__ Slots S, int parity) {
  __shared__ T s_tab[100];
  __shared__ T s_rden[TABLE ? kRden * BLOCK : 1];
  __shared__ T s_grid[STAGE ? kMaxStage : 1];
  __shared__ T s_acc[SACC ? 54 * BLOCK : 1];
  const T *sgrid = stage_grid<T, STAGE>(P, s_grid);
  VoigtK<T> K;
  voigt_block_setup<T>(K, P, s_tab);
  T *rden = TABLE ? s_rden + threadIdx.x : nullptr;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    S.jcount[parity ^ 1] = 0;
    S.rcount[parity ^ 1] = 0;
  }
  const int count = S.jcount[parity];
  const int W = S.W;
  const int nl = P.nl;
  Tally t;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const int s = S.jlist[parity * W + i];
    const double *pp = S.obs ? S.obs + s : A.prof + (size_t)S.pix[s] * 4 * nl;
    const int pstr = S.obs ? W : 1;
    double par[9], step[9], sw[4];
    load9(S.par, W, s, par);
    slot_weights(P, S, s, step, sw);
    double H45[45], g9[9];
    const double chi0 =
        SACC ? deriv_pass_sacc<T, FILT, BLOCK>(P, K, rden, par, step, pp, sw, H45, g9, sgrid,
                                               s_acc + threadIdx.x, pstr)
             : deriv_pass<T, FILT>(P, K, rden, par, step, pp, sw, H45, g9, sgrid, pstr);
    t.jac++;
    jac_store<sizeof(T) == sizeof(float)>(P, S, s, par, chi0, H45, g9);
  }
  t.flush(A, S);
}

// ---------------------------------------------------------------------------
// The SVD solves of the slots' trial steps (solve_slot), one thread per slot,
// its matrix in its own column of shared memory.  which = 0: the slots that
// just built their normal matrix (the Jacobian list of this round, first
// trials); which = 1: the slots going on after a rejected trial.  Two launches
// keep the costly decompositions of H apart from the cheap ones of orthogonal
// factors.
// ---------------------------------------------------------------------------
static __global__ void __launch_bounds__(kSvdBlock) svd_kernel(const __grid_constant__ DevPlan P,
                                                               const __grid_constant__ InvertArgs A,
                                                               const __grid_constant__ Slots S,
                                                               int parity, int which) {
  extern __shared__ double sm[];
  const int t = threadIdx.x;
  double *a = sm + t;
  double *w = sm + 81 * kSvdBlock + t;
  double *rv1 = sm + 90 * kSvdBlock + t;
  const int W = S.W;
  Tally tl;
  const int *list = which == 0 ? S.jlist + parity * W : S.rlist + parity * W;
  const int count = which == 0 ? S.jcount[parity] : S.rcount[parity];
  for (int i = blockIdx.x * kSvdBlock + t; i < count; i += gridDim.x * kSvdBlock) {
    const int s = list[i];
    if (S.state[s] != SL_TRIAL) continue;
    tl.svdlim += solve_slot<kSvdBlock, 1>(P, S, s, a, w, rv1, 0, 0u);
  }
  tl.flush(A, S);
}

// svd_kernel for plans with all nine parameters free: each thread's matrix in
// its registers (solve_slot9), no shared memory.
template <bool FAST>
static __global__ void __launch_bounds__(kSvdBlock) svd9_kernel(const __grid_constant__ DevPlan P,
                                                                const __grid_constant__ InvertArgs A,
                                                                const __grid_constant__ Slots S,
                                                                int parity, int which) {
  const int W = S.W;
  Tally tl;
  const int *list = which == 0 ? S.jlist + parity * W : S.rlist + parity * W;
  const int count = which == 0 ? S.jcount[parity] : S.rcount[parity];
  for (int i = blockIdx.x * kSvdBlock + threadIdx.x; i < count; i += gridDim.x * kSvdBlock) {
    const int s = list[i];
    if (S.state[s] != SL_TRIAL) continue;
    tl.svdlim += solve_slot9<FAST>(P, S, s);
  }
  tl.flush(A, S);
}

// ---------------------------------------------------------------------------
// One trial step for every slot; run and pixel transitions; refills.
// ---------------------------------------------------------------------------
template <class T, bool FILT, int BLOCK, bool STAGE, bool TABLE>
__global__ void __launch_bounds__(BLOCK) trial_kernel(const __grid_constant__ DevPlan P,
                                                      const __grid_constant__ InvertArgs A,
                                                      const __grid_constant__ Slots S,
                                                      int parity) {
  __shared__ T s_tab[100];
  __shared__ T s_rden[TABLE ? kRden * BLOCK : 1];
  __shared__ T s_grid[STAGE ? kMaxStage : 1];
  const T *sgrid = stage_grid<T, STAGE>(P, s_grid);
  VoigtK<T> K;
  voigt_block_setup<T>(K, P, s_tab);
  T *rden = TABLE ? s_rden + threadIdx.x : nullptr;
  const int W = S.W;
  const int nl = P.nl;
  const int next_parity = parity ^ 1;
  Tally t;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < W; s += gridDim.x * blockDim.x) {
    const int st = S.state[s];
    if (st == SL_DONE) continue;
    if (st == SL_EMPTY || st == SL_WAIT) {
      // a waiting slot counts as busy; it takes up the position it holds
      const int r = refill(P, A, S, s, t.valid, st == SL_WAIT ? S.pix[s] : -1);
      if (r == kRefilled) append_jac(S, next_parity, s);
      if (st == SL_EMPTY && r != kExhausted) t.busy_delta++;
      if (r == kExhausted) {
        S.state[s] = SL_DONE;
        if (st == SL_WAIT) t.busy_delta--;
      }
      continue;
    }
    double chi_new = 0.0;
    if (st != SL_RUN_END) {  // Trial_Synthesis's synthesis, after svd_kernel
      double ptmp[9], step[9], sw[4];
      load9(S.ptmp, W, s, ptmp);
      slot_weights(P, S, s, step, sw);
      // one call site, so that both sources of the observed values run the
      // same compiled synthesis
      const double *pp = S.obs ? S.obs + s : A.prof + (size_t)S.pix[s] * 4 * nl;
      chi_new = forward_pass<T, FILT>(P, K, rden, ptmp, step, pp, sw, nullptr, sgrid,
                                      S.obs ? W : 1);
    }
    trial_transition<true>(P, A, S, s, st, chi_new, next_parity, t);
  }
  t.flush(A, S);
}

// ---------------------------------------------------------------------------
// The tail: once the queue is empty and few pixels remain, rounds are bound by
// the latency of one thread's synthesis and SVD.  finish_kernel takes the
// remaining slots one per warp (an atomic cursor over the W slots) and runs
// each to completion with the same per-slot steps: the synthesis's
// wavelengths spread over the lanes (deriv_warp / forward_warp: per-point
// terms staged in shared memory, every sum formed by one lane in the
// thread-serial order), the SVD on gr_svd_u_grp<32>, and the scalar transitions
// in lane 0.  No lists, no refills.  The operations and their order are the
// rounds'; only the compiler's contraction of multiply-adds may differ in
// this kernel, so results agree to rounding (and, the LM being sensitive to
// the last bit, some pixels then take another path, as under a one-ulp
// change of their input).
// ---------------------------------------------------------------------------
template <class T>
struct FinishSmem {
  T tab[100];
  T J[kBlock / 32][32 * 36];       // per warp: Jacobian rows of 32 points
  double R[kBlock / 32][32 * 4];   // per warp: weighted residuals of 32 points
  double a[kBlock / 32][81];       // per warp: the SVD's matrix
  T rden[kBlock / 32][kRden];      // per warp: the Voigt reciprocal table
};

namespace detail {

// voigt_prepare for a warp: one shared reciprocal table, entry n by lane n.
template <class T>
__device__ __forceinline__ void voigt_prepare_warp(VoigtK<T> &K, T y, T *rden, int lane) {
  __syncwarp();
  voigt_prepare<T>(K, y, nullptr, 1);
  K.rden = rden;
  K.rstride = 1;
  if (sizeof(T) == sizeof(float) && lane < kRden)
    rden[lane] = T(1) / (K.aa * T(lane * lane) + K.yy);
  __syncwarp();
}

// deriv_pass across a warp.  H45 / g9 land in hg[0..53] (shared, all lanes
// may read after the call); returns chi^2 / (4 nl) in every lane.
template <class T, bool FILT>
__device__ double deriv_warp(const DevPlan &P, VoigtK<T> &K, T *rden, const double *par,
                             const double *step, const double *prof, const double sw[4],
                             int lane, T *stJ, double *stR, double *hg) {
  SynthCall<T> c;
  synth_setup<T>(c, par, P, step);
  voigt_prepare_warp<T>(K, c.p5, rden, lane);
  const int nl = P.nl;
  const T tsw[4] = {T(sw[0]), T(sw[1]), T(sw[2]), T(sw[3])};
  // this lane's sums: h entries lane and lane + 32 (upper triangle, row-major)
  // and g entry lane
  int i0 = 0, j0 = 0, i1 = 0, j1 = 0;
  {
    int idx = 0;
    for (int i = 0; i < 9; i++)
      for (int j = i; j < 9; j++, idx++) {
        if (idx == lane) i0 = i, j0 = j;
        if (idx == lane + 32) i1 = i, j1 = j;
      }
  }
  const bool has1 = lane + 32 < 45, hasg = lane < 9;
  T h0 = T(0), h1 = T(0), gl = T(0);
  double chi = 0.0;
  for (int base = 0; base < nl; base += 32) {
    const int iw = base + lane;
    if (iw < nl) {
      T syn[4], J[4][9];
      channel_point<T, true, FILT>(c, P, K, tsw, iw, syn, J);
#pragma unroll
      for (int s = 0; s < 4; s++) stR[lane * 4 + s] = ((double)syn[s] - __ldg(prof + s * nl + iw)) * sw[s];
#pragma unroll
      for (int s = 0; s < 4; s++)
#pragma unroll
        for (int k = 0; k < 9; k++) stJ[lane * 36 + s * 9 + k] = J[s][k];
    }
    __syncwarp();
    const int cnt = nl - base < 32 ? nl - base : 32;
    for (int q = 0; q < cnt; q++) {
      const double *rq = stR + q * 4;
      const T *Jq = stJ + q * 36;
      T r[4];
#pragma unroll
      for (int s = 0; s < 4; s++) {
        const double rd = rq[s];
        chi += rd * rd;
        r[s] = T(rd);
      }
      h0 += Jq[i0] * Jq[j0] + Jq[9 + i0] * Jq[9 + j0] + Jq[18 + i0] * Jq[18 + j0] +
            Jq[27 + i0] * Jq[27 + j0];
      if (has1)
        h1 += Jq[i1] * Jq[j1] + Jq[9 + i1] * Jq[9 + j1] + Jq[18 + i1] * Jq[18 + j1] +
              Jq[27 + i1] * Jq[27 + j1];
      if (hasg) gl -= Jq[lane] * r[0] + Jq[9 + lane] * r[1] + Jq[18 + lane] * r[2] + Jq[27 + lane] * r[3];
    }
    __syncwarp();
  }
  hg[lane] = (double)h0;
  if (has1) hg[lane + 32] = (double)h1;
  if (hasg) hg[45 + lane] = (double)gl;
  __syncwarp();
  return chi / (4.0 * nl);
}

// forward_pass across a warp (chi^2 only); every lane gets the result.
template <class T, bool FILT>
__device__ double forward_warp(const DevPlan &P, VoigtK<T> &K, T *rden, const double *par,
                               const double *step, const double *prof, const double sw[4],
                               int lane, double *stR) {
  SynthCall<T> c;
  synth_setup<T>(c, par, P, step);
  voigt_prepare_warp<T>(K, c.p5, rden, lane);
  const T ones[4] = {T(1), T(1), T(1), T(1)};
  const int nl = P.nl;
  double chi = 0.0;
  for (int base = 0; base < nl; base += 32) {
    const int iw = base + lane;
    if (iw < nl) {
      T syn[4];
      channel_point<T, false, FILT>(c, P, K, ones, iw, syn, nullptr);
#pragma unroll
      for (int s = 0; s < 4; s++) stR[lane * 4 + s] = ((double)syn[s] - __ldg(prof + s * nl + iw)) * sw[s];
    }
    __syncwarp();
    const int cnt = nl - base < 32 ? nl - base : 32;
    for (int q = 0; q < cnt; q++)
#pragma unroll
      for (int s = 0; s < 4; s++) {
        const double rd = stR[q * 4 + s];
        chi += rd * rd;
      }
    __syncwarp();
  }
  return chi / (4.0 * nl);
}

}  // namespace detail

// (compiled for one CTA per SM at least: 230 registers and no spill on the FP32
// path, where the default budget spilled; the kernel runs a few warps per SM)
template <class T, bool FILT>
__global__ void __launch_bounds__(kBlock, 1) finish_kernel(const __grid_constant__ DevPlan P,
                                                        const __grid_constant__ InvertArgs A,
                                                        const __grid_constant__ Slots S,
                                                        int *cursor) {
  __shared__ FinishSmem<T> sm;
  VoigtK<T> K;
  voigt_block_setup<T>(K, P, sm.tab);
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  T *stJ = sm.J[wp];
  double *stR = sm.R[wp];
  double *a = sm.a[wp];
  T *rden = sm.rden[wp];
  const int W = S.W;
  const int nl = P.nl;
  const long long cap = slot_step_cap(P);
  Tally t;
  while (true) {
    int s = 0;
    if (lane == 0) s = atomicAdd(cursor, 1);
    s = __shfl_sync(0xffffffffu, s, 0);
    if (s >= W) break;
    long long steps = 0;
    while (true) {
      __syncwarp();
      // lane 0 made the last transition: its view of the state decides
      const int st = __shfl_sync(0xffffffffu, S.state[s], 0);
      if (st == SL_DONE || st == SL_EMPTY) break;
      const long long pix = S.pix[s];
      const double *pp = A.prof + (size_t)pix * 4 * nl;
      if (++steps > cap) {  // cannot happen for a valid plan; ends the pixel with a flag
        if (lane == 0) {
          if (A.flags) A.flags[pix] = 8;
          S.state[s] = SL_DONE;
          t.busy_delta--;
        }
        __syncwarp();
        break;
      }
      double step[9], sw[4];
      slot_weights(P, S, s, step, sw);
      if (st == SL_JAC_START || st == SL_JAC_NEXT) {
        double par[9];
        load9(S.par, W, s, par);
        const double chi0 = deriv_warp<T, FILT>(P, K, rden, par, step, pp, sw, lane, stJ, stR, stR);
        if (lane == 0) {
          double H45[45], g9[9];
          for (int k = 0; k < 45; k++) H45[k] = stR[k];
          for (int k = 0; k < 9; k++) g9[k] = stR[45 + k];
          t.jac++;
          jac_store(P, S, s, par, chi0, H45, g9);
        }
        continue;
      }
      double chi_new = 0.0;
      if (st == SL_TRIAL) {
        double w[9];
        const int hits = solve_slot<1, 32>(P, S, s, a, w, nullptr, lane, 0xffffffffu);
        if (lane == 0) t.svdlim += hits;
        double ptmp[9];
        load9(S.ptmp, W, s, ptmp);
        chi_new = forward_warp<T, FILT>(P, K, rden, ptmp, step, pp, sw, lane, stR);
      }
      if (lane == 0) trial_transition<false>(P, A, S, s, st, chi_new, 0, t);
    }
  }
  if (lane == 0) t.flush(A, S);
}

// ---------------------------------------------------------------------------
// Lane-split rounds.  Once the queue is empty, the pixels still in flight are
// too few to fill the GPU one thread each, and every round waits for one
// thread's synthesis and SVD.  These variants of the round kernels give each
// slot a group of G consecutive lanes (G = 2 ... 32, chosen by the host from
// the number in flight): the group splits the wavelengths of the synthesis
// (partial sums of H, g and chi^2 per lane, then a butterfly over the group)
// and the vector loops of the SVD (gr_svd_u_grp); lane 0 makes the scalar
// transitions.  The trial kernel runs over this round's lists only (no
// refills are left).  Sums over the wavelengths are formed in another order
// than the thread-per-slot kernels', so results agree with them to rounding.
// The SVD variant also serves the full rounds (svd_lanes).
// ---------------------------------------------------------------------------
template <int G>
struct Grp {
  int lane;       // 0 .. G-1
  unsigned mask;  // the group's lanes in its warp
  __device__ __forceinline__ Grp() {
    const int wl = threadIdx.x & 31;
    lane = wl & (G - 1);
    mask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << (wl & ~(G - 1)));
  }
  template <class V>
  __device__ __forceinline__ V sum(V v) const {
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, G);
    return v;
  }
};

namespace detail {

// deriv_pass over a group: lane t takes wavelengths t, t + G, ...; every lane
// returns the full H45, g9 and chi^2 / (4 nl).
template <class T, int G, bool FILT>
__device__ __forceinline__ double deriv_grp(const DevPlan &P, VoigtK<T> &K, T *rden,
                                            const double *par, const double *step,
                                            const double *prof, const double sw[4],
                                            const Grp<G> &grp, double *H45, double *g9) {
  SynthCall<T> c;
  synth_setup<T>(c, par, P, step);
  voigt_prepare<T>(K, c.p5, rden, blockDim.x);
  T h[45], g[9];
#pragma unroll
  for (int i = 0; i < 45; i++) h[i] = T(0);
#pragma unroll
  for (int i = 0; i < 9; i++) g[i] = T(0);
  double chi = 0.0;
  const int nl = P.nl;
  const T tsw[4] = {T(sw[0]), T(sw[1]), T(sw[2]), T(sw[3])};
#pragma unroll 1
  for (int iw = grp.lane; iw < nl; iw += G) {
    T syn[4], J[4][9];
    channel_point<T, true, FILT>(c, P, K, tsw, iw, syn, J);
    T r[4];
#pragma unroll
    for (int s = 0; s < 4; s++) {
      const double rd = ((double)syn[s] - __ldg(prof + s * nl + iw)) * sw[s];
      chi += rd * rd;
      r[s] = T(rd);
    }
    int idx = 0;
#pragma unroll
    for (int i = 0; i < 9; i++) {
#pragma unroll
      for (int j = i; j < 9; j++) {
        h[idx] += J[0][i] * J[0][j] + J[1][i] * J[1][j] + J[2][i] * J[2][j] + J[3][i] * J[3][j];
        idx++;
      }
      g[i] -= J[0][i] * r[0] + J[1][i] * r[1] + J[2][i] * r[2] + J[3][i] * r[3];
    }
  }
#pragma unroll
  for (int i = 0; i < 45; i++) H45[i] = (double)grp.sum(h[i]);
#pragma unroll
  for (int i = 0; i < 9; i++) g9[i] = (double)grp.sum(g[i]);
  return grp.sum(chi) / (4.0 * nl);
}

// forward_pass over a group (chi^2 only); every lane gets the result.
template <class T, int G, bool FILT>
__device__ __forceinline__ double forward_grp(const DevPlan &P, VoigtK<T> &K, T *rden,
                                              const double *par, const double *step,
                                              const double *prof, const double sw[4],
                                              const Grp<G> &grp) {
  SynthCall<T> c;
  synth_setup<T>(c, par, P, step);
  voigt_prepare<T>(K, c.p5, rden, blockDim.x);
  const T ones[4] = {T(1), T(1), T(1), T(1)};
  double chi = 0.0;
  const int nl = P.nl;
#pragma unroll 1
  for (int iw = grp.lane; iw < nl; iw += G) {
    T syn[4];
    channel_point<T, false, FILT>(c, P, K, ones, iw, syn, nullptr);
#pragma unroll
    for (int s = 0; s < 4; s++) {
      const double rd = ((double)syn[s] - __ldg(prof + s * nl + iw)) * sw[s];
      chi += rd * rd;
    }
  }
  return grp.sum(chi) / (4.0 * nl);
}

}  // namespace detail

// jac_kernel with G lanes per slot of jlist[parity].
template <class T, int G, bool FILT>
__global__ void __launch_bounds__(kBlock, ME_JAC_MINB)
    jac_grp_kernel(const __grid_constant__ DevPlan P, const __grid_constant__ InvertArgs A,
                   const __grid_constant__ Slots S, int parity) {
  __shared__ T s_tab[100];
  __shared__ T s_rden[kRden * kBlock];
  VoigtK<T> K;
  voigt_block_setup<T>(K, P, s_tab);
  T *rden = s_rden + threadIdx.x;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    S.jcount[parity ^ 1] = 0;
    S.rcount[parity ^ 1] = 0;
  }
  const Grp<G> grp;
  const int count = S.jcount[parity];
  const int W = S.W;
  const int nl = P.nl;
  Tally t;
  const int per_grid = gridDim.x * (blockDim.x / G);
  for (int i = blockIdx.x * (blockDim.x / G) + threadIdx.x / G; i < count; i += per_grid) {
    const int s = S.jlist[parity * W + i];
    const double *pp = A.prof + (size_t)S.pix[s] * 4 * nl;
    double par[9], step[9], sw[4];
    load9(S.par, W, s, par);
    slot_weights(P, S, s, step, sw);
    double H45[45], g9[9];
    const double chi0 = deriv_grp<T, G, FILT>(P, K, rden, par, step, pp, sw, grp, H45, g9);
    if (grp.lane == 0) {
      t.jac++;
      jac_store(P, S, s, par, chi0, H45, g9);
    }
  }
  t.flush(A, S);
}

// svd_kernel with G lanes per slot, its matrix row-major in shared memory.
template <int G>
__global__ void __launch_bounds__(kBlock)
    svd_grp_kernel(const __grid_constant__ DevPlan P, const __grid_constant__ InvertArgs A,
                   const __grid_constant__ Slots S, int parity, int which) {
  __shared__ double s_a[kBlock / G][81];
  const Grp<G> grp;
  double *a = s_a[threadIdx.x / G];
  const int W = S.W;
  Tally tl;
  const int *list = which == 0 ? S.jlist + parity * W : S.rlist + parity * W;
  const int count = which == 0 ? S.jcount[parity] : S.rcount[parity];
  const int per_grid = gridDim.x * (blockDim.x / G);
  for (int i = blockIdx.x * (blockDim.x / G) + threadIdx.x / G; i < count; i += per_grid) {
    const int s = list[i];
    if (S.state[s] != SL_TRIAL) continue;  // uniform across the group
    double w[9];
    const int hits = solve_slot<1, G>(P, S, s, a, w, nullptr, grp.lane, grp.mask);
    if (grp.lane == 0) tl.svdlim += hits;
  }
  tl.flush(A, S);
}

// trial_kernel with G lanes per slot, over this round's lists (jlist: first
// trials or run ends; rlist: later trials); no refills.
template <class T, int G, bool FILT>
__global__ void __launch_bounds__(kBlock)
    trial_grp_kernel(const __grid_constant__ DevPlan P, const __grid_constant__ InvertArgs A,
                     const __grid_constant__ Slots S, int parity) {
  __shared__ T s_tab[100];
  __shared__ T s_rden[kRden * kBlock];
  VoigtK<T> K;
  voigt_block_setup<T>(K, P, s_tab);
  T *rden = s_rden + threadIdx.x;
  const Grp<G> grp;
  const int W = S.W;
  const int nl = P.nl;
  const int next_parity = parity ^ 1;
  const int nj = S.jcount[parity], nr = S.rcount[parity];
  Tally t;
  const int per_grid = gridDim.x * (blockDim.x / G);
  for (int i = blockIdx.x * (blockDim.x / G) + threadIdx.x / G; i < nj + nr; i += per_grid) {
    const int s = i < nj ? S.jlist[parity * W + i] : S.rlist[parity * W + (i - nj)];
    const int st = S.state[s];
    if (st != SL_TRIAL && st != SL_RUN_END) continue;  // uniform across the group
    double chi_new = 0.0;
    if (st == SL_TRIAL) {
      double ptmp[9], step[9], sw[4];
      load9(S.ptmp, W, s, ptmp);
      slot_weights(P, S, s, step, sw);
      chi_new = forward_grp<T, G, FILT>(P, K, rden, ptmp, step, A.prof + (size_t)S.pix[s] * 4 * nl,
                                  sw, grp);
    }
    if (grp.lane == 0) trial_transition<true>(P, A, S, s, st, chi_new, next_parity, t);
  }
  if (grp.lane == 0) t.flush(A, S);
}

// ---------------------------------------------------------------------------
// Launchers, instantiated per synthesis precision T and instrument-filter
// variant FILT by me_invert_{f32,f64}{,f}.cu (ME_INSTANTIATE_ROUNDS).
// ---------------------------------------------------------------------------
// which: 0 = jac_kernel, 1 = trial_kernel, 2 = svd_kernel, 3 = finish_kernel
// (CTAs for a full device)
template <class T, bool FILT>
int round_grid_impl(int which, int device) {
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (which == 0) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, jac_kernel<T, FILT, kBlock, false, true>,
                                                  kBlock, 0);
  } else if (which == 1) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, trial_kernel<T, FILT, kBlock, false, true>, kBlock, 0);
  } else if (which == 3) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, finish_kernel<T, FILT>, kBlock, 0);
  } else {
    // the larger of the two SVD kernels' resident grids (a grid beyond one
    // kernel's residency only queues blocks)
    cudaFuncSetAttribute(svd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSvdSmem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, svd_kernel, kSvdBlock, kSvdSmem);
    int per_sm9 = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm9, svd9_kernel<false>, kSvdBlock, 0);
    int per_sm9f = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm9f, svd9_kernel<true>, kSvdBlock, 0);
    if (per_sm9f > per_sm9) per_sm9 = per_sm9f;
    if (per_sm9 > per_sm) per_sm = per_sm9;
  }
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

// static: svd_kernel has internal linkage, so each translation unit must launch
// its own copy (the one whose shared-memory limit round_grid_impl raised); an
// inline function with external linkage would be merged across the units by
// the linker and launch one unit's kernel for every precision
static inline void launch_svd_lanes(int lanes, const DevPlan &P, const InvertArgs &A,
                                    const Slots &S, int parity, int which, int grid,
                                    cudaStream_t st) {
  switch (lanes) {
    case 2: svd_grp_kernel<2><<<grid, kBlock, 0, st>>>(P, A, S, parity, which); break;
    case 4: svd_grp_kernel<4><<<grid, kBlock, 0, st>>>(P, A, S, parity, which); break;
    case 8: svd_grp_kernel<8><<<grid, kBlock, 0, st>>>(P, A, S, parity, which); break;
    default:
      if (P.npar == 9 && P.svd_regs && P.fastg)
        svd9_kernel<true><<<grid, kSvdBlock, 0, st>>>(P, A, S, parity, which);
      else if (P.npar == 9 && P.svd_regs)
        svd9_kernel<false><<<grid, kSvdBlock, 0, st>>>(P, A, S, parity, which);
      else
        svd_kernel<<<grid, kSvdBlock, kSvdSmem, st>>>(P, A, S, parity, which);
      break;
  }
}

// The Jacobian / trial kernel of the plan's variant (P.kvar, kKernelVariants):
// `grid` CTAs of kBlock threads, or as many threads in CTAs of another size.
template <class T, bool FILT>
void launch_jac_variant(const DevPlan &P, const InvertArgs &A, const Slots &S, int parity,
                        int grid, cudaStream_t st) {
  switch (P.kvar) {
    case 1: jac_kernel<T, FILT, 64, false, true><<<grid * 2, 64, 0, st>>>(P, A, S, parity); break;
    case 2:
      jac_kernel<T, FILT, 256, false, true><<<(grid + 1) / 2, 256, 0, st>>>(P, A, S, parity);
      break;
    case 3: jac_kernel<T, FILT, kBlock, true, true><<<grid, kBlock, 0, st>>>(P, A, S, parity); break;
    case 4: jac_kernel<T, FILT, kBlock, false, false><<<grid, kBlock, 0, st>>>(P, A, S, parity); break;
    case 5:
      // FP32 only (FP64 sums would not fit in a CTA's static shared memory)
      if constexpr (sizeof(T) == sizeof(float)) {
        jac_kernel<T, FILT, kBlock, false, true, true><<<grid * 3 / 2, kBlock, 0, st>>>(P, A, S,
                                                                                     parity);
        break;
      }
      [[fallthrough]];
    default: jac_kernel<T, FILT, kBlock, false, true><<<grid, kBlock, 0, st>>>(P, A, S, parity);
  }
}
template <class T, bool FILT>
void launch_trial_variant(const DevPlan &P, const InvertArgs &A, const Slots &S, int parity,
                          int grid, cudaStream_t st) {
  switch (P.kvar) {
    case 1: trial_kernel<T, FILT, 64, false, true><<<grid * 2, 64, 0, st>>>(P, A, S, parity); break;
    case 2:
      trial_kernel<T, FILT, 256, false, true><<<(grid + 1) / 2, 256, 0, st>>>(P, A, S, parity);
      break;
    case 3: trial_kernel<T, FILT, kBlock, true, true><<<grid, kBlock, 0, st>>>(P, A, S, parity); break;
    case 4: trial_kernel<T, FILT, kBlock, false, false><<<grid, kBlock, 0, st>>>(P, A, S, parity); break;
    default: trial_kernel<T, FILT, kBlock, false, true><<<grid, kBlock, 0, st>>>(P, A, S, parity);
  }
}

// grids: jac_kernel, trial_kernel, svd; svd_lanes: lanes per matrix of the
// SVD launches (1: svd_kernel, one thread each; 2, 4, 8: svd_grp_kernel).
template <class T, bool FILT>
cudaError_t launch_round_impl(const DevPlan &P, const InvertArgs &A, const Slots &S, int parity,
                              const int grids[3], cudaStream_t st, cudaEvent_t *ev,
                              int svd_lanes, const Overlap *ov) {
  if (ov) {  // later trials' SVDs beside the Jacobian kernel
    cudaEventRecord(ov->fork, st);
    cudaStreamWaitEvent(ov->aux, ov->fork, 0);
    launch_svd_lanes(svd_lanes, P, A, S, parity, 1, grids[2], ov->aux);
    cudaEventRecord(ov->join, ov->aux);
  }
  if (ev) cudaEventRecord(ev[0], st);
  launch_jac_variant<T, FILT>(P, A, S, parity, grids[0], st);
  if (ev) cudaEventRecord(ev[1], st);
  launch_svd_lanes(svd_lanes, P, A, S, parity, 0, grids[2], st);
  if (ev) cudaEventRecord(ev[2], st);
  if (ov)
    cudaStreamWaitEvent(st, ov->join, 0);
  else
    launch_svd_lanes(svd_lanes, P, A, S, parity, 1, grids[2], st);
  if (ev) cudaEventRecord(ev[3], st);
  launch_trial_variant<T, FILT>(P, A, S, parity, grids[1], st);
  if (ev) cudaEventRecord(ev[4], st);
  return cudaGetLastError();
}

// The SVD launches of a lane-split round: G lanes per matrix in shared memory
// (svd_grp_kernel), or, with P.svd_regs == 2 and all nine parameters free,
// one thread per matrix in registers (svd9_kernel; the grid of G-lane groups
// has at least one thread per slot).
template <int G>
static inline void launch_svd_grp(const DevPlan &P, const InvertArgs &A, const Slots &S,
                                  int parity, int which, int grid, cudaStream_t st) {
  if (P.npar == 9 && P.svd_regs == 2 && P.fastg)
    svd9_kernel<true><<<grid * (kBlock / kSvdBlock), kSvdBlock, 0, st>>>(P, A, S, parity, which);
  else if (P.npar == 9 && P.svd_regs == 2)
    svd9_kernel<false><<<grid * (kBlock / kSvdBlock), kSvdBlock, 0, st>>>(P, A, S, parity, which);
  else
    svd_grp_kernel<G><<<grid, kBlock, 0, st>>>(P, A, S, parity, which);
}

template <class T, int G, bool FILT>
void launch_grp(const DevPlan &P, const InvertArgs &A, const Slots &S, int parity,
                const int grids[3], cudaStream_t st, cudaEvent_t *ev, const Overlap *ov) {
  if (ov) {
    cudaEventRecord(ov->fork, st);
    cudaStreamWaitEvent(ov->aux, ov->fork, 0);
    launch_svd_grp<G>(P, A, S, parity, 1, grids[2], ov->aux);
    cudaEventRecord(ov->join, ov->aux);
  }
  if (ev) cudaEventRecord(ev[0], st);
  jac_grp_kernel<T, G, FILT><<<grids[0], kBlock, 0, st>>>(P, A, S, parity);
  if (ev) cudaEventRecord(ev[1], st);
  launch_svd_grp<G>(P, A, S, parity, 0, grids[2], st);
  if (ev) cudaEventRecord(ev[2], st);
  if (ov)
    cudaStreamWaitEvent(st, ov->join, 0);
  else
    launch_svd_grp<G>(P, A, S, parity, 1, grids[2], st);
  if (ev) cudaEventRecord(ev[3], st);
  trial_grp_kernel<T, G, FILT><<<grids[1], kBlock, 0, st>>>(P, A, S, parity);
  if (ev) cudaEventRecord(ev[4], st);
}

// A round with G lanes per slot (G = 2, 4, 8, 16, 32), after the queue is empty.
template <class T, bool FILT>
cudaError_t launch_round_grp_impl(int G, const DevPlan &P, const InvertArgs &A, const Slots &S,
                                  int parity, const int grids[3], cudaStream_t st,
                                  cudaEvent_t *ev, const Overlap *ov) {
  switch (G) {
    case 2: launch_grp<T, 2, FILT>(P, A, S, parity, grids, st, ev, ov); break;
    case 4: launch_grp<T, 4, FILT>(P, A, S, parity, grids, st, ev, ov); break;
    case 8: launch_grp<T, 8, FILT>(P, A, S, parity, grids, st, ev, ov); break;
    case 16: launch_grp<T, 16, FILT>(P, A, S, parity, grids, st, ev, ov); break;
    case 32: launch_grp<T, 32, FILT>(P, A, S, parity, grids, st, ev, ov); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

template <class T, bool FILT>
cudaError_t launch_finish_impl(const DevPlan &P, const InvertArgs &A, const Slots &S, int *cursor,
                               int grid, cudaStream_t st) {
  finish_kernel<T, FILT><<<grid, kBlock, 0, st>>>(P, A, S, cursor);
  return cudaGetLastError();
}

// The externally visible launchers of one (T, FILT) variant, named by SUF.
#define ME_INSTANTIATE_ROUNDS(T, FILT, SUF)                                                      \
  int round_grid_##SUF(int which, int device) { return round_grid_impl<T, FILT>(which, device); } \
  cudaError_t launch_round_##SUF(const DevPlan &P, const InvertArgs &A, const Slots &S,          \
                                 int parity, const int grids[3], cudaStream_t st,                \
                                 cudaEvent_t *ev, int svd_lanes, const Overlap *ov) {            \
    return launch_round_impl<T, FILT>(P, A, S, parity, grids, st, ev, svd_lanes, ov);            \
  }                                                                                              \
  cudaError_t launch_round_grp_##SUF(int G, const DevPlan &P, const InvertArgs &A,               \
                                     const Slots &S, int parity, const int grids[3],             \
                                     cudaStream_t st, cudaEvent_t *ev, const Overlap *ov) {      \
    return launch_round_grp_impl<T, FILT>(G, P, A, S, parity, grids, st, ev, ov);                \
  }                                                                                              \
  cudaError_t launch_finish_##SUF(const DevPlan &P, const InvertArgs &A, const Slots &S,         \
                                  int *cursor, int grid, cudaStream_t st) {                      \
    return launch_finish_impl<T, FILT>(P, A, S, cursor, grid, st);                               \
  }

}  // namespace me

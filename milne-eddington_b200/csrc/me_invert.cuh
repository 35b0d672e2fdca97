// me_invert.cuh -- the inversion kernel (hot path), instantiated per precision
// by me_invert_f32.cu / me_invert_f64.cu.
//
// invert_kernel<T> is the hot path: a persistent kernel, one pixel per thread,
// each thread running the reference's INVERSION (Src/LM_FIT.c:665-742) as a
// flat state machine.  Every trip round the thread's loop performs exactly one
// LM trial step (SVD solve + forward synthesis + chi^2, Src/LM_FIT.c:473-527),
// preceded, only in lanes that need it, by a synthesis with the analytic
// Jacobian fused with the normal equations (Milne_Eddington_Single(Deriv) +
// Hessian_Compute, Src/ME_SOLVER.c:101-366 and Src/LM_FIT.c:240-350).  So the
// lanes of a warp stay in step on the dominant trial work whatever iteration,
// trial or restart each pixel is at.  A lane that finishes its pixel takes the
// next one from a global atomic counter: finished pixels leave the warp and
// restarts are queued in place, with no host round trip.
#pragma once

#include <cuda_runtime.h>

#include "me_device.cuh"
#include "me_kernels.h"

namespace me {

namespace detail {

template <class T>
__device__ __forceinline__ void load_voigt(VoigtK<T> &K, const DevPlan &P, T *s_tab) {
  K.a = T(P.fa);
  K.aa = T(P.faa);
  K.log_rmin0 = T(P.flog_rmin0);
  K.sqrt_log_rmin0 = T(P.fsqrt_log_rmin0);
  K.nmax = P.fnmax;
  K.nfig = P.nfigures;
#pragma unroll
  for (int i = 0; i < 5; i++) K.thr[i] = T(P.thr[i]);
  K.ea2n2 = s_tab;
}

template <class T>
__device__ __forceinline__ void fill_table(const DevPlan &P, T *s_tab) {
  for (int i = threadIdx.x; i < 50; i += blockDim.x) s_tab[i] = T(P.exp_a2n2[i]);
  __syncthreads();
}

// Synthesis with Jacobian fused with the weighted normal equations
// (Milne_Eddington_Single(Deriv=1) + Hessian_Compute + Loss_Function).
// sw[s] = weight_s / sqrt(norm0), so sum (J sw)(J sw) = J^T W J with
// W = weight^2 / norm0 (Noise_Init, Src/ME_SOLVER.c:410-441).
// H45 = upper triangle of the full 9x9 (row-major i <= j), g9 = -J^T W r,
// returns sum (r sw)^2 / (4 nl) accumulated in FP64.
template <class T>
__device__ __forceinline__ double deriv_pass(const DevPlan &P, const VoigtK<T> &K, const double *par,
                                             const double *step, const double *prof,
                                             const double sw[4], double *H45, double *g9) {
  SynthCall<T> c;
  synth_setup<T>(c, par, P, step);
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
    me_point<T, true>(c, shift_w<T>(c, P, iw), K, syn, J);
    T r[4];
#pragma unroll
    for (int s = 0; s < 4; s++) {
      const double rd = ((double)syn[s] - __ldg(prof + s * nl + iw)) * sw[s];
      chi += rd * rd;
      r[s] = T(rd);
#pragma unroll
      for (int k = 0; k < 9; k++) J[s][k] *= tsw[s];
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

// Forward synthesis + chi^2 (Trial_Synthesis's synthesis and Loss_Function);
// residuals and their squares accumulate in FP64.  fit (nullable) receives
// the synthetic profile.
template <class T>
__device__ __noinline__ double forward_pass(const DevPlan &P, const VoigtK<T> &K,
                                               const double *par, const double *step,
                                               const double *prof, const double sw[4],
                                               double *fit) {
  SynthCall<T> c;
  synth_setup<T>(c, par, P, step);
  double chi = 0.0;
  const int nl = P.nl;
#pragma unroll 1
  for (int iw = 0; iw < nl; iw++) {
    T syn[4];
    me_point<T, false>(c, shift_w<T>(c, P, iw), K, syn, nullptr);
#pragma unroll
    for (int s = 0; s < 4; s++) {
      if (prof) {
        const double rd = ((double)syn[s] - __ldg(prof + s * nl + iw)) * sw[s];
        chi += rd * rd;
      }
      if (fit) fit[s * nl + iw] = (double)syn[s];
    }
  }
  return chi / (4.0 * nl);
}

// Get_Regul (Src/LM_FIT.c:354-396) penalty part.
__device__ __forceinline__ double penalty_of(const DevPlan &P, const double *par) {
  double pen = 0.0;
  for (int i = 0; i < 9; i++) {
    if (P.fixed[i] || !P.regul[i]) continue;
    const double r = par[i] - P.regul_value[i];
    pen += r * r * P.regul_weight[i];
  }
  return pen;
}

enum : int { S_FETCH = 0, S_START = 1, S_NEXT = 2, S_TRIAL = 3, S_DONE = 4 };

}  // namespace detail

using namespace detail;

template <class T>
__global__ void __launch_bounds__(kInvertBlock, ME_INV_MINB) invert_kernel(const DevPlan P, InvertArgs A) {
  __shared__ T s_tab[50];
  fill_table<T>(P, s_tab);
  VoigtK<T> K;
  load_voigt<T>(K, P, s_tab);

  const int nl = P.nl;
  const int n = P.npar;
  double hess[81], vm[81];
  double jvec[9], sol[9];
  double par[9], ptmp[9], pbest[9], step[9];
  double sw[4];
  PixelInit pin;
  double chisq = 0, lmchisq = 0, ratio = 1, penalty = 0, damp = 0, chisq_best = 0;
  int run = 0, it = 0, state = S_FETCH;
  long long pix = -1;
  const double *pp = nullptr;
  unsigned int pc_runs = 0, pc_iter = 0, pc_trials = 0, pc_acc = 0;
  unsigned long long t_runs = 0, t_iter = 0, t_trials = 0, t_acc = 0, t_jac = 0, t_valid = 0,
                     t_svdlim = 0;
  bool had_trial = false;

  while (true) {
    // ---------------- take pixels until one needs inverting ----------------
    while (state == S_FETCH) {
      const unsigned long long k = atomicAdd(A.next, 1ULL);
      if (k >= (unsigned long long)A.count) {
        state = S_DONE;
        break;
      }
      pix = A.list ? A.list[k] : (long long)k;
      pp = A.prof + (size_t)pix * 4 * nl;
      const int bad = init_guess(pp, P, pin, true);  // also the INVERSION_MULTI gate
      if (bad || P.nruns <= 0) {
#pragma unroll
        for (int i = 0; i < 10; i++) A.res[(size_t)pix * 10 + i] = 0.0;
        if (A.fit)
          for (int i = 0; i < 4 * nl; i++) A.fit[(size_t)pix * 4 * nl + i] = 0.0;
        if (A.flags) A.flags[pix] = 0;
        continue;
      }
      t_valid++;
#pragma unroll
      for (int i = 0; i < 9; i++) step[i] = P.step[i];
      step[7] = pin.step7;
      const double isn = 1.0 / sqrt(pin.norm0);
#pragma unroll
      for (int s = 0; s < 4; s++) sw[s] = P.weights[s] * isn;
#pragma unroll
      for (int i = 0; i < 9; i++) par[i] = pin.guess[i];
      run = 0;
      lmchisq = A.stale ? A.stale[pix] : (pix == A.first_pixel ? A.carry : INFINITY);
      if (A.penalty0) A.penalty0[pix] = P.regul_any ? penalty_of(P, par) : 0.0;
      pc_runs = pc_iter = pc_trials = pc_acc = 0;
      had_trial = false;
      state = S_START;
    }
    if (state == S_DONE) break;

    // ------------- synthesis with Jacobian -> normal equations -------------
    bool end_run = false;
    if (state == S_START || state == S_NEXT) {
      double H45[45], g9[9];
      const double chi0 = deriv_pass<T>(P, K, par, step, pp, sw, H45, g9);
      t_jac++;
      if (state == S_START) {  // LM_FIT set-up (Src/LM_FIT.c:549-566)
        chisq = chi0;
        ratio = 1.0;
        if (P.regul_any) {
          penalty = penalty_of(P, par);
          if (penalty > 0.1 * lmchisq) ratio = 0.1 * chisq / penalty;
        }
        it = 0;
        end_run = (P.niter <= 0);
      }
      if (!end_run) {
        // Hessian_Compute's free-parameter block + Get_Regul(matrix)
        for (int a = 0; a < n; a++) {
          const int ia = P.free_idx[a];
          for (int b = a; b < n; b++) {
            const int ib = P.free_idx[b];
            const int idx = ia * 9 - ia * (ia + 1) / 2 + ib;  // (ia <= ib)
            hess[a * n + b] = H45[idx];
            hess[b * n + a] = H45[idx];
          }
          jvec[a] = g9[ia];
        }
        if (P.regul_any) {
          for (int a = 0; a < n; a++) {
            const int ia = P.free_idx[a];
            if (!P.regul[ia]) continue;
            const double r = par[ia] - P.regul_value[ia];
            jvec[a] -= r * P.regul_weight[ia] * ratio;
            hess[a * n + a] += P.regul_weight[ia] * ratio;
          }
        }
        pc_iter++;
        damp = P.damp;
        state = S_TRIAL;
      }
    }

    if (!end_run && state == S_TRIAL) {
      // ---------------- one trial step (Trial_Synthesis) ----------------
      t_svdlim += svd_solve(hess, vm, jvec, n, P.svd_thr, sol);
#pragma unroll
      for (int i = 0; i < 9; i++) ptmp[i] = par[i];
      for (int a = 0; a < n; a++) {
        const int ia = P.free_idx[a];
        ptmp[ia] += sol[a] * step[ia];
      }
      bounds_fold(ptmp, P, pin.l70, pin.l71);
      const double chi_new = forward_pass<T>(P, K, ptmp, step, pp, sw, nullptr);
      lmchisq = chi_new;
      had_trial = true;
      pc_trials++;
      if (P.regul_any) penalty = penalty_of(P, ptmp);
      if (chi_new < chisq) {  // accept (Src/LM_FIT.c:591-615)
        if (P.regul_any && penalty > 0.1 * lmchisq) ratio = 0.1 * chisq / penalty;
#pragma unroll
        for (int i = 0; i < 9; i++) par[i] = ptmp[i];
        pc_acc++;
        const bool conv = ((chisq - chi_new) / chisq) < P.convg;
        chisq = chi_new;
        it++;
        if (conv || it >= P.niter)
          end_run = true;
        else
          state = S_NEXT;
      } else {  // reject: grow the damping; past its limit the run ends
        damp *= P.lam_reject;
        if (damp > P.lam_lim[1]) end_run = true;
      }
    }

    if (end_run) {
      // ---------------- end of one LM_FIT run (INVERSION) ----------------
      const double chisq_run = chisq / pin.normp;
      pc_runs++;
      if (chisq_run < P.chisq_crit || run == 0 || chisq_run < chisq_best) {
#pragma unroll
        for (int i = 0; i < 9; i++) pbest[i] = par[i];
        chisq_best = chisq_run;
      }
      bool stop = false;
      if (chisq_run < P.chisq_crit && (run >= 4 || run == P.nruns * 4)) stop = true;
      if (run >= P.nruns * 2 && chisq_best < P.chisq_crit * 2) stop = true;
      run++;
      if (!stop && run < P.nruns * 4) {
        // Random_Jump (Src/LM_FIT.c:157-201)
        if (run < 4) {
#pragma unroll
          for (int i = 0; i < 9; i++) par[i] = pbest[i];
          par[2] = pin.guess[2] + kPi / 4. * run;
        } else {
          double z[8];
          restart_draws(P.seed, pix, run, z);
          const double *g = pin.guess;
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
        bounds_fold(par, P, pin.l70, pin.l71);
        state = S_START;
      } else {
        // pixel done: best-fit profile, theta fold, HMI_REF (Src/LM_FIT.c:727-733, 791-799)
        if (A.fit) forward_pass<T>(P, K, pbest, step, nullptr, sw, A.fit + (size_t)pix * 4 * nl);
        if (pbest[1] > kPi) pbest[1] -= kPi;
        if (P.hmi_ref) {
          pbest[2] += 0.5 * kPi;
          if (pbest[2] > kPi) pbest[2] -= kPi;
        }
        double *r = A.res + (size_t)pix * 10;
#pragma unroll
        for (int i = 0; i < 9; i++) r[i] = pbest[i];
        r[9] = chisq_best;
        if (A.flags) A.flags[pix] = 1 | (had_trial ? 2 : 0);
        if (A.lastchi) A.lastchi[pix] = lmchisq;
        if (A.counters) {
          uint4 c4 = make_uint4(pc_runs, pc_iter, pc_trials, pc_acc);
          reinterpret_cast<uint4 *>(A.counters)[pix] = c4;
        }
        t_runs += pc_runs;
        t_iter += pc_iter;
        t_trials += pc_trials;
        t_acc += pc_acc;
        state = S_FETCH;
      }
    }
  }
  if (A.totals) {
    atomicAdd(A.totals + 0, t_valid);
    atomicAdd(A.totals + 1, t_runs);
    atomicAdd(A.totals + 2, t_iter);
    atomicAdd(A.totals + 3, t_trials);
    atomicAdd(A.totals + 4, t_acc);
    atomicAdd(A.totals + 5, t_jac);
    atomicAdd(A.totals + 6, t_svdlim);
  }
}

}  // namespace me

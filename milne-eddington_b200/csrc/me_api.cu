// me_api.cu -- host side of the C ABI (include/me_b200.h): plans, batches,
// and the unit entry points.  No CPU compute path: every entry point that
// computes runs CUDA kernels and fails with ME_ERR_NODEVICE without a GPU.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <string>
#include <functional>
#include <vector>

#include "../../include/me_b200.h"
#include "me_kernels.h"

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

#define CK(call)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return fail(ME_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));      \
  } while (0)

int check_device(int device) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
    return fail(ME_ERR_NODEVICE, "no CUDA device visible: this library has no CPU path");
  if (device < 0 || device >= n) return fail(ME_ERR_ARG, "device index out of range");
  CK(cudaSetDevice(device));
  return ME_OK;
}

// Device buffer that grows on demand.
struct DevBuf {
  void *p = nullptr;
  size_t n = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= n) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e == cudaSuccess) n = bytes;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  template <class T>
  T *as() const {
    return static_cast<T *>(p);
  }
};

// A DevBuf that frees its memory when the scope ends, on every return path
// (the unit entry points' staging buffers; CK returns early on an error).
struct ScopedBuf : DevBuf {
  ScopedBuf() = default;
  ScopedBuf(const ScopedBuf &) = delete;
  ScopedBuf &operator=(const ScopedBuf &) = delete;
  ~ScopedBuf() { release(); }
};

// Alg-916 constants of Faddeeva_init (Src/FADDEEVA.c:406-436) and the region
// row of the accuracy table (Src/FADDEEVA.c:471-477).
void fill_voigt_consts(me::DevPlan &P, int nfigures) {
  static const double T[5][5] = {{1.6e4, 160.0, 107.0, 28.5, 3.5},
                                 {1.5e5, 510.0, 110.0, 39., -0.1},
                                 {1.451e6, 1.6e3, 180.0, 110.0, -0.1},
                                 {1.5e7, 5.01e3, 380.0, 115.0, 114.0},
                                 {1.3e8, 1.6e4, 810.0, 195.0, 116.0}};
  P.nfigures = nfigures;
  const double rmin0 = pow(10., -nfigures);
  P.fa = M_PI / sqrt(-log(0.5 * rmin0));
  P.faa = P.fa * P.fa;
  P.flog_rmin0 = -log(rmin0);
  P.fsqrt_log_rmin0 = sqrt(P.flog_rmin0);
  P.fnmax = 50;
  P.row = nfigures > 4 ? nfigures - 4 : 0;
  P.exp_a2n2[0] = 1.;
  for (int i = 1; i < 50; i++) P.exp_a2n2[i] = exp(-P.faa * i * i);
  for (int i = 0; i < 5; i++) P.thr[i] = T[P.row][i];
}

}  // namespace

struct me_plan {
  me_config cfg;
  me::DevPlan P;
  me_plan_facts facts;
  int device = 0;
  int precision = ME_PREC_FP32;
  int grid = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double carry = 0.0;  // LM->chisq carried between pixels (STRUCT_LM LM = {0})
  DevBuf d_lambda, d_dlambda;
  DevBuf d_flambda, d_fdlambda;  // instrument filter sub-wavelengths
  std::vector<double> h_lambda;  // the observed grid
  DevBuf d_prof, d_res, d_fit;  // staging of the host entry point
  DevBuf d_flags, d_pen0, d_lastchi, d_counters, d_totals, d_next, d_stale, d_list, d_fitpar;
  // slots of the pixels in flight (struct me::Slots), sized for `window`
  int window = 0;          // requested slot count (0 = default)
  int slots_w = 0;         // allocated slot count
  DevBuf d_slot_pix, d_slot_i32, d_slot_cnt, d_slot_u8, d_slot_sc, d_slot_vec, d_slot_hess,
      d_slot_list, d_slot_small;
  // the slot-major copy of the slots' observed profiles (me::Slots::obs;
  // me_plan_set_slot_profiles), sized for obs_w slots
  int slot_obs = 0;
  int obs_w = 0;
  DevBuf d_slot_obs;
  int grid_jac = 0, grid_trial = 0, grid_svd = 0, grid_fin = 0;
  // pixels in flight at or below which, with the queue empty, the tail kernel
  // finishes the batch (-1: half a wave of its warps; 0: rounds only)
  int tail_slots = -1;
  // largest lane group per slot in the rounds once the queue is empty (1: one
  // thread per slot throughout)
  int max_group = 32;
  bool use_graphs = true;  // rounds between polls as one CUDA graph launch
  // the later-trial SVDs run on a second stream beside the Jacobian kernel
  bool overlap = true;
  cudaStream_t stream2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  int svd_lanes = 1;  // lanes per matrix of the SVD launches in the full rounds
  long long finish_launches = 0;  // tail-kernel launches of the current batch
  // per-kernel device time (me_plan_set_profiling): events recorded around
  // every launch of a batch, read when it ends
  bool profile = false;
  std::vector<cudaEvent_t> evpool;
  size_t ev_used = 0;
  std::vector<std::pair<int, size_t>> ev_marks;  // (kind, first event): 0 = round, 1 = tail
  unsigned long long tail_start_totals[8] = {};
  bool tail_seen = false;
  int poll_rounds = 8;     // rounds launched between checks of the queue
  // once the queue is empty: rounds between checks, and how many lanes each
  // pixel in flight gets -- the most (a power of two, at most max_group) for
  // which pixels x lanes stay within group_fill half waves of the Jacobian
  // kernel (me_plan_set_drain)
  int drain_poll = 4;
  int group_fill = 4;
  unsigned long long *h_poll = nullptr;  // pinned: next, busy
  long long rounds_last = 0;
  std::vector<unsigned char> h_flags;
  std::vector<double> h_pen0, h_lastchi, h_stale, h_used;
  std::vector<long long> h_list;
  me_mlp *init = nullptr;  // learned initialiser (not owned), or null
  DevBuf d_init;           // [npix][9] its guesses for the current batch
  // with a learned start, queue the pixels by descending misfit of their
  // start (me_plan_set_queue_order): keys, histograms and the order
  bool queue_order = true;
  DevBuf d_okey, d_ohist, d_order;
  // the host entry point's chunked copy of a map in page-locked memory,
  // overlapped with the inversion (me_plan_set_feed): the copy stream, the
  // stream that makes each chunk's learned guesses and queue order, the
  // device count of queue positions that have arrived and its host values
  bool feed = true;
  cudaStream_t copy_stream = nullptr, prep_stream = nullptr;
  DevBuf d_avail;
  unsigned long long *h_feed = nullptr;  // pinned, kMaxFeedChunks
  std::vector<cudaEvent_t> feed_events;
  // with a learned start and the queue order, the queue's untaken part is
  // re-sorted globally once the whole map has arrived (me_plan_set_feed 2:
  // chunk order only); its scratch
  bool feed_resort = true;
  bool resort_pending = false;
  DevBuf d_tkey, d_tval, d_perm;
  // the queue checks of the last batch (me_plan_poll_trace) and its start
  std::vector<me_poll_record> trace;
  std::chrono::steady_clock::time_point trace_t0;
};

// chunks of the host entry point's overlapped copy (at most)
constexpr int kMaxFeedChunks = 64;

extern "C" const char *me_version(void) { return "me_b200 0.1 (sm_100a)"; }

extern "C" const char *me_last_error(void) { return g_last_error.c_str(); }

extern "C" const char *me_strerror(int status) {
  switch (status) {
    case ME_OK: return "ok";
    case ME_ERR_ARG: return "invalid argument";
    case ME_ERR_CONFIG: return "invalid control file";
    case ME_ERR_IO: return "I/O error";
    case ME_ERR_CUDA: return "CUDA error";
    case ME_ERR_NODEVICE: return "no CUDA device (no CPU fallback)";
    case ME_ERR_TIMEOUT: return "device work exceeded its budget";
    case ME_ERR_NOMEM: return "out of memory";
    case ME_ERR_FORMAT: return "unsupported file format";
    default: return "unknown status";
  }
}

namespace me {

int record_error(int code, const char *msg) { return fail(code, msg); }

void gaussian_filter(double fwhm, int points, std::vector<double> &off, std::vector<double> &w);

// The plan constants INIT_INV derives (Src/INV_INIT.c:112-201) from a parsed
// control file and a wavelength grid; P.lambda / P.dlambda are left null.
int build_devplan(const me_config *cfg, const double *lambda, int nl, DevPlan &P) {
  if (!cfg || !lambda) return fail(ME_ERR_ARG, "null argument");
  if (nl < 4 || nl > ME_MAX_NL) return fail(ME_ERR_ARG, "nl must be in [4, 512]");
  if (cfg->nline < 1) return fail(ME_ERR_CONFIG, "no spectral line (keyword lines)");
  if (cfg->nfigures > 8) return fail(ME_ERR_CONFIG, "Nfigures above 8 has no accuracy row");
  // the trial loop of an LM iteration ends only when the damping passes its
  // upper limit (Src/LM_FIT.c:144-150)
  if (!(cfg->damp > 0) || !(cfg->lambda_reject > 1) || !isfinite(cfg->lambda_limits[1]))
    return fail(ME_ERR_CONFIG, "damp must be > 0, lambda_reject > 1, lambda_limits finite");
  memset(&P, 0, sizeof(P));
  const double lam0 = cfg->line_lambda0[0];
  P.nl = nl;
  P.lambda0 = lam0;
  P.bshift = 4.6686e-10 * cfg->line_geff[0] * lam0 * lam0;
  P.npar = 0;
  for (int i = 0; i < 9; i++) {
    P.fixed[i] = cfg->fixed[i] ? 1 : 0;
    if (!P.fixed[i]) P.free_idx[P.npar++] = i;
    P.limits[i][0] = cfg->bounds[i][0];
    P.limits[i][1] = cfg->bounds[i][1];
    P.step[i] = cfg->step[i];
    P.regul[i] = cfg->regul[i] ? 1 : 0;
    P.regul_value[i] = cfg->regul_value[i];
    P.regul_weight[i] = cfg->regul_weight[i];
  }
  if (P.npar == 0) return fail(ME_ERR_CONFIG, "all nine parameters are fixed");
  // measured defaults on a B200 (the autotuner may choose others): the
  // shared-memory SVD; on the FP32 path the Jacobian kernel with its sums in
  // shared memory
  P.svd_regs = 0;
  P.kvar = 0;
  P.faddeeva = cfg->precision == ME_PREC_FP32 ? 1 : 0;
  P.fastg = cfg->precision == ME_PREC_FP32 ? 1 : 0;
  P.ncut = nl / 5;
  const double c = 299792458.0;
  double t = (lambda[P.ncut] - lam0) * c / 1e3;  // the reference omits /lambda0 here
  if (P.limits[3][0] < t) P.limits[3][0] = t;
  t = (lambda[nl - 1 - P.ncut] - lam0) * c / 1e3;
  if (P.limits[3][1] > t) P.limits[3][1] = t;
  // line-centre index by the reference's boolean arithmetic (Src/INV_INIT.c:150-156):
  // in practice the last iw < nl-1 with lambda[iw] < lambda0; 0 when none.
  P.ic = 0;
  for (int iw = 0; iw < nl - 1; iw++) {
    const double t1 = lam0 > lambda[iw];
    const double t2 = lambda[iw + 1] * lam0;
    if (t1 > 0 && t2 > 0) P.ic = t1 < t2 ? iw : iw + 1;
  }
  int r1 = 2, r2 = 2;
  if (P.ic - P.ncut >= 2) r1 = P.ic - P.ncut;
  if (nl - 1 - P.ncut - P.ic >= 2) r2 = nl - 1 - P.ncut - P.ic;
  int range = r1 > r2 ? r1 : r2;
  P.i0 = P.ic - range;
  if (P.i0 < 0) {
    P.i0 = 0;
    range = P.ic - P.i0;
  }
  P.i1 = P.ic + range;
  if (P.i1 > nl - 1) {
    P.i1 = nl - 1;
    range = P.i1 - P.ic;
    P.i0 = P.ic - range;
  }
  for (int s = 0; s < 4; s++) {
    P.weights[s] = cfg->weights[s];
    P.w2[s] = cfg->weights[s] * cfg->weights[s];
  }
  P.icriteria = cfg->icriteria;
  P.convg = cfg->convg_criteria;
  P.chisq_crit = cfg->chisq_criteria;
  P.damp = cfg->damp;
  P.lam_accept = cfg->lambda_accept;
  P.lam_reject = cfg->lambda_reject;
  P.lam_lim[0] = cfg->lambda_limits[0];
  P.lam_lim[1] = cfg->lambda_limits[1];
  P.svd_thr = cfg->svd_threshold;
  P.vcoeffi = cfg->vcoeffi;
  P.lcoeffi = cfg->lcoeffi;
  P.niter = cfg->num_iter;
  P.nruns = cfg->num_run;
  // the LM's trials end only when the damping outgrows its limit, and every
  // loop on the device is bounded by these (slot_step_cap)
  if (!(P.lam_reject >= 1.5 && P.lam_accept >= 1.5 && P.lam_reject < 1e300))
    return fail(ME_ERR_CONFIG, "lambda_accept and lambda_reject should be larger than 1.5");
  if (!(P.damp > 0 && P.damp < 1e300 && P.lam_lim[1] > 0 && P.lam_lim[1] < 1e300))
    return fail(ME_ERR_CONFIG, "damp and lambda_limits must be positive and finite");
  if (P.niter < 0 || P.niter > 100000 || P.nruns < 0 || P.nruns > 100000)
    return fail(ME_ERR_CONFIG, "num_iter and num_run must lie in [0, 100000]");
  P.hmi_ref = cfg->hmi_ref ? 1 : 0;
  P.regul_any = cfg->regul_any ? 1 : 0;
  P.seed = cfg->rng_seed;
  fill_voigt_consts(P, cfg->nfigures);
  P.nsub = 1;
  if (cfg->filter_fwhm > 0 && cfg->filter_points > 1) {
    if (cfg->filter_points > ME_MAX_FILTER || cfg->filter_points % 2 == 0)
      return fail(ME_ERR_CONFIG, "filter needs an odd number of points up to 63");
    std::vector<double> off, w;
    gaussian_filter(cfg->filter_fwhm, cfg->filter_points, off, w);
    P.nsub = cfg->filter_points;
    for (int k = 0; k < P.nsub; k++) P.sub_w[k] = w[k];
  }
  return ME_OK;
}

// The table of the `filter` keyword: `points` offsets [mA] uniform over +-1.5
// FWHM, weights exp(-d^2 / 2 sigma^2) normalised to sum 1.
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

}  // namespace me

namespace {
// Sub-wavelengths and weights of an instrument filter on the plan's device.
int set_filter_grid(me_plan *p, const double *off_mA, const double *w, int k) {
  me::DevPlan &P = p->P;
  const int nl = P.nl;
  if (k <= 1) {
    P.nsub = 1;
    P.flambda = P.fdlambda = nullptr;
    return ME_OK;
  }
  std::vector<double> fl((size_t)nl * k), fdl((size_t)nl * k);
  for (int i = 0; i < nl; i++)
    for (int q = 0; q < k; q++) {
      fl[(size_t)i * k + q] = p->h_lambda[i] + off_mA[q] * 1e-3;
      fdl[(size_t)i * k + q] = fl[(size_t)i * k + q] - P.lambda0;
    }
  const size_t bytes = sizeof(double) * fl.size();
  if (p->d_flambda.ensure(bytes) || p->d_fdlambda.ensure(bytes) ||
      cudaMemcpy(p->d_flambda.p, fl.data(), bytes, cudaMemcpyHostToDevice) ||
      cudaMemcpy(p->d_fdlambda.p, fdl.data(), bytes, cudaMemcpyHostToDevice))
    return fail(ME_ERR_CUDA, "filter grid allocation failed");
  P.nsub = k;
  for (int q = 0; q < k; q++) P.sub_w[q] = w[q];
  P.flambda = p->d_flambda.as<double>();
  P.fdlambda = p->d_fdlambda.as<double>();
  return ME_OK;
}
}  // namespace

extern "C" int me_plan_set_filter(me_plan *p, const double *offsets_mA, const double *weights,
                                  int k) {
  if (!p || k < 1 || k > ME_MAX_FILTER || (k > 1 && (!offsets_mA || !weights)))
    return fail(ME_ERR_ARG, "filter: 1 <= k <= ME_MAX_FILTER offsets and weights");
  CK(cudaSetDevice(p->device));
  return set_filter_grid(p, offsets_mA, weights, k);
}

// a non-blocking stream at the device's highest priority (returns nonzero on
// failure, like the CUDA calls it sits among)
static cudaError_t create_priority_stream(cudaStream_t *s) {
  int lo = 0, hi = 0;
  cudaError_t e = cudaDeviceGetStreamPriorityRange(&lo, &hi);
  if (e != cudaSuccess) return e;
  return cudaStreamCreateWithPriority(s, cudaStreamNonBlocking, hi);
}

extern "C" int me_plan_create(const me_config *cfg, const double *lambda, int nl, int device,
                              me_plan **out) {
  if (!cfg || !lambda || !out) return fail(ME_ERR_ARG, "null argument");
  *out = nullptr;
  me::DevPlan P0;
  int st = me::build_devplan(cfg, lambda, nl, P0);
  if (st) return st;
  st = check_device(device);
  if (st) return st;

  me_plan *p = new me_plan();
  p->cfg = *cfg;
  p->device = device;
  p->precision = cfg->precision == ME_PREC_FP64 ? ME_PREC_FP64 : ME_PREC_FP32;
  me::DevPlan &P = p->P;
  P = P0;
  const double lam0 = P.lambda0;
  std::vector<double> dl(nl);
  for (int i = 0; i < nl; i++) dl[i] = lambda[i] - lam0;
  if (p->d_lambda.ensure(sizeof(double) * nl) || p->d_dlambda.ensure(sizeof(double) * nl) ||
      p->d_totals.ensure(sizeof(unsigned long long) * 8) ||
      p->d_next.ensure(sizeof(unsigned long long)) ||
      cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) ||
      cudaStreamCreateWithFlags(&p->stream2, cudaStreamNonBlocking) ||
      cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking) ||
      create_priority_stream(&p->prep_stream) ||
      cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming) ||
      cudaEventCreateWithFlags(&p->ev_join, cudaEventDisableTiming) ||
      cudaEventCreate(&p->ev0) || cudaEventCreate(&p->ev1) ||
      cudaMemcpy(p->d_lambda.p, lambda, sizeof(double) * nl, cudaMemcpyHostToDevice) ||
      cudaMemcpy(p->d_dlambda.p, dl.data(), sizeof(double) * nl, cudaMemcpyHostToDevice)) {
    me_plan_destroy(p);
    return fail(ME_ERR_CUDA, "plan allocation failed");
  }
  P.lambda = p->d_lambda.as<double>();
  P.dlambda = p->d_dlambda.as<double>();
  p->h_lambda.assign(lambda, lambda + nl);
  if (P.nsub > 1) {
    std::vector<double> off, w;
    me::gaussian_filter(cfg->filter_fwhm, cfg->filter_points, off, w);
    const int rc = set_filter_grid(p, off.data(), w.data(), P.nsub);
    if (rc) {
      me_plan_destroy(p);
      return rc;
    }
  }
  p->grid_jac = me::round_grid(p->precision, 0, device);
  p->grid_trial = me::round_grid(p->precision, 1, device);
  p->grid_svd = me::round_grid(p->precision, 2, device);
  p->grid_fin = me::round_grid(p->precision, 3, device);
  p->grid = p->grid_trial;
  if (cudaMallocHost((void **)&p->h_poll, 2 * sizeof(unsigned long long)) != cudaSuccess ||
      cudaMallocHost((void **)&p->h_feed, kMaxFeedChunks * sizeof(unsigned long long)) !=
          cudaSuccess) {
    me_plan_destroy(p);
    return fail(ME_ERR_CUDA, "pinned allocation failed");
  }

  me_plan_facts &f = p->facts;
  f.nl = nl;
  f.ncut = P.ncut;
  f.ic = P.ic;
  f.i0 = P.i0;
  f.i1 = P.i1;
  f.npar = P.npar;
  f.bshift = P.bshift;
  memcpy(f.limits, P.limits, sizeof(f.limits));
  f.fadd_a = P.fa;
  *out = p;
  return ME_OK;
}

extern "C" void me_plan_destroy(me_plan *p) {
  if (!p) return;
  cudaSetDevice(p->device);
  DevBuf *bufs[] = {&p->d_lambda, &p->d_dlambda, &p->d_prof,     &p->d_res,
                    &p->d_fit,    &p->d_flags,   &p->d_pen0,     &p->d_lastchi,
                    &p->d_counters, &p->d_totals, &p->d_next,    &p->d_stale,
                    &p->d_list,   &p->d_slot_pix, &p->d_slot_i32, &p->d_slot_cnt,
                    &p->d_slot_u8, &p->d_slot_sc, &p->d_slot_vec, &p->d_slot_hess,
                    &p->d_slot_list, &p->d_slot_small, &p->d_fitpar, &p->d_init,
                    &p->d_flambda, &p->d_fdlambda, &p->d_okey, &p->d_ohist, &p->d_order,
                    &p->d_avail, &p->d_tkey, &p->d_tval, &p->d_perm};
  for (DevBuf *b : bufs) b->release();
  if (p->h_poll) cudaFreeHost(p->h_poll);
  if (p->h_feed) cudaFreeHost(p->h_feed);
  for (cudaEvent_t e : p->feed_events) cudaEventDestroy(e);
  if (p->copy_stream) cudaStreamDestroy(p->copy_stream);
  if (p->prep_stream) cudaStreamDestroy(p->prep_stream);
  if (p->ev0) cudaEventDestroy(p->ev0);
  if (p->ev1) cudaEventDestroy(p->ev1);
  for (cudaEvent_t e : p->evpool) cudaEventDestroy(e);
  if (p->stream) cudaStreamDestroy(p->stream);
  if (p->stream2) cudaStreamDestroy(p->stream2);
  if (p->ev_fork) cudaEventDestroy(p->ev_fork);
  if (p->ev_join) cudaEventDestroy(p->ev_join);
  delete p;
}

extern "C" int me_plan_get_facts(const me_plan *p, me_plan_facts *out) {
  if (!p || !out) return ME_ERR_ARG;
  *out = p->facts;
  return ME_OK;
}

extern "C" double me_plan_get_carry_chisq(const me_plan *p) { return p ? p->carry : 0.0; }
extern "C" void me_plan_set_carry_chisq(me_plan *p, double v) {
  if (p) p->carry = v;
}

extern "C" int me_plan_grid(const me_plan *p) { return p ? p->grid : 0; }
extern "C" void me_plan_set_grid(me_plan *p, int grid) {
  if (p && grid > 0) p->grid = grid;
}

extern "C" int me_plan_window(const me_plan *p) { return p ? p->window : 0; }
extern "C" void me_plan_set_window(me_plan *p, int window) {
  if (p && window >= 0) p->window = window;
}

extern "C" void me_plan_set_profiling(me_plan *p, int on) {
  if (p) p->profile = on != 0;
}

extern "C" int me_plan_last_counters(const me_plan *p, unsigned int *counters, long npix) {
  if (!p || !counters || npix < 0) return fail(ME_ERR_ARG, "null argument");
  if ((size_t)npix * 4 * sizeof(unsigned int) > p->d_counters.n)
    return fail(ME_ERR_ARG, "more pixels than the last batch had");
  CK(cudaSetDevice(p->device));
  CK(cudaMemcpy(counters, p->d_counters.p, (size_t)npix * 4 * sizeof(unsigned int),
                cudaMemcpyDeviceToHost));
  return ME_OK;
}

extern "C" void me_plan_set_overlap(me_plan *p, int on) {
  if (p) p->overlap = on != 0;
}

extern "C" void me_plan_set_queue_order(me_plan *p, int on) {
  if (p) p->queue_order = on != 0;
}

extern "C" int me_order_by_key(int device, const unsigned char *keys, long n, long long *order) {
  if (n < 0 || (n > 0 && (!keys || !order))) return fail(ME_ERR_ARG, "null argument");
  for (long i = 0; i < n; i++)
    if (keys[i] >= me::kOrderBuckets) return fail(ME_ERR_ARG, "keys must be below 128");
  if (n == 0) return ME_OK;
  int nd = 0;
  if (cudaGetDeviceCount(&nd) != cudaSuccess || nd == 0)
    return fail(ME_ERR_NODEVICE, "no CUDA device");
  if (device < 0 || device >= nd) return fail(ME_ERR_ARG, "device out of range");
  CK(cudaSetDevice(device));
  ScopedBuf dk, dh, dord;
  CK(dk.ensure((size_t)n));
  CK(dh.ensure((size_t)me::kOrderBuckets * me::kOrderBlocks * sizeof(int)));
  CK(dord.ensure((size_t)n * sizeof(long long)));
  CK(cudaMemcpy(dk.p, keys, (size_t)n, cudaMemcpyHostToDevice));
  CK(me::launch_order_by_key(dk.as<unsigned char>(), n, dh.as<int>(), dord.as<long long>(), nullptr));
  CK(cudaDeviceSynchronize());
  CK(cudaMemcpy(order, dord.p, (size_t)n * sizeof(long long), cudaMemcpyDeviceToHost));
  return ME_OK;
}

extern "C" void me_plan_set_graphs(me_plan *p, int on) {
  if (p) p->use_graphs = on != 0;
}

extern "C" int me_plan_poll_trace(const me_plan *p, me_poll_record *out, int cap) {
  if (!p) return 0;
  const int n = (int)p->trace.size();
  if (out)
    for (int i = 0; i < n && i < cap; i++) out[i] = p->trace[i];
  return n;
}

extern "C" int me_plan_svd_lanes(const me_plan *p) { return p ? p->svd_lanes : 0; }
extern "C" int me_plan_svd_registers(const me_plan *p) { return p ? p->P.svd_regs : 0; }
extern "C" int me_plan_kernel_variant(const me_plan *p) { return p ? p->P.kvar : 0; }
extern "C" void me_plan_set_kernel_variant(me_plan *p, int v) {
  if (p) p->P.kvar = (v >= 0 && v < me::kKernelVariants) ? v : 0;
}
extern "C" int me_plan_faddeeva(const me_plan *p) { return p ? p->P.faddeeva : 0; }
extern "C" void me_plan_set_faddeeva(me_plan *p, int mode) {
  if (p) p->P.faddeeva = (mode == 1 && p->precision == ME_PREC_FP32) ? 1 : 0;
}
extern "C" void me_plan_set_slot_profiles(me_plan *p, int on) {
  if (p) p->slot_obs = on != 0 ? 1 : 0;
}
extern "C" int me_plan_givens(const me_plan *p) { return p ? p->P.fastg : 0; }
extern "C" void me_plan_set_givens(me_plan *p, int mode) {
  if (p) p->P.fastg = (mode == 1 && p->precision == ME_PREC_FP32) ? 1 : 0;
}
extern "C" void me_weideman16(float *coef, float *L) {
#define ME_WEID_COPY(n, c) \
  if (coef) coef[n] = c;
  ME_WEIDEMAN16(ME_WEID_COPY)
#undef ME_WEID_COPY
  if (L) *L = ME_WEIDEMAN16_L;
}
extern "C" void me_plan_set_svd_registers(me_plan *p, int mode) {
  if (p) p->P.svd_regs = mode <= 0 ? 0 : (mode >= 2 ? 2 : 1);
}
extern "C" void me_plan_set_svd_lanes(me_plan *p, int lanes) {
  if (p) p->svd_lanes = lanes >= 8 ? 8 : lanes >= 4 ? 4 : lanes >= 2 ? 2 : 1;
}

extern "C" int me_plan_max_group(const me_plan *p) { return p ? p->max_group : 0; }
extern "C" void me_plan_set_max_group(me_plan *p, int lanes) {
  if (!p) return;
  int g = 1;
  while (g * 2 <= lanes && g < 32) g *= 2;
  p->max_group = g;
}

extern "C" void me_plan_set_drain(me_plan *p, int group_fill, int poll_rounds) {
  if (!p) return;
  p->group_fill = group_fill < 1 ? 1 : (group_fill > 8 ? 8 : group_fill);
  const int r = poll_rounds < 2 ? 2 : (poll_rounds > 64 ? 64 : poll_rounds);
  p->drain_poll = r & ~1;  // even: a captured batch of rounds starts at parity 0
}
extern "C" void me_plan_get_drain(const me_plan *p, int *group_fill, int *poll_rounds) {
  if (group_fill) *group_fill = p ? p->group_fill : 0;
  if (poll_rounds) *poll_rounds = p ? p->drain_poll : 0;
}

extern "C" int me_plan_tail_slots(const me_plan *p) { return p ? p->tail_slots : 0; }
extern "C" void me_plan_set_tail_slots(me_plan *p, int slots) {
  if (p) p->tail_slots = slots < 0 ? -1 : slots;
}

extern "C" int me_plan_set_initializer(me_plan *p, me_mlp *mlp) {
  if (!p) return fail(ME_ERR_ARG, "null plan");
  if (mlp) {
    int nl = 0;
    const int rc = me_mlp_shape(mlp, &nl, nullptr, nullptr);
    if (rc) return rc;
    if (nl != p->P.nl)
      return fail(ME_ERR_ARG, "initialiser trained for a grid of another size");
  }
  p->init = mlp;
  return ME_OK;
}

namespace me {
int plan_devplan(const me_plan *p, DevPlan *out, int *device) {
  if (!p || !out || !device) return fail(ME_ERR_ARG, "null argument");
  *out = p->P;
  *device = p->device;
  return ME_OK;
}
}  // namespace me

namespace {

// Grows the slot buffers to W slots and returns the device view.
int ensure_slots(me_plan *p, int W, me::Slots &S) {
  if (W > p->slots_w) {
    const size_t w = (size_t)W;
    CK(p->d_slot_pix.ensure(w * sizeof(long long)));
    CK(p->d_slot_i32.ensure(4 * w * sizeof(int)));
    CK(p->d_slot_cnt.ensure(4 * w * sizeof(unsigned int)));
    CK(p->d_slot_u8.ensure(w));
    CK(p->d_slot_sc.ensure((size_t)me::SC_COUNT * w * sizeof(double)));
    CK(p->d_slot_vec.ensure(5 * 9 * w * sizeof(double)));
    CK(p->d_slot_hess.ensure(81 * w * sizeof(double)));
    CK(p->d_slot_list.ensure(4 * w * sizeof(int)));
    CK(p->d_slot_small.ensure(8 * sizeof(int)));
    p->slots_w = W;
  }
  const size_t w = (size_t)W;
  S.W = W;
  S.pix = p->d_slot_pix.as<long long>();
  int *i32 = p->d_slot_i32.as<int>();
  S.state = i32;
  S.run = i32 + w;
  S.it = i32 + 2 * w;
  S.tk = i32 + 3 * w;
  S.cnt = p->d_slot_cnt.as<unsigned int>();
  S.had_trial = p->d_slot_u8.as<unsigned char>();
  S.sc = p->d_slot_sc.as<double>();
  double *v = p->d_slot_vec.as<double>();
  S.guess = v;
  S.par = v + 9 * w;
  S.pbest = v + 18 * w;
  S.jvec = v + 27 * w;
  S.ptmp = v + 36 * w;
  S.hess = p->d_slot_hess.as<double>();
  S.jlist = p->d_slot_list.as<int>();
  S.rlist = S.jlist + 2 * w;
  int *small = p->d_slot_small.as<int>();
  S.jcount = small;
  S.rcount = small + 2;
  S.busy = small + 4;
  S.obs = nullptr;
  if (p->slot_obs) {
    if (W > p->obs_w) {
      CK(p->d_slot_obs.ensure(w * 4 * (size_t)p->P.nl * sizeof(double)));
      p->obs_w = W;
    }
    S.obs = p->d_slot_obs.as<double>();
  }
  return ME_OK;
}

// n consecutive events from the plan's pool (profiling only).
cudaEvent_t *take_events(me_plan *p, size_t n) {
  while (p->evpool.size() < p->ev_used + n) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    p->evpool.push_back(e);
  }
  cudaEvent_t *ev = p->evpool.data() + p->ev_used;
  p->ev_used += n;
  return ev;
}

void trace_poll(me_plan *p, long long rounds, long long next, int busy, int group) {
  const std::chrono::duration<double, std::milli> t =
      std::chrono::steady_clock::now() - p->trace_t0;
  p->trace.push_back({t.count(), rounds, next, busy, group});
}

// Runs one queue (A.count items) to completion: rounds of jac_kernel,
// svd_kernel and trial_kernel on the plan's slots while the queue feeds them,
// then, once it is empty and at most tail_slots pixels remain, finish_kernel
// (one warp per pixel, no per-round launches) for the rest.
int run_queue(me_plan *p, const me::InvertArgs &A, cudaStream_t st, long long &rounds,
              cudaEvent_t feed_done = nullptr) {
  const long long cap = p->window > 0 ? p->window : 131072;
  const int W = (int)(A.count < cap ? A.count : cap);
  if (W <= 0) return ME_OK;
  me::Slots S;
  int rc = ensure_slots(p, W, S);
  if (rc) return rc;
  CK(cudaMemsetAsync(S.state, 0, (size_t)W * sizeof(int), st));  // SL_EMPTY
  CK(cudaMemsetAsync(S.jcount, 0, 5 * sizeof(int), st));           // jcount[2], rcount[2], busy
  CK(cudaMemsetAsync(A.next, 0, sizeof(unsigned long long), st));
  int grids[3];
  grids[0] = std::min(p->grid_jac, (W + me::kBlock - 1) / me::kBlock);
  grids[1] = std::min(p->grid_trial, (W + me::kBlock - 1) / me::kBlock);
  grids[2] = p->svd_lanes > 1
                 ? (int)std::min<long long>(p->grid_trial,
                                            ((long long)W * p->svd_lanes + me::kBlock - 1) / me::kBlock)
                 : std::min(p->grid_svd, (W + me::kSvdBlock - 1) / me::kSvdBlock);
  int parity = 0;
  int group = 1;              // lanes per slot of the next rounds
  int ggrids[3] = {1, 1, 1};  // their grids
  // executable graphs of poll_rounds rounds: index 0 one thread per slot,
  // 1..5 lane groups of 2..32; they hold this queue's arguments, so they live
  // for this call only
  cudaGraphExec_t graphs[6] = {};
  // a group size's first rounds in this queue run as direct launches, so
  // that every kernel a graph holds has run (and been loaded) before its
  // capture; a capture that fails all the same falls back to direct launches
  // for the rest of the queue
  bool ran_direct[6] = {};
  bool graphs_ok = true;
  auto group_index = [](int g) {
    int i = 0;
    while (g > 1) {
      g >>= 1;
      i++;
    }
    return i;
  };
  auto release_graphs = [&]() {
    for (cudaGraphExec_t &x : graphs)
      if (x) {
        cudaGraphExecDestroy(x);
        x = nullptr;
      }
  };
  struct GraphGuard {
    std::function<void()> f;
    ~GraphGuard() { f(); }
  } graph_guard{release_graphs};
  rounds = 0;
  // every slot step is one round: a bound no valid batch reaches
  const double round_cap = (double)me::slot_step_cap(p->P) * (double)((A.count + W - 1) / W + 1);
  // with a feed (A.avail), slots may hold queue positions that have not
  // arrived (SL_WAIT); the queue counts as drained only after a batch of full
  // rounds that started once the last position had arrived (its trial
  // kernels took every held position up)
  bool fed = feed_done == nullptr;
  while (true) {
    if ((double)rounds > round_cap)
      return fail(ME_ERR_TIMEOUT, "inversion rounds exceeded their bound");
    bool fed_before = fed;
    if (!fed_before) {
      const cudaError_t q = cudaEventQuery(feed_done);
      if (q == cudaSuccess) {
        fed_before = true;
      } else if (q == cudaErrorNotReady) {
        cudaGetLastError();  // not an error: clear it
      } else {
        return fail(ME_ERR_CUDA, std::string("feed: ") + cudaGetErrorString(q));
      }
    }
    // the rounds between two polls: one CUDA graph per lane-group size,
    // captured once per queue on the plan's stream (an even number of rounds
    // starts every batch at parity 0), or direct launches when profiling
    me::Overlap ov_storage{p->stream2, p->ev_fork, p->ev_join};
    const me::Overlap *ov = (p->overlap && !p->profile) ? &ov_storage : nullptr;
    const int gi = group_index(group);
    const int nr = group > 1 ? p->drain_poll : p->poll_rounds;
    cudaGraphExec_t *gx =
        (graphs_ok && ran_direct[gi] && p->use_graphs && !p->profile && nr % 2 == 0)
            ? &graphs[gi]
            : nullptr;
    ran_direct[gi] = true;
    if (gx && !*gx) {
      cudaGraph_t g = nullptr;
      CK(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
      cudaError_t e = cudaSuccess;
      for (int r = 0; r < nr && e == cudaSuccess; r++)
        e = group > 1 ? me::launch_round_grp(p->precision, group, p->P, A, S, r & 1, ggrids,
                                             p->stream, nullptr, ov)
                      : me::launch_round(p->precision, p->P, A, S, r & 1, grids, p->stream,
                                         nullptr, p->svd_lanes, ov);
      const cudaError_t e2 = cudaStreamEndCapture(p->stream, &g);
      if (e == cudaSuccess) e = e2;
      if (e == cudaSuccess) e = cudaGraphInstantiate(gx, g, 0);
      if (g) cudaGraphDestroy(g);
      if (e != cudaSuccess) {
        // nothing captured ran; clear the capture's error and launch directly
        cudaGetLastError();
        release_graphs();
        graphs_ok = false;
        gx = nullptr;
      }
    }
    if (gx) {
      const cudaError_t e = cudaGraphLaunch(*gx, st);
      if (e != cudaSuccess) {
        release_graphs();
        return fail(ME_ERR_CUDA, std::string("round graph launch: ") + cudaGetErrorString(e));
      }
      rounds += nr;
    } else {
      for (int r = 0; r < nr; r++) {
        cudaEvent_t *ev = nullptr;
        if (p->profile) {
          const size_t first = p->ev_used;
          ev = take_events(p, 5);
          if (ev) p->ev_marks.push_back({0, first});
        }
        if (group > 1)
          CK(me::launch_round_grp(p->precision, group, p->P, A, S, parity, ggrids, st, ev, ov));
        else
          CK(me::launch_round(p->precision, p->P, A, S, parity, grids, st, ev, p->svd_lanes,
                              ov));
        parity ^= 1;
        rounds++;
      }
    }
    CK(cudaMemcpyAsync(p->h_poll, A.next, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(p->h_poll + 1, S.busy, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const int busy = *reinterpret_cast<int *>(p->h_poll + 1);
    trace_poll(p, rounds, (long long)p->h_poll[0], busy, group);
    if (fed_before) fed = true;
    if (fed && p->resort_pending) {
      // the whole map is on the device and the stream is idle: the queue
      // positions not taken yet go into the global misfit order
      p->resort_pending = false;
      const long long first = (long long)p->h_poll[0];
      if (first < A.count && A.list)
        CK(me::launch_resort_tail(const_cast<long long *>(A.list), first, A.count - first,
                                  p->d_okey.as<unsigned char>(), p->d_tkey.as<unsigned char>(),
                                  p->d_tval.as<long long>(), p->d_ohist.as<int>(),
                                  p->d_perm.as<long long>(), st));
    }
    const bool drained = p->h_poll[0] >= (unsigned long long)A.count && fed;
    if (drained && busy == 0) break;
    if (drained && p->max_group > 1) {
      // the queue is empty: give each slot in flight as many lanes as fill
      // group_fill half waves of the Jacobian kernel on the whole device
      const long long wave = (long long)p->grid_jac * me::kBlock;
      int g = 1;
      while (g < p->max_group && (long long)busy * g * 2 <= wave * p->group_fill) g *= 2;
      group = g;
      const long long need = ((long long)W * g + me::kBlock - 1) / me::kBlock;
      ggrids[0] = (int)std::min<long long>(p->grid_jac, need);
      ggrids[1] = (int)std::min<long long>(p->grid_trial, need);
      ggrids[2] = (int)std::min<long long>(p->grid_trial, need);
    }
    // default: half a wave of the tail kernel's warps
    const int tail = p->tail_slots < 0 ? p->grid_fin * (me::kBlock / 32) / 2 : p->tail_slots;
    if (drained && busy <= tail) {
      // the queue is empty and few pixels remain: one warp per pixel to the end
      int *cursor = S.busy + 1;
      CK(cudaMemsetAsync(cursor, 0, sizeof(int), st));
      const int g = std::min(p->grid_fin, (busy + me::kBlock / 32 - 1) / (me::kBlock / 32));
      cudaEvent_t *ev = nullptr;
      if (p->profile) {
        // event counts the rounds did, to attribute the rest to the tail
        CK(cudaMemcpyAsync(p->tail_start_totals, A.totals, sizeof(p->tail_start_totals),
                           cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        p->tail_seen = true;
        const size_t first = p->ev_used;
        ev = take_events(p, 2);
        if (ev) {
          p->ev_marks.push_back({1, first});
          CK(cudaEventRecord(ev[0], st));
        }
      }
      CK(me::launch_finish(p->precision, p->P, A, S, cursor, std::max(g, 1), st));
      if (ev) CK(cudaEventRecord(ev[1], st));
      trace_poll(p, rounds, (long long)p->h_poll[0], busy, 0);
      p->finish_launches++;
      break;
    }
  }
  return ME_OK;
}

}  // namespace

namespace {

// A map that the host entry point is still copying in (me_invert_batch): the
// queue positions below *avail are on the device; `done` is recorded once
// the last has arrived.  With a learned start the feed also made each chunk's
// guesses (plan d_init) and, with the queue order, its order (plan d_order,
// sorted within the chunk); init_ms is their device time.
struct Feed {
  const unsigned long long *avail;
  cudaEvent_t done;
  float init_ms;
};

int invert_impl(me_plan *p, const double *d_prof, long npix, double *d_res, double *d_fit,
                cudaStream_t st, me_stats *stats, const Feed *feed) {
  if (stats) memset(stats, 0, sizeof(*stats));
  if (npix == 0) return ME_OK;
  const size_t n = (size_t)npix;
  CK(p->d_flags.ensure(n));
  CK(p->d_pen0.ensure(n * sizeof(double)));
  CK(p->d_lastchi.ensure(n * sizeof(double)));
  CK(p->d_counters.ensure(n * 4 * sizeof(unsigned int)));
  CK(cudaMemsetAsync(p->d_totals.p, 0, 8 * sizeof(unsigned long long), st));

  me::InvertArgs A;
  memset(&A, 0, sizeof(A));
  A.prof = d_prof;
  A.res = d_res;
  A.fit = d_fit;
  if (d_fit) {
    CK(p->d_fitpar.ensure(n * 9 * sizeof(double)));
    A.fitpar = p->d_fitpar.as<double>();
  }
  A.flags = p->d_flags.as<unsigned char>();
  A.penalty0 = p->d_pen0.as<double>();
  A.lastchi = p->d_lastchi.as<double>();
  A.counters = p->d_counters.as<unsigned int>();
  A.totals = p->d_totals.as<unsigned long long>();
  A.next = p->d_next.as<unsigned long long>();
  A.list = nullptr;
  A.count = npix;
  A.stale = nullptr;
  A.carry = p->carry;
  A.first_pixel = 0;
  A.avail = feed ? feed->avail : nullptr;
  float init_ms = 0.f;
  if (p->init && feed) {
    // guesses and order came with the chunks (me_invert_batch)
    A.init_par = p->d_init.as<double>();
    if (p->queue_order) A.list = p->d_order.as<long long>();
  } else if (p->init) {
    CK(p->d_init.ensure(n * 9 * sizeof(double)));
    CK(cudaEventRecord(p->ev0, st));
    const int rc = me_mlp_predict_device(p->init, d_prof, npix, p->d_init.as<double>(), st);
    if (rc) return rc;
    CK(cudaEventRecord(p->ev1, st));
    CK(cudaEventSynchronize(p->ev1));
    cudaEventElapsedTime(&init_ms, p->ev0, p->ev1);
    const int grc = me::mlp_gemm_status(p->init);
    if (grc) return grc;
    A.init_par = p->d_init.as<double>();
    if (p->queue_order) {
      CK(p->d_okey.ensure(n));
      CK(p->d_ohist.ensure((size_t)me::kOrderBuckets * me::kOrderBlocks * sizeof(int)));
      CK(p->d_order.ensure(n * sizeof(long long)));
      CK(cudaEventRecord(p->ev0, st));
      CK(me::launch_start_order(p->precision, p->P, d_prof, A.init_par, npix,
                            p->d_okey.as<unsigned char>(), p->d_ohist.as<int>(),
                            p->d_order.as<long long>(), st));
      CK(cudaEventRecord(p->ev1, st));
      CK(cudaEventSynchronize(p->ev1));
      float order_ms = 0.f;
      cudaEventElapsedTime(&order_ms, p->ev0, p->ev1);
      init_ms += order_ms;
      A.list = p->d_order.as<long long>();
    }
  }

  long long rounds = 0, rounds_total = 0;
  p->finish_launches = 0;
  p->ev_used = 0;
  p->ev_marks.clear();
  p->tail_seen = false;
  p->trace.clear();
  p->trace_t0 = std::chrono::steady_clock::now();
  CK(cudaEventRecord(p->ev0, st));
  int rc = run_queue(p, A, st, rounds, feed ? feed->done : nullptr);
  if (rc) return rc;
  CK(cudaEventRecord(p->ev1, st));
  rounds_total += rounds;
  if (p->init && feed) {
    const int grc = me::mlp_gemm_status(p->init);
    if (grc) return grc;
    init_ms = feed->init_ms;
  }

  // The reference carries LM->chisq from pixel to pixel; it enters only the
  // first regularisation ratio test of each pixel (Src/LM_FIT.c:555-559).  The
  // batch above assumed the carried value for pixel 0 and "no ratio change"
  // for every later pixel; pixels for which the true carried value (the last
  // trial chi^2 of the previous inverted pixel) flips that test are re-run,
  // until no flip remains.
  p->h_flags.resize(n);
  p->h_pen0.resize(n);
  p->h_lastchi.resize(n);
  CK(cudaMemcpyAsync(p->h_flags.data(), A.flags, n, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(p->h_lastchi.data(), A.lastchi, n * sizeof(double), cudaMemcpyDeviceToHost,
                     st));
  if (p->P.regul_any)
    CK(cudaMemcpyAsync(p->h_pen0.data(), A.penalty0, n * sizeof(double), cudaMemcpyDeviceToHost,
                       st));
  CK(cudaStreamSynchronize(st));
  trace_poll(p, rounds, npix, 0, -1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, p->ev0, p->ev1);
  double kernel_ms = ms;
  long long redo_total = 0, passes = 1;
  p->h_used.assign(n, INFINITY);
  p->h_used[0] = p->carry;
  while (true) {
    for (size_t i = 0; i < n; i++)
      if (p->h_flags[i] & 8) return fail(ME_ERR_TIMEOUT, "a pixel exceeded its LM step bound");
    double prev = p->carry;
    p->h_list.clear();
    for (size_t i = 0; i < n; i++) {
      if (!(p->h_flags[i] & 1)) continue;
      if (p->P.regul_any) {
        const bool want = p->h_pen0[i] > 0.1 * prev;
        const bool used = p->h_pen0[i] > 0.1 * p->h_used[i];
        if (want != used) {
          p->h_list.push_back((long long)i);
          p->h_used[i] = prev;
        }
      }
      if (p->h_flags[i] & 2) prev = p->h_lastchi[i];
    }
    if (p->h_list.empty()) {
      p->carry = prev;
      break;
    }
    redo_total += (long long)p->h_list.size();
    passes++;
    const size_t m = p->h_list.size();
    CK(p->d_list.ensure(m * sizeof(long long)));
    CK(p->d_stale.ensure(n * sizeof(double)));
    CK(cudaMemcpyAsync(p->d_list.p, p->h_list.data(), m * sizeof(long long),
                       cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(p->d_stale.p, p->h_used.data(), n * sizeof(double), cudaMemcpyHostToDevice,
                       st));
    me::InvertArgs B = A;
    B.list = p->d_list.as<long long>();
    B.count = (long long)m;
    B.stale = p->d_stale.as<double>();
    B.avail = nullptr;  // the whole map is on the device by now
    CK(cudaEventRecord(p->ev0, st));
    rc = run_queue(p, B, st, rounds);
    if (rc) return rc;
    CK(cudaEventRecord(p->ev1, st));
    rounds_total += rounds;
    CK(cudaMemcpyAsync(p->h_flags.data(), A.flags, n, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(p->h_lastchi.data(), A.lastchi, n * sizeof(double),
                       cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    cudaEventElapsedTime(&ms, p->ev0, p->ev1);
    kernel_ms += ms;
  }
  if (d_fit)
    CK(me::launch_fit(p->precision, p->P, A.fitpar, A.flags, npix, d_fit, st));
  p->rounds_last = rounds_total;
  if (stats) {
    unsigned long long tot[8];
    CK(cudaMemcpy(tot, A.totals, sizeof(tot), cudaMemcpyDeviceToHost));
    stats->pixels = npix;
    stats->valid = (long long)tot[0];
    stats->runs = (long long)tot[1];
    stats->iterations = (long long)tot[2];
    stats->trials = (long long)tot[3];
    stats->accepted = (long long)tot[4];
    stats->syntheses = (long long)tot[3];
    stats->jacobians = (long long)tot[5];
    stats->wavelengths = (long long)(tot[3] + tot[5]) * p->P.nl;
    stats->redo_pixels = redo_total;
    stats->launches = 4 * rounds_total + p->finish_launches + (d_fit ? 1 : 0) +
                      (p->init ? me::kMlpPredLaunches *
                                     ((npix + me::kMlpPredChunk - 1) / me::kMlpPredChunk)
                               : 0);
    stats->rounds = rounds_total;
    stats->kernel_ms = kernel_ms;
    stats->init_ms = init_ms;
    stats->learned_done = (long long)tot[7];
    if (p->profile) {
      // per-kernel device time from the events of every launch of the batch
      for (const auto &m : p->ev_marks) {
        cudaEvent_t *e = p->evpool.data() + m.second;
        float t = 0.f;
        if (m.first == 0) {
          cudaEventElapsedTime(&t, e[0], e[1]);
          stats->jac_ms += t;
          cudaEventElapsedTime(&t, e[1], e[3]);
          stats->svd_ms += t;
          cudaEventElapsedTime(&t, e[3], e[4]);
          stats->trial_ms += t;
        } else {
          cudaEventElapsedTime(&t, e[0], e[1]);
          stats->tail_ms += t;
        }
      }
      if (p->tail_seen) {
        stats->tail_trials = (long long)(tot[3] - p->tail_start_totals[3]);
        stats->tail_jacobians = (long long)(tot[5] - p->tail_start_totals[5]);
      }
    }
  }
  return ME_OK;
}

// Pixels per chunk of the overlapped copy of an npix map (0: copy it whole).
// A multiple of 64 pixels, so that no 128-byte line of the profiles, the
// guesses or the queue order straddles two chunks.
long long feed_chunk(long long npix) {
  constexpr long long kMin = 65536;
  if (npix < 2 * kMin) return 0;
  long long c = (npix + 7) / 8;
  if (c < kMin) c = kMin;
  c = (c + 63) / 64 * 64;
  while ((npix + c - 1) / c > kMaxFeedChunks) c += 64;
  return c;
}

bool host_page_locked(const void *ptr) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// The copy of the map in chunks on the copy stream, each chunk announced to
// the rounds by raising *avail once it is on the device -- after, with a
// learned start, its guesses and its queue order (sorted within the chunk)
// were made on the priority stream -- so that the inversion starts on the
// first chunk while the rest is still on its way.  Fills f; the copy's own
// device time goes to *h2d_ms once the batch is over (events e0, e1).
int start_feed(me_plan *p, const double *prof, long long npix, long long chunk, Feed &f,
               cudaEvent_t e0, cudaEvent_t e1) {
  const long long nl = p->P.nl;
  const long long nch = (npix + chunk - 1) / chunk;
  const size_t n = (size_t)npix;
  const bool learned = p->init != nullptr;
  CK(p->d_avail.ensure(sizeof(unsigned long long)));
  p->resort_pending = false;
  if (learned) {
    CK(p->d_init.ensure(n * 9 * sizeof(double)));
    if (p->queue_order) {
      CK(p->d_okey.ensure(n));
      CK(p->d_ohist.ensure((size_t)me::kOrderBuckets * me::kOrderBlocks * sizeof(int)));
      CK(p->d_order.ensure(n * sizeof(long long)));
      if (p->feed_resort) {
        CK(p->d_tkey.ensure(n));
        CK(p->d_tval.ensure(n * sizeof(long long)));
        CK(p->d_perm.ensure(n * sizeof(long long)));
        p->resort_pending = true;
      }
    }
  }
  // events: start, feed done, and per chunk arrival + prep start/end
  const size_t need = 2 + 3 * (size_t)nch;
  while (p->feed_events.size() < need) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    p->feed_events.push_back(e);
  }
  cudaEvent_t ev_start = p->feed_events[0], ev_done = p->feed_events[1];
  unsigned long long *d_avail = p->d_avail.as<unsigned long long>();
  // avail = 0 before the rounds look at it; the feed streams start after that
  CK(cudaMemsetAsync(d_avail, 0, sizeof(unsigned long long), p->stream));
  CK(cudaEventRecord(ev_start, p->stream));
  CK(cudaStreamWaitEvent(p->copy_stream, ev_start, 0));
  if (learned) CK(cudaStreamWaitEvent(p->prep_stream, ev_start, 0));
  CK(cudaEventRecord(e0, p->copy_stream));
  double *d_prof = p->d_prof.as<double>();
  for (long long k = 0; k < nch; k++) {
    const long long s0 = k * chunk, s1 = std::min(npix, s0 + chunk);
    const size_t off = (size_t)s0 * 4 * nl;
    CK(cudaMemcpyAsync(d_prof + off, prof + off, (size_t)(s1 - s0) * 4 * nl * sizeof(double),
                       cudaMemcpyHostToDevice, p->copy_stream));
    p->h_feed[k] = (unsigned long long)s1;
    if (!learned) {
      // in order on the copy stream: the count rises after the chunk landed
      CK(cudaMemcpyAsync(d_avail, p->h_feed + k, sizeof(unsigned long long),
                         cudaMemcpyHostToDevice, p->copy_stream));
      continue;
    }
    cudaEvent_t arrived = p->feed_events[2 + 3 * k];
    cudaEvent_t pb = p->feed_events[3 + 3 * k], pe = p->feed_events[4 + 3 * k];
    CK(cudaEventRecord(arrived, p->copy_stream));
    CK(cudaStreamWaitEvent(p->prep_stream, arrived, 0));
    CK(cudaEventRecord(pb, p->prep_stream));
    double *d_init = p->d_init.as<double>() + (size_t)s0 * 9;
    const int rc = me_mlp_predict_device(p->init, d_prof + off, s1 - s0, d_init, p->prep_stream);
    if (rc) return rc;
    if (p->queue_order)
      CK(me::launch_start_order(p->precision, p->P, d_prof + off, d_init, s1 - s0,
                                p->d_okey.as<unsigned char>() + s0, p->d_ohist.as<int>(),
                                p->d_order.as<long long>() + s0, p->prep_stream, s0));
    CK(cudaEventRecord(pe, p->prep_stream));
    CK(cudaMemcpyAsync(d_avail, p->h_feed + k, sizeof(unsigned long long),
                       cudaMemcpyHostToDevice, p->prep_stream));
  }
  CK(cudaEventRecord(e1, p->copy_stream));
  CK(cudaEventRecord(ev_done, learned ? p->prep_stream : p->copy_stream));
  f.avail = d_avail;
  f.done = ev_done;
  f.init_ms = 0.f;
  return ME_OK;
}

// Device time of the feed's learned-start work (after the batch).
float feed_init_ms(me_plan *p, long long npix, long long chunk) {
  if (!p->init) return 0.f;
  float sum = 0.f;
  const long long nch = (npix + chunk - 1) / chunk;
  for (long long k = 0; k < nch; k++) {
    float t = 0.f;
    cudaEventElapsedTime(&t, p->feed_events[3 + 3 * k], p->feed_events[4 + 3 * k]);
    sum += t;
  }
  return sum;
}

}  // namespace

extern "C" int me_invert_batch_device(me_plan *p, const double *d_prof, long npix, double *d_res,
                                      double *d_fit, void *stream, me_stats *stats) {
  if (!p || !d_prof || !d_res || npix < 0) return fail(ME_ERR_ARG, "null argument");
  CK(cudaSetDevice(p->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : p->stream;
  return invert_impl(p, d_prof, npix, d_res, d_fit, st, stats, nullptr);
}

extern "C" void me_plan_set_feed(me_plan *p, int mode) {
  if (!p) return;
  p->feed = mode != 0;
  p->feed_resort = mode != 2;
}

extern "C" int me_invert_batch(me_plan *p, const double *prof, long npix, double *res, double *fit,
                               me_stats *stats) {
  if (!p || !prof || !res || npix < 0) return fail(ME_ERR_ARG, "null argument");
  if (npix == 0) {
    if (stats) memset(stats, 0, sizeof(*stats));
    return ME_OK;
  }
  CK(cudaSetDevice(p->device));
  const size_t n = (size_t)npix;
  const size_t pbytes = n * 4 * p->P.nl * sizeof(double);
  CK(p->d_prof.ensure(pbytes));
  CK(p->d_res.ensure(n * 10 * sizeof(double)));
  if (fit) CK(p->d_fit.ensure(pbytes));
  cudaEvent_t e0, e1, e2, e3;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventCreate(&e2);
  cudaEventCreate(&e3);
  // a map in page-locked memory goes in chunks that the inversion starts on
  // as they land; from pageable memory a copy cannot run beside the host's
  // launches, so it goes whole first
  const long long chunk = p->feed ? feed_chunk(npix) : 0;
  int rc = ME_OK;
  if (chunk > 0 && host_page_locked(prof)) {
    Feed f;
    rc = start_feed(p, prof, npix, chunk, f, e0, e1);
    if (rc == ME_OK)
      rc = invert_impl(p, p->d_prof.as<double>(), npix, p->d_res.as<double>(),
                       fit ? p->d_fit.as<double>() : nullptr, p->stream, stats, &f);
    if (rc == ME_OK && stats) {
      stats->init_ms = feed_init_ms(p, npix, chunk);
      CK(cudaStreamSynchronize(p->copy_stream));
    }
    if (rc != ME_OK) {  // leave no copy running into the plan's buffers
      cudaStreamSynchronize(p->copy_stream);
      cudaStreamSynchronize(p->prep_stream);
    }
  } else {
    cudaEventRecord(e0, p->stream);
    CK(cudaMemcpyAsync(p->d_prof.p, prof, pbytes, cudaMemcpyHostToDevice, p->stream));
    cudaEventRecord(e1, p->stream);
    rc = invert_impl(p, p->d_prof.as<double>(), npix, p->d_res.as<double>(),
                     fit ? p->d_fit.as<double>() : nullptr, p->stream, stats, nullptr);
  }
  if (rc == ME_OK) {
    cudaEventRecord(e2, p->stream);
    cudaError_t e = cudaMemcpyAsync(res, p->d_res.p, n * 10 * sizeof(double),
                                    cudaMemcpyDeviceToHost, p->stream);
    if (e == cudaSuccess && fit)
      e = cudaMemcpyAsync(fit, p->d_fit.p, pbytes, cudaMemcpyDeviceToHost, p->stream);
    cudaEventRecord(e3, p->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(p->stream);
    if (e != cudaSuccess) rc = fail(ME_ERR_CUDA, cudaGetErrorString(e));
    if (rc == ME_OK && stats) {
      float a = 0, b = 0;
      cudaEventElapsedTime(&a, e0, e1);
      cudaEventElapsedTime(&b, e2, e3);
      stats->h2d_ms = a;
      stats->d2h_ms = b;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaEventDestroy(e2);
  cudaEventDestroy(e3);
  return rc;
}

extern "C" int me_synthesize_jacobian(me_plan *p, const double *par, long npix, double step7,
                                      double *prof, double *jac) {
  if (!p || !par || !prof || npix < 0) return fail(ME_ERR_ARG, "null argument");
  if (npix == 0) return ME_OK;
  CK(cudaSetDevice(p->device));
  const size_t n = (size_t)npix, nl = (size_t)p->P.nl;
  ScopedBuf dp, dprof, djac;
  CK(dp.ensure(n * 9 * sizeof(double)));
  CK(dprof.ensure(n * 4 * nl * sizeof(double)));
  if (jac) CK(djac.ensure(n * 36 * nl * sizeof(double)));
  CK(cudaMemcpyAsync(dp.p, par, n * 9 * sizeof(double), cudaMemcpyHostToDevice, p->stream));
  CK(me::launch_synth(p->precision, p->P, dp.as<double>(), npix, step7, dprof.as<double>(),
                      jac ? djac.as<double>() : nullptr, p->stream));
  CK(cudaMemcpyAsync(prof, dprof.p, n * 4 * nl * sizeof(double), cudaMemcpyDeviceToHost,
                     p->stream));
  if (jac)
    CK(cudaMemcpyAsync(jac, djac.p, n * 36 * nl * sizeof(double), cudaMemcpyDeviceToHost,
                       p->stream));
  CK(cudaStreamSynchronize(p->stream));
  dp.release();
  dprof.release();
  djac.release();
  return ME_OK;
}

extern "C" int me_synthesize(me_plan *p, const double *par, long npix, double *prof) {
  return me_synthesize_jacobian(p, par, npix, p ? p->P.step[7] : 0.0, prof, nullptr);
}

extern "C" int me_synthesize_device(me_plan *p, const double *d_par, long npix, double *d_prof,
                                    void *stream) {
  if (!p || !d_par || !d_prof || npix < 0) return fail(ME_ERR_ARG, "null argument");
  CK(cudaSetDevice(p->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : p->stream;
  CK(me::launch_synth(p->precision, p->P, d_par, npix, p->P.step[7], d_prof, nullptr, st));
  if (!stream) CK(cudaStreamSynchronize(st));
  return ME_OK;
}

extern "C" int me_faddeeva(int nfigures, int precision, const double *nu, const double *a, long n,
                           double *H, double *L, int device) {
  if (!nu || !a || !H || !L || n < 0 || nfigures > 8) return fail(ME_ERR_ARG, "bad argument");
  int st = check_device(device);
  if (st) return st;
  if (n == 0) return ME_OK;
  me::DevPlan P;
  memset(&P, 0, sizeof(P));
  fill_voigt_consts(P, nfigures);
  ScopedBuf dn, da, dh, dl;
  const size_t b = (size_t)n * sizeof(double);
  CK(dn.ensure(b));
  CK(da.ensure(b));
  CK(dh.ensure(b));
  CK(dl.ensure(b));
  CK(cudaMemcpy(dn.p, nu, b, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(da.p, a, b, cudaMemcpyHostToDevice));
  CK(me::launch_voigt(precision == ME_PREC_FP64 ? 1 : 0, P, dn.as<double>(), da.as<double>(), n,
                      dh.as<double>(), dl.as<double>(), 0));
  CK(cudaMemcpy(H, dh.p, b, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(L, dl.p, b, cudaMemcpyDeviceToHost));
  dn.release();
  da.release();
  dh.release();
  dl.release();
  return ME_OK;
}

extern "C" int me_faddeeva_weideman(const double *nu, const double *a, long n, double *H,
                                    double *L, int device) {
  if (!nu || !a || !H || !L || n < 0) return fail(ME_ERR_ARG, "bad argument");
  int st = check_device(device);
  if (st) return st;
  if (n == 0) return ME_OK;
  me::DevPlan P;
  memset(&P, 0, sizeof(P));
  fill_voigt_consts(P, 6);
  P.faddeeva = 1;
  ScopedBuf dn, da, dh, dl;
  const size_t b = (size_t)n * sizeof(double);
  CK(dn.ensure(b));
  CK(da.ensure(b));
  CK(dh.ensure(b));
  CK(dl.ensure(b));
  CK(cudaMemcpy(dn.p, nu, b, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(da.p, a, b, cudaMemcpyHostToDevice));
  CK(me::launch_voigt(0, P, dn.as<double>(), da.as<double>(), n, dh.as<double>(),
                      dl.as<double>(), 0));
  CK(cudaMemcpy(H, dh.p, b, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(L, dl.p, b, cudaMemcpyDeviceToHost));
  return ME_OK;
}

extern "C" int me_svd(const double *a, long nmat, int n, double *u, double *w, double *v,
                      int device) {
  if (!a || !u || !w || !v || nmat < 0 || n < 1 || n > 9) return fail(ME_ERR_ARG, "bad argument");
  int st = check_device(device);
  if (st) return st;
  if (nmat == 0) return ME_OK;
  const size_t mb = (size_t)nmat * n * n * sizeof(double), wb = (size_t)nmat * n * sizeof(double);
  ScopedBuf da, du, dw, dv, dh;
  CK(da.ensure(mb));
  CK(du.ensure(mb));
  CK(dv.ensure(mb));
  CK(dw.ensure(wb));
  CK(dh.ensure(sizeof(int)));
  CK(cudaMemset(dh.p, 0, sizeof(int)));
  CK(cudaMemcpy(da.p, a, mb, cudaMemcpyHostToDevice));
  CK(me::launch_svd(da.as<double>(), nmat, n, du.as<double>(), dw.as<double>(), dv.as<double>(),
                    dh.as<int>(), 0));
  CK(cudaMemcpy(u, du.p, mb, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(v, dv.p, mb, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(w, dw.p, wb, cudaMemcpyDeviceToHost));
  da.release();
  du.release();
  dv.release();
  dw.release();
  dh.release();
  return ME_OK;
}

extern "C" int me_svd_u(const double *a, long nmat, int n, int lanes, int fast, double *u,
                        double *w, int *limit_hits, int device) {
  if (!a || !u || !w || nmat < 0 || n < 1 || n > 9) return fail(ME_ERR_ARG, "bad argument");
  if (lanes != 1 && lanes != 2 && lanes != 4 && lanes != 8 && lanes != 16 && lanes != 32)
    return fail(ME_ERR_ARG, "lanes must be 1, 2, 4, 8, 16 or 32");
  int st = check_device(device);
  if (st) return st;
  if (limit_hits) *limit_hits = 0;
  if (nmat == 0) return ME_OK;
  const size_t mb = (size_t)nmat * n * n * sizeof(double), wb = (size_t)nmat * n * sizeof(double);
  ScopedBuf da, du, dw, dh;
  CK(da.ensure(mb));
  CK(du.ensure(mb));
  CK(dw.ensure(wb));
  CK(dh.ensure(sizeof(int)));
  CK(cudaMemset(dh.p, 0, sizeof(int)));
  CK(cudaMemcpy(da.p, a, mb, cudaMemcpyHostToDevice));
  CK(me::launch_svd_u(da.as<double>(), nmat, n, lanes, fast ? 1 : 0, du.as<double>(),
                      dw.as<double>(), dh.as<int>(), 0));
  CK(cudaMemcpy(u, du.p, mb, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(w, dw.p, wb, cudaMemcpyDeviceToHost));
  if (limit_hits) CK(cudaMemcpy(limit_hits, dh.p, sizeof(int), cudaMemcpyDeviceToHost));
  da.release();
  du.release();
  dw.release();
  dh.release();
  return ME_OK;
}

extern "C" int me_init_guess(me_plan *p, const double *prof, long npix, double *guess,
                             double *extra, int *status) {
  if (!p || !prof || !guess || !extra || !status || npix < 0)
    return fail(ME_ERR_ARG, "null argument");
  if (npix == 0) return ME_OK;
  CK(cudaSetDevice(p->device));
  const size_t n = (size_t)npix, nl = (size_t)p->P.nl;
  ScopedBuf dp, dg, de, ds;
  CK(dp.ensure(n * 4 * nl * sizeof(double)));
  CK(dg.ensure(n * 9 * sizeof(double)));
  CK(de.ensure(n * 5 * sizeof(double)));
  CK(ds.ensure(n * sizeof(int)));
  CK(cudaMemcpyAsync(dp.p, prof, n * 4 * nl * sizeof(double), cudaMemcpyHostToDevice, p->stream));
  CK(me::launch_init_guess(p->P, dp.as<double>(), npix, dg.as<double>(), de.as<double>(),
                           ds.as<int>(), p->stream));
  CK(cudaMemcpyAsync(guess, dg.p, n * 9 * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
  CK(cudaMemcpyAsync(extra, de.p, n * 5 * sizeof(double), cudaMemcpyDeviceToHost, p->stream));
  CK(cudaMemcpyAsync(status, ds.p, n * sizeof(int), cudaMemcpyDeviceToHost, p->stream));
  CK(cudaStreamSynchronize(p->stream));
  dp.release();
  dg.release();
  de.release();
  ds.release();
  return ME_OK;
}

extern "C" int me_svd_device(const double *d_a, long nmat, int n, double *d_u, double *d_w,
                             double *d_v, void *stream) {
  if (!d_a || !d_u || !d_w || !d_v || nmat < 0 || n < 1 || n > 9)
    return fail(ME_ERR_ARG, "bad argument");
  cudaStream_t st = (cudaStream_t)stream;
  CK(me::launch_svd(d_a, nmat, n, d_u, d_w, d_v, nullptr, st));
  if (!stream) CK(cudaStreamSynchronize(st));
  return ME_OK;
}

extern "C" int me_svd_u_device(const double *d_a, long nmat, int n, int lanes, int fast,
                               double *d_u, double *d_w, void *stream) {
  if (!d_a || !d_u || !d_w || nmat < 0 || n < 1 || n > 9) return fail(ME_ERR_ARG, "bad argument");
  if (lanes != 1 && lanes != 2 && lanes != 4 && lanes != 8 && lanes != 16 && lanes != 32)
    return fail(ME_ERR_ARG, "lanes must be 1, 2, 4, 8, 16 or 32");
  cudaStream_t st = (cudaStream_t)stream;
  CK(me::launch_svd_u(d_a, nmat, n, lanes, fast ? 1 : 0, d_u, d_w, nullptr, st));
  if (!stream) CK(cudaStreamSynchronize(st));
  return ME_OK;
}

extern "C" int me_synthesize_jacobian_device(me_plan *p, const double *d_par, long npix,
                                             double step7, double *d_prof, double *d_jac,
                                             void *stream) {
  if (!p || !d_par || !d_prof || npix < 0) return fail(ME_ERR_ARG, "null argument");
  CK(cudaSetDevice(p->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : p->stream;
  CK(me::launch_synth(p->precision, p->P, d_par, npix, step7, d_prof, d_jac, st));
  if (!stream) CK(cudaStreamSynchronize(st));
  return ME_OK;
}

// ---------------------------------------------------------------------------
// Autotuner: a greedy coordinate search over the plan's runtime knobs, each
// candidate timed (CUDA events on the stream) on the caller's batch.
// ---------------------------------------------------------------------------
extern "C" int me_plan_autotune(me_plan *p, const double *d_prof, long npix, void *stream,
                                me_tune_result *out) {
  if (!p || !d_prof || npix <= 0) return fail(ME_ERR_ARG, "autotune needs a non-empty batch");
  CK(cudaSetDevice(p->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : p->stream;
  CK(p->d_res.ensure((size_t)npix * 10 * sizeof(double)));
  const double carry = p->carry;
  const bool prof = p->profile;
  p->profile = false;
  int trials = 0;
  auto run = [&](double &ms) -> int {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    p->carry = carry;
    cudaEventRecord(a, st);
    int rc = me_invert_batch_device(p, d_prof, npix, p->d_res.as<double>(), nullptr, st, nullptr);
    cudaEventRecord(b, st);
    if (!rc) rc = cudaEventSynchronize(b) == cudaSuccess ? ME_OK : fail(ME_ERR_CUDA, "autotune");
    float t = 0.f;
    cudaEventElapsedTime(&t, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    ms = t;
    trials++;
    return rc;
  };
  double best = 0.0;
  int rc = run(best);  // warm-up (buffers sized for the batch)
  if (!rc) rc = run(best);
  struct Knob {
    int *field;
    std::vector<int> cand;
  };
  const int w0 = p->window > 0 ? p->window : 131072;
  p->window = w0;  // the default made explicit, so the result names it
  std::vector<Knob> knobs = {
      {&p->window, {w0 / 2, w0, w0 * 2}},
      {&p->max_group, {1, 4, 8, 16, 32}},
      // the tail kernel's threshold: none, a quarter, half (the default), one
      // and two waves of its warps
      {&p->tail_slots,
       {0, p->grid_fin * (me::kBlock / 32) / 4, -1, p->grid_fin * (me::kBlock / 32),
        p->grid_fin * (me::kBlock / 32) * 2}},
      {&p->svd_lanes, {1, 2}},
      // the Jacobian / trial kernels' variant: 64, 128 or 256 pixels per CTA,
      // the wavelength grid staged in shared memory, no reciprocal table, the
      // normal-equation sums in shared memory
      {&p->P.kvar, {0, 1, 2, 3, 4, 5}},
      // the 9x9 SVD in registers in the full rounds, also in the lane-split
      // rounds, or in shared memory throughout (the default)
      {&p->P.svd_regs, {1, 2, 0}},
      // after the queue drains: lanes per pixel in flight (half a wave to four
      // waves of the Jacobian kernel) and rounds between checks
      {&p->group_fill, {1, 2, 4, 8}},
      {&p->drain_poll, {8, 4, 2}},
      // the FP32 syntheses' Faddeeva evaluation: the reference's regions and
      // Alg-916, or Weideman's series (FP64 plans keep the former)
      {&p->P.faddeeva, {0, p->precision == ME_PREC_FP32 ? 1 : 0}},
      // the observed profiles read from a slot-major copy made at refill
      {&p->slot_obs, {0, 1}},
  };
  for (Knob &k : knobs) {
    if (rc) break;
    int keep = *k.field;
    for (int c : k.cand) {
      if (c == keep) continue;
      const int old = *k.field;
      *k.field = c;
      double ms = 0.0;
      rc = run(ms);
      if (rc) break;
      if (ms < best) {
        best = ms;
        keep = c;
      } else {
        *k.field = old;
      }
    }
    *k.field = keep;
  }
  p->carry = carry;
  p->profile = prof;
  if (rc) return rc;
  if (out) {
    out->window = p->window;
    out->max_group = p->max_group;
    out->tail_slots = p->tail_slots;
    out->svd_lanes = p->svd_lanes;
    out->ms = best;
    out->trials = trials;
    out->kernel_variant = p->P.kvar;
    out->svd_registers = p->P.svd_regs;
    out->group_fill = p->group_fill;
    out->drain_poll = p->drain_poll;
    out->faddeeva = p->P.faddeeva;
    out->slot_profiles = p->slot_obs;
  }
  return ME_OK;
}

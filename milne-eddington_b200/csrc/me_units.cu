// me_units.cu -- unit kernels (synthesis, Voigt, SVD, initial guess) and the
// launch dispatch.  The inversion kernel itself lives in me_invert.cuh.
//
#include <cuda_runtime.h>

#include "me_device.cuh"
#include "me_kernels.h"

namespace me {

namespace {

}  // namespace

// ---------------------------------------------------------------------------
// Building blocks exposed for the unit entry points.
// ---------------------------------------------------------------------------

template <class T>
__global__ void synth_kernel(const DevPlan P, const double *par, long long npix, double step7,
                             double *prof, double *jac) {
  __shared__ T s_tab[100];
  __shared__ T s_rden[kRden * 128];
  VoigtK<T> K;
  voigt_block_setup<T>(K, P, s_tab);
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= npix) return;
  const int nl = P.nl;
  double step[9];
#pragma unroll
  for (int k = 0; k < 9; k++) step[k] = P.step[k];
  step[7] = step7;
  double mp[9];
#pragma unroll
  for (int k = 0; k < 9; k++) mp[k] = par[i * 9 + k];
  SynthCall<T> c;
  synth_setup<T>(c, mp, P, step);
  voigt_prepare<T>(K, c.p5, s_rden + threadIdx.x, blockDim.x);
  const T ones[4] = {T(1), T(1), T(1), T(1)};
  for (int iw = 0; iw < nl; iw++) {
    T syn[4], J[4][9];
    if (jac) {
      if (P.nsub > 1)
        channel_point<T, true, true>(c, P, K, ones, iw, syn, J);
      else
        channel_point<T, true, false>(c, P, K, ones, iw, syn, J);
      for (int s = 0; s < 4; s++)
        for (int k = 0; k < 9; k++) jac[((size_t)i * 36 + s * 9 + k) * nl + iw] = (double)J[s][k];
    } else if (P.nsub > 1) {
      channel_point<T, false, true>(c, P, K, ones, iw, syn, nullptr);
    } else {
      channel_point<T, false, false>(c, P, K, ones, iw, syn, nullptr);
    }
    for (int s = 0; s < 4; s++) prof[((size_t)i * 4 + s) * nl + iw] = (double)syn[s];
  }
}

template <class T>
__global__ void fit_kernel(const DevPlan P, const double *fitpar, const unsigned char *flags,
                           long long npix, double *fit) {
  __shared__ T s_tab[100];
  __shared__ T s_rden[kRden * 128];
  VoigtK<T> K;
  voigt_block_setup<T>(K, P, s_tab);
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= npix) return;
  const int nl = P.nl;
  double *out = fit + (size_t)i * 4 * nl;
  if (!(flags[i] & 1)) {
    for (int k = 0; k < 4 * nl; k++) out[k] = 0.0;
    return;
  }
  double mp[9];
#pragma unroll
  for (int k = 0; k < 9; k++) mp[k] = fitpar[i * 9 + k];
  SynthCall<T> c;
  synth_setup<T>(c, mp, P, P.step);
  voigt_prepare<T>(K, c.p5, s_rden + threadIdx.x, blockDim.x);
  const T ones[4] = {T(1), T(1), T(1), T(1)};
  for (int iw = 0; iw < nl; iw++) {
    T syn[4];
    if (P.nsub > 1)
      channel_point<T, false, true>(c, P, K, ones, iw, syn, nullptr);
    else
      channel_point<T, false, false>(c, P, K, ones, iw, syn, nullptr);
    for (int s = 0; s < 4; s++) out[s * nl + iw] = (double)syn[s];
  }
}

template <class T>
__global__ void voigt_kernel(const DevPlan P, const double *nu, const double *a, long long n,
                             double *H, double *L) {
  __shared__ T s_tab[100];
  __shared__ T s_rden[kRden * 256];
  VoigtK<T> K;
  voigt_block_setup<T>(K, P, s_tab);
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const T y = T(a[i]);
  voigt_prepare<T>(K, y, s_rden + threadIdx.x, blockDim.x);
  const HL<T> r = voigt<T>(T(nu[i]), y, erfcx_t<T>(y), K);
  H[i] = (double)r.h;
  L[i] = (double)r.l;
}

__global__ void svd_kernel(const double *a, long long nmat, int n, double *u, double *w,
                           double *v, int *limit_hits) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= nmat) return;
  double am[81], vv[81], ww[9];
  for (int k = 0; k < n * n; k++) am[k] = a[i * n * n + k];
  const int hit = gr_svd(am, n, ww, vv);
  for (int k = 0; k < n * n; k++) {
    u[i * n * n + k] = am[k];
    v[i * n * n + k] = vv[k];
  }
  for (int k = 0; k < n; k++) w[i * n + k] = ww[k];
  if (hit && limit_hits) atomicAdd(limit_hits, 1);
}

__global__ void init_guess_kernel(const DevPlan P, const double *prof, long long npix,
                                  double *guess, double *extra, int *status) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= npix) return;
  PixelInit o;
  const int st = init_guess(prof + (size_t)i * 4 * P.nl, P, o, false);
  status[i] = st;
  for (int k = 0; k < 9; k++) guess[i * 9 + k] = st ? 0.0 : o.guess[k];
  extra[i * 5 + 0] = st ? 0.0 : o.norm0;
  extra[i * 5 + 1] = st ? 0.0 : o.normp;
  extra[i * 5 + 2] = st ? 0.0 : o.l70;
  extra[i * 5 + 3] = st ? 0.0 : o.l71;
  extra[i * 5 + 4] = st ? 0.0 : o.step7;
}

// ---------------------------------------------------------------------------
// Queue order of a learned start.  A pixel whose start is far from its profile
// tends to need many LM iterations and restarts; queued late, it runs on alone
// at the end of the batch while the GPU idles.  The misfit of each pixel's
// start -- the run -1 parameters exactly as the queue sets them up (Init_Guess,
// the network's free parameters, the bounds fold) -- is Loss_Function's chi^2
// (Src/LM_FIT.c:150-156; weights / sqrt(norm0), Src/ME_SOLVER.c:410-441) on
// every `stride`-th wavelength.  Pixels are queued by descending misfit in
// quarter-octave buckets, by a stable counting sort, so the order, and with it
// every result, is reproducible.  A pixel's steps are the same in any order;
// which kernel runs each of them (full rounds, lane-split rounds, the tail
// kernel) depends on when it is queued, so results agree with pixel order to
// rounding.
// ---------------------------------------------------------------------------
template <class T, bool FILT>
__global__ void start_misfit_kernel(const DevPlan P, const double *prof, const double *init_par,
                                    long long npix, int stride, unsigned char *key) {
  __shared__ T s_tab[100];
  __shared__ T s_rden[kRden * 128];
  VoigtK<T> K;
  voigt_block_setup<T>(K, P, s_tab);
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= npix) return;
  const int nl = P.nl;
  const double *pp = prof + (size_t)i * 4 * nl;
  PixelInit pin;
  if (init_guess(pp, P, pin, true) || P.nruns <= 0) {
    key[i] = (unsigned char)(kOrderBuckets - 1);  // skipped by the queue: last
    return;
  }
  double q[9], step[9];
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const double v = init_par[(size_t)i * 9 + k];
    q[k] = (P.fixed[k] || !isfinite(v)) ? pin.guess[k] : v;
    step[k] = P.step[k];
  }
  bounds_fold(q, P, pin.l70, pin.l71);
  step[7] = pin.step7;
  const double isn = 1.0 / sqrt(pin.norm0);
  SynthCall<T> c;
  synth_setup<T>(c, q, P, step);
  voigt_prepare<T>(K, c.p5, s_rden + threadIdx.x, blockDim.x);
  const T ones[4] = {T(1), T(1), T(1), T(1)};
  double chi = 0.0;
  int used = 0;
  for (int iw = 0; iw < nl; iw += stride, used++) {
    T syn[4];
    channel_point<T, false, FILT>(c, P, K, ones, iw, syn, nullptr);
#pragma unroll
    for (int s = 0; s < 4; s++) {
      const double rd = ((double)syn[s] - pp[s * nl + iw]) * P.weights[s] * isn;
      chi += rd * rd;
    }
  }
  chi /= 4.0 * used;
  // bucket 0: chi^2 >= 2^32 or not finite; a quarter octave per bucket below,
  // down to bucket kOrderBuckets - 2 (chi^2 < 2^0.5 and all below)
  int b = 0;
  if (chi < 4294967296.0) {
    b = (int)floor((32.0 - log2(fmax(chi, 1e-300))) * 4.0);
    b = b < 0 ? 0 : (b > kOrderBuckets - 2 ? kOrderBuckets - 2 : b);
  }
  key[i] = (unsigned char)b;
}

// Stable counting sort of pixel indices by an 8-bit key, in three launches:
// per-block histograms of contiguous chunks (bucket-major), an exclusive scan
// of them, and a scatter in which each block walks its chunk in index order.
__global__ void order_hist_kernel(const unsigned char *key, long long n, long long chunk,
                                  int *hist) {
  __shared__ int h[kOrderBuckets];
  for (int t = threadIdx.x; t < kOrderBuckets; t += blockDim.x) h[t] = 0;
  __syncthreads();
  const long long lo = blockIdx.x * chunk;
  const long long hi = lo + chunk < n ? lo + chunk : n;
  for (long long i = lo + threadIdx.x; i < hi; i += blockDim.x) atomicAdd(&h[key[i]], 1);
  __syncthreads();
  for (int t = threadIdx.x; t < kOrderBuckets; t += blockDim.x)
    hist[(size_t)t * gridDim.x + blockIdx.x] = h[t];
}

// exclusive prefix sums of hist[0..m) in place; one block of 1024 threads
__global__ void __launch_bounds__(1024) order_scan_kernel(int *hist, int m) {
  __shared__ int part[1024];
  const int t = threadIdx.x;
  const int per = (m + 1023) / 1024;
  const int lo = t * per, hi = lo + per < m ? lo + per : m;
  int sum = 0;
  for (int i = lo; i < hi; i++) sum += hist[i];
  part[t] = sum;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {  // inclusive scan of the segment sums
    const int v = t >= o ? part[t - o] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int run = part[t] - sum;
  for (int i = lo; i < hi; i++) {
    const int v = hist[i];
    hist[i] = run;
    run += v;
  }
}

__global__ void __launch_bounds__(256) order_scatter_kernel(const unsigned char *key, long long n,
                                                            long long chunk, const int *offs,
                                                            long long *order, long long first) {
  __shared__ int base[kOrderBuckets];
  __shared__ int wcnt[8][kOrderBuckets];
  for (int t = threadIdx.x; t < kOrderBuckets; t += blockDim.x) {
    base[t] = offs[(size_t)t * gridDim.x + blockIdx.x];
    for (int w = 0; w < 8; w++) wcnt[w][t] = 0;
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long lo = blockIdx.x * chunk;
  const long long hi = lo + chunk < n ? lo + chunk : n;
  for (long long r0 = lo; r0 < hi; r0 += 256) {
    const long long i = r0 + threadIdx.x;
    const bool in = i < hi;
    const int k = in ? (int)key[i] : kOrderBuckets + lane;  // absent lanes match nobody
    const unsigned peers = __match_any_sync(0xffffffffu, k);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    const bool leader = lane == __ffs(peers) - 1;
    if (in && leader) wcnt[warp][k] = __popc(peers);
    __syncthreads();
    if (in) {
      int pos = base[k] + rank;
      for (int w = 0; w < warp; w++) pos += wcnt[w][k];
      order[pos] = first + i;
    }
    __syncthreads();
    if (in && leader) {
      atomicAdd(&base[k], __popc(peers));
      wcnt[warp][k] = 0;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------

#define ME_DECLARE_ROUNDS(SUF)                                                                   \
  int round_grid_##SUF(int which, int device);                                                  \
  cudaError_t launch_round_##SUF(const DevPlan &P, const InvertArgs &A, const Slots &S,          \
                                 int parity, const int grids[3], cudaStream_t st,                \
                                 cudaEvent_t *ev, int svd_lanes, const Overlap *ov);             \
  cudaError_t launch_round_grp_##SUF(int G, const DevPlan &P, const InvertArgs &A,               \
                                     const Slots &S, int parity, const int grids[3],             \
                                     cudaStream_t st, cudaEvent_t *ev, const Overlap *ov);       \
  cudaError_t launch_finish_##SUF(const DevPlan &P, const InvertArgs &A, const Slots &S,         \
                                  int *cursor, int grid, cudaStream_t st);
ME_DECLARE_ROUNDS(f32)
ME_DECLARE_ROUNDS(f64)
ME_DECLARE_ROUNDS(f32f)
ME_DECLARE_ROUNDS(f64f)

// the variant of a plan: synthesis precision, and the instrument filter or not
#define ME_PICK(FN, ...)                                                                   \
  (precision == 1 ? (P.nsub > 1 ? FN##_f64f(__VA_ARGS__) : FN##_f64(__VA_ARGS__))           \
                  : (P.nsub > 1 ? FN##_f32f(__VA_ARGS__) : FN##_f32(__VA_ARGS__)))

cudaError_t launch_finish(int precision, const DevPlan &P, const InvertArgs &A, const Slots &S,
                          int *cursor, int grid, cudaStream_t st) {
  return ME_PICK(launch_finish, P, A, S, cursor, grid, st);
}

cudaError_t launch_round_grp(int precision, int G, const DevPlan &P, const InvertArgs &A,
                             const Slots &S, int parity, const int grids[3], cudaStream_t st,
                             cudaEvent_t *ev, const Overlap *ov) {
  return ME_PICK(launch_round_grp, G, P, A, S, parity, grids, st, ev, ov);
}

// grids of the unfiltered kernels (the filtered ones run grid-stride loops
// over the same grids).  Each precision and filter unit has its own SVD
// kernel, whose dynamic shared memory exceeds the default limit; the sizing of
// the SVD grid raises that limit, so it is done in the filtered unit of the
// precision too (a plan may take a filter after it is made).
int round_grid(int precision, int which, int device) {
  if (which == 2) {
    if (precision == 1)
      round_grid_f64f(2, device);
    else
      round_grid_f32f(2, device);
  }
  return precision == 1 ? round_grid_f64(which, device) : round_grid_f32(which, device);
}

cudaError_t launch_round(int precision, const DevPlan &P, const InvertArgs &A, const Slots &S,
                         int parity, const int grids[3], cudaStream_t st, cudaEvent_t *ev,
                         int svd_lanes, const Overlap *ov) {
  return ME_PICK(launch_round, P, A, S, parity, grids, st, ev, svd_lanes, ov);
}

cudaError_t launch_synth(int precision, const DevPlan &P, const double *d_par, long long npix,
                         double step7, double *d_prof, double *d_jac, cudaStream_t st) {
  const int b = 128;
  const unsigned g = (unsigned)((npix + b - 1) / b);
  if (g == 0) return cudaSuccess;
  if (precision == 1)
    synth_kernel<double><<<g, b, 0, st>>>(P, d_par, npix, step7, d_prof, d_jac);
  else
    synth_kernel<float><<<g, b, 0, st>>>(P, d_par, npix, step7, d_prof, d_jac);
  return cudaGetLastError();
}

cudaError_t launch_fit(int precision, const DevPlan &P, const double *d_fitpar,
                       const unsigned char *d_flags, long long npix, double *d_fit,
                       cudaStream_t st) {
  const int b = 128;
  const unsigned g = (unsigned)((npix + b - 1) / b);
  if (g == 0) return cudaSuccess;
  if (precision == 1)
    fit_kernel<double><<<g, b, 0, st>>>(P, d_fitpar, d_flags, npix, d_fit);
  else
    fit_kernel<float><<<g, b, 0, st>>>(P, d_fitpar, d_flags, npix, d_fit);
  return cudaGetLastError();
}

cudaError_t launch_voigt(int precision, const DevPlan &P, const double *d_nu, const double *d_a,
                         long long n, double *d_H, double *d_L, cudaStream_t st) {
  const int b = 256;
  const unsigned g = (unsigned)((n + b - 1) / b);
  if (g == 0) return cudaSuccess;
  if (precision == 1)
    voigt_kernel<double><<<g, b, 0, st>>>(P, d_nu, d_a, n, d_H, d_L);
  else
    voigt_kernel<float><<<g, b, 0, st>>>(P, d_nu, d_a, n, d_H, d_L);
  return cudaGetLastError();
}

cudaError_t launch_svd(const double *d_a, long long nmat, int n, double *d_u, double *d_w,
                       double *d_v, int *d_hits, cudaStream_t st) {
  const int b = 128;
  const unsigned g = (unsigned)((nmat + b - 1) / b);
  if (g == 0) return cudaSuccess;
  svd_kernel<<<g, b, 0, st>>>(d_a, nmat, n, d_u, d_w, d_v, d_hits);
  return cudaGetLastError();
}

// The trial-step solve's U-only decomposition (gr_svd_u, gr_svd_u_grp) of
// nmat n x n matrices: G = 1, one thread per matrix in a column of shared
// memory (stride 32), as svd_kernel of the rounds holds it; G > 1, a group of
// G lanes per matrix, row-major in shared memory, as svd_grp_kernel and the
// tail kernel hold it.  Blocks of 32 threads.
template <int G, bool FAST>
__global__ void __launch_bounds__(32) svd_u_kernel(const double *a, long long nmat, int n,
                                                   double *u, double *w, int *limit_hits) {
  constexpr int kPer = 32 / G;  // matrices per block
  constexpr int kWords = G == 1 ? 99 * 32 : kPer * 81;
  __shared__ double sm[kWords];
  const int t = threadIdx.x;
  const long long i = blockIdx.x * (long long)kPer + t / G;
  if (i >= nmat) return;  // uniform across each group
  const int nn = n * n;
  int hit;
  if constexpr (G == 1) {
    double *am = sm + t, *wm = sm + 81 * 32 + t, *rv = sm + 90 * 32 + t;
    for (int k = 0; k < nn; k++) am[k * 32] = a[i * nn + k];
    hit = gr_svd_u<32, FAST>(am, n, wm, rv);
    for (int k = 0; k < nn; k++) u[i * nn + k] = am[k * 32];
    for (int k = 0; k < n; k++) w[i * n + k] = wm[k * 32];
  } else {
    const int lane = t % G;
    const unsigned mask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << (t & ~(G - 1)));
    double *am = sm + (t / G) * 81;
    for (int k = lane; k < nn; k += G) am[k] = a[i * nn + k];
    __syncwarp(mask);
    double wl[9];
    hit = gr_svd_u_grp<G, FAST>(am, n, wl, lane, mask);
    for (int k = lane; k < nn; k += G) u[i * nn + k] = am[k];
    if (lane == 0)
      for (int k = 0; k < n; k++) w[i * n + k] = wl[k];
  }
  if (hit && limit_hits && (G == 1 || t % G == 0)) atomicAdd(limit_hits, 1);
}

template <int G>
static void launch_svd_u_g(const double *d_a, long long nmat, int n, int fast, double *d_u,
                           double *d_w, int *d_hits, cudaStream_t st) {
  const unsigned g = (unsigned)((nmat + 32 / G - 1) / (32 / G));
  if (fast)
    svd_u_kernel<G, true><<<g, 32, 0, st>>>(d_a, nmat, n, d_u, d_w, d_hits);
  else
    svd_u_kernel<G, false><<<g, 32, 0, st>>>(d_a, nmat, n, d_u, d_w, d_hits);
}

cudaError_t launch_svd_u(const double *d_a, long long nmat, int n, int lanes, int fast,
                         double *d_u, double *d_w, int *d_hits, cudaStream_t st) {
  if (nmat <= 0) return cudaSuccess;
  switch (lanes) {
    case 1: launch_svd_u_g<1>(d_a, nmat, n, fast, d_u, d_w, d_hits, st); break;
    case 2: launch_svd_u_g<2>(d_a, nmat, n, fast, d_u, d_w, d_hits, st); break;
    case 4: launch_svd_u_g<4>(d_a, nmat, n, fast, d_u, d_w, d_hits, st); break;
    case 8: launch_svd_u_g<8>(d_a, nmat, n, fast, d_u, d_w, d_hits, st); break;
    case 16: launch_svd_u_g<16>(d_a, nmat, n, fast, d_u, d_w, d_hits, st); break;
    case 32: launch_svd_u_g<32>(d_a, nmat, n, fast, d_u, d_w, d_hits, st); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_order_by_key(const unsigned char *d_key, long long n, int *d_hist,
                                long long *d_order, cudaStream_t st, long long base) {
  if (n <= 0) return cudaSuccess;
  const long long chunk = n / kOrderBlocks + 1 > 1024 ? n / kOrderBlocks + 1 : 1024;
  const int nb = (int)((n + chunk - 1) / chunk);
  order_hist_kernel<<<nb, 256, 0, st>>>(d_key, n, chunk, d_hist);
  order_scan_kernel<<<1, 1024, 0, st>>>(d_hist, kOrderBuckets * nb);
  order_scatter_kernel<<<nb, 256, 0, st>>>(d_key, n, chunk, d_hist, d_order, base);
  return cudaGetLastError();
}

// Re-sort of the queue positions [first, first + n) of `list` by the pixels'
// misfit keys, stable (the streamed host entry point: once the whole map has
// arrived, the part of the queue not yet taken goes into one global order).
__global__ void tail_gather_kernel(const long long *list, long long first, long long n,
                                   const unsigned char *key, unsigned char *tkey,
                                   long long *tval) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long long pix = list[first + i];
  tval[i] = pix;
  tkey[i] = key[pix];
}

__global__ void tail_scatter_kernel(long long *list, long long first, long long n,
                                    const long long *perm, const long long *tval) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  list[first + i] = tval[perm[i]];
}

cudaError_t launch_resort_tail(long long *d_list, long long first, long long n,
                               const unsigned char *d_key, unsigned char *d_tkey,
                               long long *d_tval, int *d_hist, long long *d_perm,
                               cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int b = 256;
  const unsigned g = (unsigned)((n + b - 1) / b);
  tail_gather_kernel<<<g, b, 0, st>>>(d_list, first, n, d_key, d_tkey, d_tval);
  cudaError_t e = launch_order_by_key(d_tkey, n, d_hist, d_perm, st, 0);
  if (e != cudaSuccess) return e;
  tail_scatter_kernel<<<g, b, 0, st>>>(d_list, first, n, d_perm, d_tval);
  return cudaGetLastError();
}

cudaError_t launch_start_order(int precision, const DevPlan &P, const double *d_prof,
                               const double *d_init, long long npix, unsigned char *d_key,
                               int *d_hist, long long *d_order, cudaStream_t st,
                               long long base) {
  if (npix <= 0) return cudaSuccess;
  const int b = 128;
  const unsigned g = (unsigned)((npix + b - 1) / b);
  // about 16 wavelengths of the grid
  const int stride = P.nl / 16 > 1 ? P.nl / 16 : 1;
  if (precision == 1) {
    if (P.nsub > 1)
      start_misfit_kernel<double, true><<<g, b, 0, st>>>(P, d_prof, d_init, npix, stride, d_key);
    else
      start_misfit_kernel<double, false><<<g, b, 0, st>>>(P, d_prof, d_init, npix, stride, d_key);
  } else {
    if (P.nsub > 1)
      start_misfit_kernel<float, true><<<g, b, 0, st>>>(P, d_prof, d_init, npix, stride, d_key);
    else
      start_misfit_kernel<float, false><<<g, b, 0, st>>>(P, d_prof, d_init, npix, stride, d_key);
  }
  return launch_order_by_key(d_key, npix, d_hist, d_order, st, base);
}

cudaError_t launch_init_guess(const DevPlan &P, const double *d_prof, long long npix,
                              double *d_guess, double *d_extra, int *d_status, cudaStream_t st) {
  const int b = 128;
  const unsigned g = (unsigned)((npix + b - 1) / b);
  if (g == 0) return cudaSuccess;
  init_guess_kernel<<<g, b, 0, st>>>(P, d_prof, npix, d_guess, d_extra, d_status);
  return cudaGetLastError();
}

}  // namespace me

// me_invert_batch_device_noalloc -- the inversion entry point that allocates
// nothing.  It has no counterpart in the reference; it is an addition of this
// library.
//
// Some callers cannot allocate device memory when they run the inversion:
// data-reduction pipelines and frameworks that reserve the GPU's memory for
// their own pool when they start (a cudaMalloc of ours would then fail, or
// take memory their pool counts on), and real-time loops at the instrument,
// where cudaMalloc and cudaFree can synchronise the device and stall the
// loop for an unbounded time.
// For them me_invert_batch_device_noalloc() does the work of
// me_invert_batch_device() with all of its scratch -- the in-flight pixel
// slots, the per-pixel bookkeeping of the carried LM chi^2, the wavelength
// grid and the counters -- in one static device array of fixed size, declared
// below.  That array exists on every GPU the library is loaded on until the
// process exits (about 12.4 MB).  The caller still owns the profiles and the
// results.
//
// Limits: at most ME_NOALLOC_MAX_PIXELS pixels per call (larger maps go in
// chunks, chaining carry_chisq from one call to the next exactly as the
// reference's pixel loop carries it) and ME_NOALLOC_SLOTS pixels in flight.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <mutex>

#include "../../include/me_b200.h"
#include "me_kernels.h"

namespace {

constexpr int kSlots = ME_NOALLOC_SLOTS;
constexpr long kMaxPix = ME_NOALLOC_MAX_PIXELS;

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Byte offsets of the regions inside the scratch array.
constexpr size_t kOffLambda = 0;                                            // [512] double
constexpr size_t kOffDlambda = align256(kOffLambda + 8 * ME_MAX_NL);        // [512] double
constexpr size_t kOffSmall = align256(kOffDlambda + 8 * ME_MAX_NL);         // counters
constexpr size_t kOffPix = align256(kOffSmall + 256);                       // [W] long long
constexpr size_t kOffI32 = align256(kOffPix + 8 * (size_t)kSlots);          // [4][W] int
constexpr size_t kOffCnt = align256(kOffI32 + 16 * (size_t)kSlots);         // [4][W] uint
constexpr size_t kOffU8 = align256(kOffCnt + 16 * (size_t)kSlots);          // [W] uchar
constexpr size_t kOffSc = align256(kOffU8 + (size_t)kSlots);                // [SC][W] double
constexpr size_t kOffVec = align256(kOffSc + 8 * me::SC_COUNT * (size_t)kSlots);  // [45][W]
constexpr size_t kOffHess = align256(kOffVec + 8 * 45 * (size_t)kSlots);    // [81][W] double
constexpr size_t kOffList = align256(kOffHess + 8 * 81 * (size_t)kSlots);   // [4][W] int
constexpr size_t kOffFlags = align256(kOffList + 16 * (size_t)kSlots);      // [P] uchar
constexpr size_t kOffPen0 = align256(kOffFlags + (size_t)kMaxPix);          // [P] double
constexpr size_t kOffLast = align256(kOffPen0 + 8 * (size_t)kMaxPix);       // [P] double
constexpr size_t kOffCount = align256(kOffLast + 8 * (size_t)kMaxPix);      // [P][4] uint
constexpr size_t kOffUsed = align256(kOffCount + 16 * (size_t)kMaxPix);     // [P] double
constexpr size_t kOffRedo = align256(kOffUsed + 8 * (size_t)kMaxPix);       // [P] long long
constexpr size_t kScratchBytes = align256(kOffRedo + 8 * (size_t)kMaxPix);

// The scratch.  In host code this name is only a stand-in for the symbol: its
// device address comes from cudaGetSymbolAddress (setup()).  Device code below
// names it directly.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Small-counter block (kOffSmall): jcount[2], rcount[2], busy, pad, next,
// totals[8], redo count, carry out.
struct Small {
  int jcount[2];
  int rcount[2];
  int busy;
  int pad;
  unsigned long long next;
  unsigned long long totals[8];
  long long redo;
  double carry_out;
};
static_assert(sizeof(Small) <= 256, "small-counter block");

// Scan of the carried LM chi^2 in pixel order, the device-side twin of the
// fix-up in me_invert_batch_device: lists the pixels whose first
// regularisation ratio test (Src/LM_FIT.c:555-559) saw a carried value on the
// other side of the threshold than the true one, and records the value each
// is re-run with.  One thread (the dependency is sequential); pass 0 first
// initialises the carried value each pixel was run with.
__global__ void carry_scan_kernel(long npix, double carry, int regul_any, int pass) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  Small *sm = reinterpret_cast<Small *>(g_scratch + kOffSmall);
  const unsigned char *flags = g_scratch + kOffFlags;
  const double *pen0 = reinterpret_cast<const double *>(g_scratch + kOffPen0);
  const double *last = reinterpret_cast<const double *>(g_scratch + kOffLast);
  double *used = reinterpret_cast<double *>(g_scratch + kOffUsed);
  long long *redo = reinterpret_cast<long long *>(g_scratch + kOffRedo);
  if (pass == 0)
    for (long i = 0; i < npix; i++) used[i] = i == 0 ? carry : INFINITY;
  double prev = carry;
  long long m = 0;
  for (long i = 0; i < npix; i++) {
    if (!(flags[i] & 1)) continue;
    if (regul_any) {
      const bool want = pen0[i] > 0.1 * prev;
      const bool was = pen0[i] > 0.1 * used[i];
      if (want != was) {
        redo[m++] = i;
        used[i] = prev;
      }
    }
    if (flags[i] & 2) prev = last[i];
  }
  sm->redo = m;
  sm->carry_out = prev;
}

struct DeviceSetup {
  bool ready = false;
  unsigned char *base = nullptr;
  int grids[3] = {0, 0, 0};  // jac, trial, svd at full occupancy
};
std::mutex g_mu;
DeviceSetup g_dev[64][2];  // [device][precision]

// failures are reported through me_last_error(), like every other entry point
int set_err(int code, const char *msg) { return me::record_error(code, msg); }

#define NA_CK(call)                                                       \
  do {                                                                    \
    cudaError_t e_ = (call);                                              \
    if (e_ != cudaSuccess) return set_err(ME_ERR_CUDA, cudaGetErrorString(e_)); \
  } while (0)

// Per-device, per-precision set-up with the device current: the device
// address of the scratch array and the occupancy-derived grids.
int setup(int prec, DeviceSetup **out) {
  int dev = 0;
  NA_CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return set_err(ME_ERR_ARG, "device index above 63");
  std::lock_guard<std::mutex> lock(g_mu);
  DeviceSetup &d = g_dev[dev][prec];
  if (!d.ready) {
    void *ptr = nullptr;
    NA_CK(cudaGetSymbolAddress(&ptr, g_scratch));
    d.base = static_cast<unsigned char *>(ptr);
    d.grids[0] = me::round_grid(prec, 0, dev);
    d.grids[1] = me::round_grid(prec, 1, dev);
    d.grids[2] = me::round_grid(prec, 2, dev);
    d.ready = true;
  }
  *out = &d;
  return ME_OK;
}

// Rounds until the queue of A is exhausted and every slot is empty.  A pixel
// ends within slot_step_cap(P) LM steps, and while the queue feeds the slots
// every round advances each of the W slots by one step, so the queue empties
// within about ceil(count / W) x cap rounds and the last pixels end within cap
// more (the bound me_invert_batch_device uses); rounds beyond it (a
// non-finite damping value, say) end the call with ME_ERR_TIMEOUT.
int run_rounds(int prec, const me::DevPlan &P, const me::InvertArgs &A, const me::Slots &S,
               const int grids[3], cudaStream_t st, Small *d_small) {
  NA_CK(cudaMemsetAsync(S.state, 0, sizeof(int) * (size_t)S.W, st));  // SL_EMPTY
  NA_CK(cudaMemsetAsync(d_small, 0, offsetof(Small, totals), st));  // lists, busy, next
  const double round_cap =
      (double)me::slot_step_cap(P) * (double)((A.count + S.W - 1) / S.W + 1);
  long long rounds = 0;
  int parity = 0;
  while (true) {
    if ((double)rounds > round_cap)
      return set_err(ME_ERR_TIMEOUT, "inversion rounds exceeded their bound");
    for (int r = 0; r < 8; r++) {
      NA_CK(me::launch_round(prec, P, A, S, parity, grids, st));
      parity ^= 1;
    }
    rounds += 8;
    unsigned long long next = 0;
    int busy = 0;
    NA_CK(cudaMemcpyAsync(&next, &d_small->next, sizeof(next), cudaMemcpyDeviceToHost, st));
    NA_CK(cudaMemcpyAsync(&busy, &d_small->busy, sizeof(busy), cudaMemcpyDeviceToHost, st));
    NA_CK(cudaStreamSynchronize(st));
    if (next >= (unsigned long long)A.count && busy == 0) break;
  }
  return ME_OK;
}

}  // namespace

extern "C" int me_invert_batch_device_noalloc(const me_config *cfg, const double *lambda, int nl,
                                              const double *d_prof, long npix, double *d_res,
                                              double *carry_chisq, void *stream) {
  if (!cfg || !lambda || !d_prof || !d_res || !carry_chisq)
    return set_err(ME_ERR_ARG, "null argument");
  if (npix < 0 || npix > kMaxPix)
    return set_err(ME_ERR_ARG, "npix exceeds ME_NOALLOC_MAX_PIXELS (65536): split the map");
  me::DevPlan P;
  int rc = me::build_devplan(cfg, lambda, nl, P);
  if (rc) return rc;  // build_devplan recorded the cause
  // the sub-wavelength grid of an instrument filter would need scratch of its
  // own: filtered plans go through me_invert_batch_device
  if (P.nsub > 1) return set_err(ME_ERR_CONFIG, "no instrument filter without allocation");
  if (npix == 0) return ME_OK;
  const int prec = cfg->precision == ME_PREC_FP64 ? 1 : 0;
  DeviceSetup *d = nullptr;
  rc = setup(prec, &d);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  unsigned char *base = d->base;

  // wavelength grid into the scratch
  double dl[ME_MAX_NL];
  for (int i = 0; i < nl; i++) dl[i] = lambda[i] - P.lambda0;
  NA_CK(cudaMemcpyAsync(base + kOffLambda, lambda, sizeof(double) * nl, cudaMemcpyHostToDevice,
                        st));
  NA_CK(cudaMemcpyAsync(base + kOffDlambda, dl, sizeof(double) * nl, cudaMemcpyHostToDevice, st));
  P.lambda = reinterpret_cast<const double *>(base + kOffLambda);
  P.dlambda = reinterpret_cast<const double *>(base + kOffDlambda);

  Small *d_small = reinterpret_cast<Small *>(base + kOffSmall);
  const int W = (int)(npix < kSlots ? npix : kSlots);
  const size_t w = (size_t)kSlots;
  me::Slots S;
  S.W = W;
  S.pix = reinterpret_cast<long long *>(base + kOffPix);
  int *i32 = reinterpret_cast<int *>(base + kOffI32);
  S.state = i32;
  S.run = i32 + w;
  S.it = i32 + 2 * w;
  S.tk = i32 + 3 * w;
  S.cnt = reinterpret_cast<unsigned int *>(base + kOffCnt);
  S.had_trial = base + kOffU8;
  S.sc = reinterpret_cast<double *>(base + kOffSc);
  double *v = reinterpret_cast<double *>(base + kOffVec);
  S.guess = v;
  S.par = v + 9 * w;
  S.pbest = v + 18 * w;
  S.jvec = v + 27 * w;
  S.ptmp = v + 36 * w;
  S.hess = reinterpret_cast<double *>(base + kOffHess);
  S.jlist = reinterpret_cast<int *>(base + kOffList);
  S.rlist = S.jlist + 2 * w;
  S.jcount = d_small->jcount;
  S.rcount = d_small->rcount;
  S.busy = &d_small->busy;
  S.obs = nullptr;  // the kernels read the pixels' rows of the map
  // (the kernels index the [k][W] arrays with the active slot count W as
  // their stride; with W < kSlots each region is used densely from its start)

  me::InvertArgs A;
  memset(&A, 0, sizeof(A));
  A.prof = d_prof;
  A.res = d_res;
  A.fit = nullptr;
  A.flags = base + kOffFlags;
  A.penalty0 = reinterpret_cast<double *>(base + kOffPen0);
  A.lastchi = reinterpret_cast<double *>(base + kOffLast);
  A.counters = reinterpret_cast<unsigned int *>(base + kOffCount);
  A.totals = d_small->totals;
  A.next = &d_small->next;
  A.count = npix;
  A.carry = *carry_chisq;
  A.first_pixel = 0;
  NA_CK(cudaMemsetAsync(d_small->totals, 0, sizeof(d_small->totals), st));

  int grids[3];
  grids[0] = d->grids[0] < (W + me::kBlock - 1) / me::kBlock ? d->grids[0]
                                                             : (W + me::kBlock - 1) / me::kBlock;
  grids[1] = d->grids[1] < (W + me::kBlock - 1) / me::kBlock ? d->grids[1]
                                                             : (W + me::kBlock - 1) / me::kBlock;
  grids[2] = d->grids[2] < (W + me::kSvdBlock - 1) / me::kSvdBlock
                 ? d->grids[2]
                 : (W + me::kSvdBlock - 1) / me::kSvdBlock;
  rc = run_rounds(prec, P, A, S, grids, st, d_small);
  if (rc) return rc;

  // the LM chi^2 carried from pixel to pixel: re-run the pixels whose first
  // ratio test it flips, until none is left (as me_invert_batch_device).  A
  // pass settles at least the first flipped pixel for good (only later pixels
  // depend on it), so npix + 1 passes bound the loop.
  for (long pass = 0;; pass++) {
    if (pass > npix) return set_err(ME_ERR_TIMEOUT, "carried chi^2 passes exceeded their bound");
    carry_scan_kernel<<<1, 1, 0, st>>>(npix, *carry_chisq, P.regul_any, pass);
    NA_CK(cudaGetLastError());
    long long redo = 0;
    NA_CK(cudaMemcpyAsync(&redo, &d_small->redo, sizeof(redo), cudaMemcpyDeviceToHost, st));
    NA_CK(cudaStreamSynchronize(st));
    if (redo == 0) break;
    me::InvertArgs B = A;
    B.list = reinterpret_cast<const long long *>(base + kOffRedo);
    B.count = redo;
    B.stale = reinterpret_cast<const double *>(base + kOffUsed);
    const int Wr = (int)(redo < W ? redo : W);
    me::Slots Sr = S;
    Sr.W = Wr;
    rc = run_rounds(prec, P, B, Sr, grids, st, d_small);
    if (rc) return rc;
  }
  double carry = 0.0;
  NA_CK(cudaMemcpyAsync(&carry, &d_small->carry_out, sizeof(carry), cudaMemcpyDeviceToHost, st));
  NA_CK(cudaStreamSynchronize(st));
  *carry_chisq = carry;
  return ME_OK;
}

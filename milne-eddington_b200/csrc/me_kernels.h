// me_kernels.h -- launch interface between the host plan (me_api.cu) and the
// CUDA kernels (me_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "me_device.cuh"

namespace me {

constexpr int kInvertBlock = 128;
// minimum resident CTAs per SM the inversion kernel is compiled for (caps
// its registers at 65536 / (128 * ME_INV_MINB))
#ifndef ME_INV_MINB
#define ME_INV_MINB 3
#endif

// Buffers of one inversion launch (all device pointers).
struct InvertArgs {
  const double *prof;          // [npix][4][nl]
  double *res;                 // [npix][10]
  double *fit;                 // [npix][4][nl] or null
  unsigned char *flags;        // [npix] bit0 inverted, bit1 made a trial step (or null)
  double *penalty0;            // [npix] regularisation penalty at the first guess (or null)
  double *lastchi;             // [npix] chi^2 of the pixel's last trial step (or null)
  unsigned int *counters;      // [npix][4] runs, iterations, trials, accepted (or null)
  unsigned long long *totals;  // [8] valid, runs, iterations, trials, accepted, jacobians, svd limit hits
  unsigned long long *next;    // work counter (zeroed before the launch)
  const long long *list;       // pixel indices to process (null = 0..count-1)
  long long count;             // number of work items
  const double *stale;         // [npix] carried LM chi^2 per pixel (null = use carry/first_pixel)
  double carry;                // carried LM chi^2 for pixel first_pixel
  long long first_pixel;
};

int invert_grid(int precision, int device);
cudaError_t launch_invert(int precision, const DevPlan &P, const InvertArgs &A, int grid,
                          cudaStream_t st);
cudaError_t launch_synth(int precision, const DevPlan &P, const double *d_par, long long npix,
                         double step7, double *d_prof, double *d_jac, cudaStream_t st);
cudaError_t launch_voigt(int precision, const DevPlan &P, const double *d_nu, const double *d_a,
                         long long n, double *d_H, double *d_L, cudaStream_t st);
cudaError_t launch_svd(const double *d_a, long long nmat, int n, double *d_u, double *d_w,
                       double *d_v, int *d_hits, cudaStream_t st);
cudaError_t launch_init_guess(const DevPlan &P, const double *d_prof, long long npix,
                              double *d_guess, double *d_extra, int *d_status, cudaStream_t st);

}  // namespace me

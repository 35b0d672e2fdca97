// me_invert_f64.cu -- double instantiation of the inversion round kernels.
#include "me_invert.cuh"

namespace me {

template __global__ void jac_kernel<double>(const __grid_constant__ DevPlan P,
                                            const __grid_constant__ InvertArgs A,
                                            const __grid_constant__ Slots S, int parity);
template __global__ void trial_kernel<double>(const __grid_constant__ DevPlan P,
                                              const __grid_constant__ InvertArgs A,
                                              const __grid_constant__ Slots S, int parity);
template __global__ void finish_kernel<double>(const __grid_constant__ DevPlan P,
                                              const __grid_constant__ InvertArgs A,
                                              const __grid_constant__ Slots S, int *cursor);

// which: 0 = jac_kernel, 1 = trial_kernel, 2 = svd_kernel, 3 = finish_kernel
// (CTAs for a full device)
int round_grid_f64(int which, int device) {
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (which == 0) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, jac_kernel<double>, kBlock, 0);
  } else if (which == 1) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trial_kernel<double>, kBlock, 0);
  } else if (which == 3) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, finish_kernel<double>, kBlock, 0);
  } else {
    cudaFuncSetAttribute(svd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSvdSmem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, svd_kernel, kSvdBlock, kSvdSmem);
  }
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

static void launch_svd_lanes(int lanes, const DevPlan &P, const InvertArgs &A, const Slots &S,
                             int parity, int which, int grid, cudaStream_t st) {
  switch (lanes) {
    case 2: svd_grp_kernel<2><<<grid, kBlock, 0, st>>>(P, A, S, parity, which); break;
    case 4: svd_grp_kernel<4><<<grid, kBlock, 0, st>>>(P, A, S, parity, which); break;
    case 8: svd_grp_kernel<8><<<grid, kBlock, 0, st>>>(P, A, S, parity, which); break;
    default: svd_kernel<<<grid, kSvdBlock, kSvdSmem, st>>>(P, A, S, parity, which); break;
  }
}

// grids: jac_kernel, trial_kernel, svd; svd_lanes: lanes per matrix of the
// SVD launches (1: svd_kernel, one thread each; 2, 4, 8: svd_grp_kernel).
cudaError_t launch_round_f64(const DevPlan &P, const InvertArgs &A, const Slots &S, int parity,
                           const int grids[3], cudaStream_t st, cudaEvent_t *ev, int svd_lanes) {
  if (ev) cudaEventRecord(ev[0], st);
  jac_kernel<double><<<grids[0], kBlock, 0, st>>>(P, A, S, parity);
  if (ev) cudaEventRecord(ev[1], st);
  launch_svd_lanes(svd_lanes, P, A, S, parity, 0, grids[2], st);
  if (ev) cudaEventRecord(ev[2], st);
  launch_svd_lanes(svd_lanes, P, A, S, parity, 1, grids[2], st);
  if (ev) cudaEventRecord(ev[3], st);
  trial_kernel<double><<<grids[1], kBlock, 0, st>>>(P, A, S, parity);
  if (ev) cudaEventRecord(ev[4], st);
  return cudaGetLastError();
}

cudaError_t launch_finish_f64(const DevPlan &P, const InvertArgs &A, const Slots &S, int *cursor,
                              int grid, cudaStream_t st) {
  finish_kernel<double><<<grid, kBlock, 0, st>>>(P, A, S, cursor);
  return cudaGetLastError();
}

template <int G>
static void launch_grp(const DevPlan &P, const InvertArgs &A, const Slots &S, int parity,
                       const int grids[3], cudaStream_t st, cudaEvent_t *ev) {
  if (ev) cudaEventRecord(ev[0], st);
  jac_grp_kernel<double, G><<<grids[0], kBlock, 0, st>>>(P, A, S, parity);
  if (ev) cudaEventRecord(ev[1], st);
  svd_grp_kernel<G><<<grids[2], kBlock, 0, st>>>(P, A, S, parity, 0);
  if (ev) cudaEventRecord(ev[2], st);
  svd_grp_kernel<G><<<grids[2], kBlock, 0, st>>>(P, A, S, parity, 1);
  if (ev) cudaEventRecord(ev[3], st);
  trial_grp_kernel<double, G><<<grids[1], kBlock, 0, st>>>(P, A, S, parity);
  if (ev) cudaEventRecord(ev[4], st);
}

// A round with G lanes per slot (G = 2, 4, 8, 16, 32), after the queue is empty.
cudaError_t launch_round_grp_f64(int G, const DevPlan &P, const InvertArgs &A, const Slots &S,
                               int parity, const int grids[3], cudaStream_t st, cudaEvent_t *ev) {
  switch (G) {
    case 2: launch_grp<2>(P, A, S, parity, grids, st, ev); break;
    case 4: launch_grp<4>(P, A, S, parity, grids, st, ev); break;
    case 8: launch_grp<8>(P, A, S, parity, grids, st, ev); break;
    case 16: launch_grp<16>(P, A, S, parity, grids, st, ev); break;
    case 32: launch_grp<32>(P, A, S, parity, grids, st, ev); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace me

// me_invert_f32.cu -- float instantiation of the inversion round kernels.
#include "me_invert.cuh"

namespace me {

template __global__ void jac_kernel<float>(const __grid_constant__ DevPlan P,
                                            const __grid_constant__ InvertArgs A,
                                            const __grid_constant__ Slots S, int parity);
template __global__ void trial_kernel<float>(const __grid_constant__ DevPlan P,
                                              const __grid_constant__ InvertArgs A,
                                              const __grid_constant__ Slots S, int parity);
template __global__ void finish_kernel<float>(const __grid_constant__ DevPlan P,
                                              const __grid_constant__ InvertArgs A,
                                              const __grid_constant__ Slots S, int *cursor);

// which: 0 = jac_kernel, 1 = trial_kernel, 2 = svd_kernel, 3 = finish_kernel
// (CTAs for a full device)
int round_grid_f32(int which, int device) {
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (which == 0) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, jac_kernel<float>, kBlock, 0);
  } else if (which == 1) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trial_kernel<float>, kBlock, 0);
  } else if (which == 3) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, finish_kernel<float>, kBlock, 0);
  } else {
    cudaFuncSetAttribute(svd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSvdSmem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, svd_kernel, kSvdBlock, kSvdSmem);
  }
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

cudaError_t launch_round_f32(const DevPlan &P, const InvertArgs &A, const Slots &S, int parity,
                           const int grids[3], cudaStream_t st, cudaEvent_t *ev) {
  if (ev) cudaEventRecord(ev[0], st);
  jac_kernel<float><<<grids[0], kBlock, 0, st>>>(P, A, S, parity);
  if (ev) cudaEventRecord(ev[1], st);
  svd_kernel<<<grids[2], kSvdBlock, kSvdSmem, st>>>(P, A, S, parity, 0);
  if (ev) cudaEventRecord(ev[2], st);
  svd_kernel<<<grids[2], kSvdBlock, kSvdSmem, st>>>(P, A, S, parity, 1);
  if (ev) cudaEventRecord(ev[3], st);
  trial_kernel<float><<<grids[1], kBlock, 0, st>>>(P, A, S, parity);
  if (ev) cudaEventRecord(ev[4], st);
  return cudaGetLastError();
}

cudaError_t launch_finish_f32(const DevPlan &P, const InvertArgs &A, const Slots &S, int *cursor,
                              int grid, cudaStream_t st) {
  finish_kernel<float><<<grid, kBlock, 0, st>>>(P, A, S, cursor);
  return cudaGetLastError();
}

}  // namespace me

// me_invert_f32.cu -- float instantiation of the inversion kernel.
#include "me_invert.cuh"

namespace me {

template __global__ void invert_kernel<float>(const DevPlan P, InvertArgs A);

int invert_grid_f32(int device) {
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, invert_kernel<float>, kInvertBlock, 0);
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

cudaError_t launch_invert_f32(const DevPlan &P, const InvertArgs &A, int grid, cudaStream_t st) {
  invert_kernel<float><<<grid, kInvertBlock, 0, st>>>(P, A);
  return cudaGetLastError();
}

}  // namespace me

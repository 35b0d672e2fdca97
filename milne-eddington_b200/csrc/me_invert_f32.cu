// me_invert_f32.cu -- the inversion kernels' launchers, float synthesis.
#include "me_invert.cuh"

namespace me {

ME_INSTANTIATE_ROUNDS(float, false, f32)

}  // namespace me

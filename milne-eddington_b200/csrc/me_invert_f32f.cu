// me_invert_f32f.cu -- the inversion kernels' launchers, float synthesis, instrument filter.
#include "me_invert.cuh"

namespace me {

ME_INSTANTIATE_ROUNDS(float, true, f32f)

}  // namespace me

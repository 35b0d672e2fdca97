// me_invert_f64.cu -- the inversion kernels' launchers, double synthesis.
#include "me_invert.cuh"

namespace me {

ME_INSTANTIATE_ROUNDS(double, false, f64)

}  // namespace me

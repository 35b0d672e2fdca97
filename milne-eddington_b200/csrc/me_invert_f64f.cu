// me_invert_f64f.cu -- the inversion kernels' launchers, double synthesis, instrument filter.
#include "me_invert.cuh"

namespace me {

ME_INSTANTIATE_ROUNDS(double, true, f64f)

}  // namespace me

// amhd_f32.cu -- float32 instantiation of the kernels (fp32 state and fluxes,
// float64 pressure recovery / CFL reduction inside them).
#include "amhd_launch_impl.cuh"

namespace amhd {
template struct Launch<float>;
}  // namespace amhd

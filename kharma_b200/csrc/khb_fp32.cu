// khb_fp32.cu -- the FP32-flux form: reconstruction, Riemann fluxes and EMF averaging in FP32,
// with the zone pass (RK update accumulated in FP64, inversion, floors, P->U) in FP64.
// Built with FMA contraction.  Instantiates Launch<float>.
#include "khb_kernels.cuh"

namespace khb {
template struct Launch<float>;
}

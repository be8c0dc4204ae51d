// khb_fp64.cu -- the FP64 path: flux, zone-pass and ghost-zone kernels in double precision.
//
// Built with -fmad=false: every multiply and add rounds separately, in the evaluation order of the
// reference's device functions, so results agree with a reference (or oracle) build bit for bit
// where no library transcendental is involved.  Instantiates Launch<double> and LaunchCommon.
#define KHB_COMMON_KERNELS 1
#include "khb_kernels.cuh"

namespace khb {
template struct Launch<double>;
}

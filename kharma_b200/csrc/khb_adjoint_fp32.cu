// khb_adjoint_fp32.cu -- the FP32-flux form's face-flux adjoint (k_adj_flux in float arithmetic),
// built like khb_fp32.cu (FMA contraction, fast FP32 divide and square root, FTZ) so that the
// adjoint of the FP32 faces uses the forward FP32 kernels' arithmetic.
#include "khb_adjoint_flux.cuh"

namespace khb {

template <int DIR, int NV, int RECON>
void launch_adj_flux_f32(cudaStream_t st, const Dims& d, const DevGeom& g, const Phys& ph, const khb_fields& P,
                         const double* Fbar, const double* Uupd, double w, double area, const double* seed,
                         double seed_scale, const khb_fields& Pbar, const Box& bx)
{
    k_adj_flux<DIR, NV, RECON, float><<<box_blocks(bx), 128, 0, st>>>(d, g, ph, P, Fbar, Uupd, w, area, seed,
                                                                      seed_scale, Pbar, bx);
}

#define KHB_ADJ_F32(DIR, NV)                                                                                    \
    template void launch_adj_flux_f32<DIR, NV, RECON_MC>(cudaStream_t, const Dims&, const DevGeom&, const Phys&,  \
                                                         const khb_fields&, const double*, const double*, double,  \
                                                         double, const double*, double, const khb_fields&,        \
                                                         const Box&);                                             \
    template void launch_adj_flux_f32<DIR, NV, RECON_DONOR>(cudaStream_t, const Dims&, const DevGeom&,            \
                                                            const Phys&, const khb_fields&, const double*,        \
                                                            const double*, double, double, const double*, double,  \
                                                            const khb_fields&, const Box&);
KHB_ADJ_F32(1, 5)
KHB_ADJ_F32(2, 5)
KHB_ADJ_F32(3, 5)
KHB_ADJ_F32(1, 8)
KHB_ADJ_F32(2, 8)
KHB_ADJ_F32(3, 8)
#undef KHB_ADJ_F32

} // namespace khb

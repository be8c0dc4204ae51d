// khb_kernels.cuh -- sm_100a kernels of libkhb (host side in khb_api.cu, C ABI in include/khb.h).
//
// Per RK stage the work is:
//   k_flux (x ndim)   reconstruction + prim_to_flux + vchar + LLF/HLLE at every face needed,
//                     fluxes to scratch (FP64, or FP32 in the FP32-flux form)
//   k_fix_flux        polar and inflow flux corrections on the raw fluxes (spherical runs)
//   k_zone            ONE pass per zone: flux-CT EMFs from the raw B fluxes, flux divergence,
//                     geometric source, RK combination, 1D_W inversion, floors, lock-step P->U,
//                     CFL reduction (last stage) and the failed-zone list
//   k_fixup           neighbour averaging of failed zones (grid sized once, reads the list)
//   k_bc_* / k_periodic  ghost zones
// Every loop in device code is bounded; failures are reported through pflag, never by trapping.
#include "khb_device.cuh"
#include "khb_types.cuh"

#include <cstdio>
#include <cstring>
#include <cmath>
#include <string>
#include <vector>
#include <limits>

namespace khb {

__device__ __forceinline__ void zone_kji(const Dims& d, long long c, int& k, int& j, int& i)
{
    i = (int)(c % d.n1);
    const long long r = c / d.n1;
    j = (int)(r % d.n2);
    k = (int)(r / d.n2);
}

// Thread -> (k, j, i) of a box [lo, lo + cnt) in 32-bit arithmetic (no 64-bit division).  A block
// of 128 threads covers 128/kz consecutive (j, i) plane positions, i fastest, in each of kz
// consecutive k planes (kz = 1, 2 or 4; by default 4 when the box is at least 4 planes thick, else
// 1), so the warps of a block read the same x3-independent geometry and all but the first find it
// in L1.
// blk: the block's index within the box (blockIdx.x for a single-box launch)
__device__ __forceinline__ bool box_cell(const Box& b, unsigned blk, int& i, int& j, int& k)
{
    const unsigned w = threadIdx.x >> b.pshift, q = threadIdx.x & ((1u << b.pshift) - 1u);
    const unsigned bk = blk / b.nbp, bp = blk - bk * b.nbp;
    const unsigned p = (bp << b.pshift) + q, kk = bk * (unsigned)b.kz + w;
    if (p >= b.np || kk >= (unsigned)b.cnt_k) return false;
    const unsigned jj = p / (unsigned)b.cnt_i;
    i = b.lo_i + (int)(p - jj * (unsigned)b.cnt_i);
    j = b.lo_j + (int)jj;
    k = b.lo_k + (int)kk;
    return true;
}

// Load the centre geometry of zone (j,i)
// SYM: the upper triangles only, mirrored (10 values per metric held in registers instead of 16).
// The host tables are symmetric to rounding, not bit for bit, so only the FP32-flux form, which has
// no bitwise contract, reads them this way.
template <bool SYM = false>
__device__ __forceinline__ void load_zone_geom(const DevGeom& g, int j, int i, ZoneGeom& G)
{
    const long long gi = (long long)j*g.G1 + i;
#pragma unroll
    for (int m = 0; m < 16; ++m) {
        const int r = m/4, q = m%4;
        if (SYM && q < r) continue;
        G.gcov[r][q] = __ldg(g.gcov[3] + m*g.gs + gi);
        G.gcon[r][q] = __ldg(g.gcon[3] + m*g.gs + gi);
        if (SYM) { G.gcov[q][r] = G.gcov[r][q]; G.gcon[q][r] = G.gcon[r][q]; }
    }
    G.gdet = __ldg(g.gdet[3] + gi);
}

// The floor prescription of zone (j, i): the inner one inside floors_switch_r when radius-dependent
// floors are on (floors_functions.hpp:56-57, 89-90; inverter.cpp:165-168)
__device__ __forceinline__ const Prescription& floors_at(const Phys& ph, const DevGeom& g, int j, int i)
{
    return (ph.fl.radius_dependent_floors && __ldg(g.rcen + (long long)j*g.n1 + i) < ph.fl.floors_switch_r)
               ? ph.fl_inner : ph.fl;
}

// Flux::p_to_u for one zone (all NV conserved variables), flux_functions.hpp:343-352
template <int NV>
__device__ __forceinline__ void p_to_u_zone(const ZoneGeom& G, double gam, const double* P, double* U)
{
    FourVec<double> D;
    const double gcon0[4] = {G.gcon[0][0], G.gcon[0][1], G.gcon[0][2], G.gcon[0][3]};
    calc_4vecs<double, (NV > 5)>(G.gcov, G.gcon[0][0], gcon0, P, D);
    prim_to_flux<double, NV>(P, D, gam, G.gdet, 0, U);
}

// ===================================================================================== fluxes
// One thread per face.  Face (k,j,i) along dir lies between zones c - st and c.
template <typename R> struct FaceTables;
template <> struct FaceTables<double> {
    static __device__ __forceinline__ const double* gcov(const DevGeom& g, int loc) { return g.gcov[loc]; }
    static __device__ __forceinline__ const double* gcon(const DevGeom& g, int loc) { return g.gcon[loc]; }
    static __device__ __forceinline__ const double* gdet(const DevGeom& g, int loc) { return g.gdet[loc]; }
};
template <> struct FaceTables<float> {
    static __device__ __forceinline__ const float* gcov(const DevGeom& g, int loc) { return g.gcov_f[loc]; }
    static __device__ __forceinline__ const float* gcon(const DevGeom& g, int loc) { return g.gcon_f[loc]; }
    static __device__ __forceinline__ const float* gdet(const DevGeom& g, int loc) { return g.gdet_f[loc]; }
};

// Resident 128-thread blocks per SM requested from the compiler for each kernel (register caps
// of 65536 / (128 x blocks)), chosen by measurement on B200: FP64 faces 6 blocks along x1/x2 and 5
// along x3 (with the L2 prefetch of each zone's primitives; 5 and 4 before it), FP32 faces 8, the update half of the zone pass 4 (FP64 fluxes; no spills) or 5 (FP32
// fluxes) and its inversion half 5 (6 in the FP32-flux form, whose zone pass holds the metric's
// upper triangles only).  Each can be overridden at build time.
#ifndef KHB_FLUX64_MINB
#define KHB_FLUX64_MINB 6
#endif
#ifndef KHB_FLUX64_X3_MINB
#define KHB_FLUX64_X3_MINB 5
#endif
#ifndef KHB_FLUX32_MINB
#define KHB_FLUX32_MINB 8
#endif
#ifndef KHB_ZONE_UPDATE_MINB
#define KHB_ZONE_UPDATE_MINB 4
#endif
#ifndef KHB_ZONE_UPDATE32_MINB
#define KHB_ZONE_UPDATE32_MINB 5
#endif
#ifndef KHB_ZONE_CELL_MINB
#define KHB_ZONE_CELL_MINB 5
#endif
#ifndef KHB_ZONE_CELL32_MINB
#define KHB_ZONE_CELL32_MINB 6
#endif
#ifndef KHB_ZONE_INV_MINB
#define KHB_ZONE_INV_MINB 6
#endif
#ifndef KHB_ZONE_FLOOR_MINB
#define KHB_ZONE_FLOOR_MINB 6
#endif
template <typename R, int DIR> struct FluxMinBlocks { static constexpr int value = KHB_FLUX32_MINB; };
template <int DIR> struct FluxMinBlocks<double, DIR> {
    static constexpr int value = (DIR == 3) ? KHB_FLUX64_X3_MINB : KHB_FLUX64_MINB;
};
template <int MODE_, typename FT> struct ZoneMinBlocks {
    static constexpr int MODE = MODE_ & ~(M_KASTAUN | M_BCT);
    static constexpr int value = (MODE == M_UPDATE) ? (sizeof(FT) == 8 ? KHB_ZONE_UPDATE_MINB : KHB_ZONE_UPDATE32_MINB) :
                                 (MODE == M_UTOP) ? KHB_ZONE_INV_MINB :
                                 (MODE == M_ZONE_FLOORS) ? KHB_ZONE_FLOOR_MINB :
                                 ((MODE & M_UTOP) ? (sizeof(FT) == 8 ? KHB_ZONE_CELL_MINB : KHB_ZONE_CELL32_MINB) : 1);
};

// L2 prefetch of the line holding p (PTX prefetch.global.L2: a hint, no register result)
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

template <int DIR, int RECON, int NV, typename R, typename FT>
__device__ __forceinline__ void flux_face(const Dims& d, const DevGeom& g, const Phys& ph, const khb_fields& P,
                                          FT* __restrict__ F, FT* __restrict__ ctop, int i, int j, int k)
{
    constexpr int dir = DIR;
    const long long c = kchk(d, ((long long)k*d.n2 + j)*d.n1 + i, d.N, CHK_FLUX_STORE);
    const long long st = (dir == 1) ? 1 : ((dir == 2) ? d.sj : d.sk);
    const int loc = dir - 1;
    const R gam = (R)ph.gam;

    // FP64 faces: start the zone's own primitives towards L2 first (measured: 2.6% off the FP64
    // step; the FP32 faces, issue bound, do not gain)
    if (sizeof(R) == 8) {
#pragma unroll
        for (int p = 0; p < NV; ++p) prefetch_l2(P.v[p] + c);
    }
    // geometry at the face
    const long long gi = kchk(d, (long long)j*g.G1 + i, g.gs, CHK_GEOM);
    const auto* tcov = FaceTables<R>::gcov(g, loc);
    const auto* tcon = FaceTables<R>::gcon(g, loc);
    R gcov[4][4];
#pragma unroll
    for (int m = 0; m < 16; ++m) gcov[m/4][m%4] = (R)__ldg(tcov + m*g.gs + gi);
    R gcon0[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) gcon0[m] = (R)__ldg(tcon + m*g.gs + gi);
    const R gcondd = (R)__ldg(tcon + (dir*4 + dir)*g.gs + gi);
    const R gdet = (R)__ldg(FaceTables<R>::gdet(g, loc) + gi);

    // reconstruction: left state = right face of zone c-st, right state = left face of zone c
    R Pl[NV], Pr[NV];
    // WENO5 lowered to linear MC (reconstruction.hpp:694-771): near the X1 block edges for X1 faces
    // (zones within 4 of the first and 2 of the last interior zone, as ReconstructX1's split of the
    // [is-1, ie+2] zone range places them), or in the rows j <= 6 and j >= n2 - 6 for every direction
    bool mc_l = false, mc_r = false;
    if (RECON == RECON_WENO5X && ph.weno_lower) {
        if (ph.weno_lower == 1) {
            if (dir == 1) {
                mc_l = (i - 1 <= d.is + 3) || (i - 1 >= d.ie - 2);
                mc_r = (i <= d.is + 3) || (i >= d.ie - 2);
            }
        } else {
            mc_l = mc_r = !(j > 6 && j < d.n2 - 6);
        }
    }
#pragma unroll
    for (int p = 0; p < NV; ++p) {
        const double* q = P.v[p];
        const R x0 = (R)__ldg(q + kchk(d, c - 3*st, d.N, CHK_FLUX_STENCIL)), x1 = (R)__ldg(q + kchk(d, c - 2*st, d.N, CHK_FLUX_STENCIL));
        const R x2 = (R)__ldg(q + kchk(d, c - st, d.N, CHK_FLUX_STENCIL)), x3 = (R)__ldg(q + c);
        const R x4 = (R)__ldg(q + kchk(d, c + st, d.N, CHK_FLUX_STENCIL)), x5 = (R)__ldg(q + kchk(d, c + 2*st, d.N, CHK_FLUX_STENCIL));
        if (RECON == RECON_EXTRA) {
            Pl[p] = recon_extra<R>(ph.recon_extra, true, x0, x1, x2, x3, x4);
            Pr[p] = recon_extra<R>(ph.recon_extra, false, x1, x2, x3, x4, x5);
        } else if (RECON == RECON_WENO5X) {
            Pl[p] = mc_l ? recon_right<RECON_MC, R>(x0, x1, x2, x3, x4) : recon_right<RECON_WENO5, R>(x0, x1, x2, x3, x4);
            Pr[p] = mc_r ? recon_left<RECON_MC, R>(x1, x2, x3, x4, x5) : recon_left<RECON_WENO5, R>(x1, x2, x3, x4, x5);
        } else {
            Pl[p] = recon_right<RECON, R>(x0, x1, x2, x3, x4);
            Pr[p] = recon_left<RECON, R>(x1, x2, x3, x4, x5);
        }
    }
    constexpr bool HIGH = (RECON == RECON_WENO5X || RECON == RECON_EXTRA);
    if (ph.recon_floors || (HIGH && ph.recon_fallback)) {
        // floors_functions.hpp:301-333 applied to both reconstructed states (get_flux.hpp:174-181)
        const double rf = __ldg(g.floor_rho + (long long)j*g.n1 + i), uf = __ldg(g.floor_u + (long long)j*g.n1 + i);
        const bool hit = ((R)rf > Pl[0]) || ((R)uf > Pl[1]) || ((R)rf > Pr[0]) || ((R)uf > Pr[1]);
        Pl[0] += kmax(R(0), (R)rf - Pl[0]); Pl[1] += kmax(R(0), (R)uf - Pl[1]);
        Pr[0] += kmax(R(0), (R)rf - Pr[0]); Pr[1] += kmax(R(0), (R)uf - Pr[1]);
        if (HIGH && ph.recon_fallback && hit) {
            // reconstruction_fallback (get_flux.hpp:185-199): a face whose states hit the floors
            // takes the PPM states instead
#pragma unroll
            for (int p = 0; p < NV; ++p) {
                const double* q = P.v[p];
                const R x0 = (R)__ldg(q + kchk(d, c - 3*st, d.N, CHK_FLUX_STENCIL)), x1 = (R)__ldg(q + kchk(d, c - 2*st, d.N, CHK_FLUX_STENCIL));
                const R x2 = (R)__ldg(q + kchk(d, c - st, d.N, CHK_FLUX_STENCIL)), x3 = (R)__ldg(q + c);
                const R x4 = (R)__ldg(q + kchk(d, c + st, d.N, CHK_FLUX_STENCIL)), x5 = (R)__ldg(q + kchk(d, c + 2*st, d.N, CHK_FLUX_STENCIL));
                Pl[p] = recon_right<RECON_PPM, R>(x0, x1, x2, x3, x4);
                Pr[p] = recon_left<RECON_PPM, R>(x1, x2, x3, x4, x5);
            }
        }
    }

    constexpr bool HAS_B = NV > 5;
    FourVec<R> D;
    R Ul[NV], Fl[NV], Ur[NV], Fr[NV];
    R cmaxL, cminL, cmaxR, cminR;
    calc_4vecs<R, HAS_B>(gcov, gcon0[0], gcon0, Pl, D);
    prim_to_flux<R, NV>(Pl, D, gam, gdet, 0, Ul);
    prim_to_flux<R, NV>(Pl, D, gam, gdet, dir, Fl);
    vchar<R, HAS_B>(Pl, D, gam, gcon0[0], gcon0[dir], gcondd, dir, cmaxL, cminL);
    calc_4vecs<R, HAS_B>(gcov, gcon0[0], gcon0, Pr, D);
    prim_to_flux<R, NV>(Pr, D, gam, gdet, 0, Ur);
    prim_to_flux<R, NV>(Pr, D, gam, gdet, dir, Fr);
    vchar<R, HAS_B>(Pr, D, gam, gcon0[0], gcon0[dir], gcondd, dir, cmaxR, cminR);
    // get_flux.hpp:274-275, 330-331
    const R cmax = kmax(kmax(R(0), cmaxL), cmaxR);
    const R cmin = -kmin(kmin(R(0), cminL), cminR);
    if (ph.riemann == 0) {
        const R ctp = kmax(cmax, cmin);
#pragma unroll
        for (int p = 0; p < NV; ++p)
            F[p*d.N + c] = (FT)(R(0.5) * (Fl[p] + Fr[p] - ctp * (Ur[p] - Ul[p])));
    } else {
#pragma unroll
        for (int p = 0; p < NV; ++p)
            F[p*d.N + c] = (FT)((cmax*Fl[p] + cmin*Fr[p] - cmax*cmin*(Ur[p] - Ul[p])) / (cmax + cmin));
    }
    ctop[c] = (FT)kmax(cmax, cmin);
}

template <int DIR, int RECON, int NV, typename R, typename FT>
__global__ void __launch_bounds__(128, FluxMinBlocks<R, DIR>::value)
k_flux(Dims d, DevGeom g, Phys ph, khb_fields P, FT* __restrict__ F, FT* __restrict__ ctop, Box bx)
{
    int i, j, k;
    if (!box_cell(bx, blockIdx.x, i, j, k)) return;
    flux_face<DIR, RECON, NV, R, FT>(d, g, ph, P, F, ctop, i, j, k);
}

// ===================================================================================== flux fixes
// B_FluxCT::ZeroBoundaryFlux on X2 faces (b_flux_ct.cpp:404-430) and KBoundaries::FixFlux
// (boundaries.cpp:611-690) for inflow checks on X1 faces and zero polar fluxes on X2 faces.
// One thread per (k, i) of an X2 face or (k, j) of an X1 face; the halo is one zone.
template <int NV, typename FT>
__device__ __forceinline__ void fix_x2_zone(const Dims& d, const Phys& ph, FT* F1, FT* F2, FT* F3, int inner, int t)
{
    const int ni = d.ie - d.is + 3;
    const int nk = (d.ndim > 2) ? d.ke - d.ks + 3 : 1;
    if (t >= ni*nk) return;
    const int i = d.is - 1 + t % ni;
    const int k = (d.ndim > 2) ? d.ks - 1 + t / ni : d.ks;
    const int j = inner ? d.js : d.je + 1;
    const long long c = ((long long)k*d.n2 + j)*d.n1 + i;
    const long long N = d.N;
    if (NV > 5 && ph.fix_polar_flux) {
        F2[5*N + c] = (FT)0; F2[7*N + c] = (FT)0;
        if (inner) {
            F1[6*N + c - d.sj] = -F1[6*N + c];
            if (d.ndim > 2) F3[6*N + c - d.sj] = -F3[6*N + c];
        } else {
            F1[6*N + c] = -F1[6*N + c - d.sj];
            if (d.ndim > 2) F3[6*N + c] = -F3[6*N + c - d.sj];
        }
    }
    if (ph.zero_polar_flux)
#pragma unroll
        for (int p = 0; p < NV; ++p) F2[p*N + c] = (FT)0;
}
template <int NV, typename FT>
__global__ void k_fix_flux_x2(Dims d, Phys ph, FT* F1, FT* F2, FT* F3, int inner)
{
    fix_x2_zone<NV, FT>(d, ph, F1, F2, F3, inner, blockIdx.x * blockDim.x + threadIdx.x);
}
template <typename FT>
__device__ __forceinline__ void fix_x1_zone(const Dims& d, FT* F1, int inner, int t)
{
    const int nj = (d.ndim > 1) ? d.je - d.js + 3 : 1;
    const int nk = (d.ndim > 2) ? d.ke - d.ks + 3 : 1;
    if (t >= nj*nk) return;
    const int j = (d.ndim > 1) ? d.js - 1 + t % nj : d.js;
    const int k = (d.ndim > 2) ? d.ks - 1 + t / nj : d.ks;
    const int i = inner ? d.is : d.ie + 1;
    const long long c = ((long long)k*d.n2 + j)*d.n1 + i;
    FT& f = F1[c];
    f = inner ? kmin(f, (FT)0) : kmax(f, (FT)0);
}
template <typename FT>
__global__ void k_fix_flux_x1(Dims d, FT* F1, int inner)
{
    fix_x1_zone<FT>(d, F1, inner, blockIdx.x * blockDim.x + threadIdx.x);
}
// The flux fixes of every block of a batch in one launch: blockIdx.y picks a block's fix (its faces
// and slots are disjoint from every other fix's)
template <int NV, typename FT>
__global__ void __launch_bounds__(128) k_fix_tasks(const FixTask<FT>* __restrict__ tasks)
{
    const FixTask<FT>& T = tasks[blockIdx.y];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (T.x1) fix_x1_zone<FT>(T.d, T.F1, T.inner, t);
    else fix_x2_zone<NV, FT>(T.d, T.ph, T.F1, T.F2, T.F3, T.inner, t);
}

// ===================================================================================== zone pass

// Raw flux, as double
template <typename FT>
__device__ __forceinline__ double ldf(const FT* F, long long x) { return (double)__ldg(F + x); }

// Divergence of the B fluxes with flux-CT applied on the fly (b_flux_ct.cpp:307-370): corner EMFs
// from the raw B fluxes in FT arithmetic, the face B fluxes from the EMFs, then -div over the zone.
// F1..F3 hold nvar-major fluxes with the B components in slots 5-7 (stride d.N).
template <typename FT>
__device__ __forceinline__ void ct_divergence(const Dims& d, const Phys& ph, const FT* F1, const FT* F2, const FT* F3,
                                              long long c, int j, double dudt_b[3])
{
    const long long N = d.N, sj = d.sj, sk = d.sk;
    const double a1 = ph.dx2*ph.dx3, a2 = ph.dx1*ph.dx3, a3 = ph.dx1*ph.dx2;
    const double vol = ph.dx1*ph.dx2*ph.dx3;
    double fb[3][3][2];   // [face dir][B component][lo/hi face]
    if (d.ndim >= 2) {
        const long long B1 = 5*N, B2 = 6*N, B3 = 7*N;
        // corner EMFs; the checked build verifies the furthest reaches of each (x itself, x - sj or
        // x - sk, x - 1) against the field's extent
        auto e3 = [&](long long x) -> FT {
            x = kchk(d, x, N, CHK_ZONE_CT); kchk(d, x - sj, N, CHK_ZONE_CT); kchk(d, x - 1, N, CHK_ZONE_CT);
            return (FT)0.25 * (__ldg(F1 + B2 + x) + __ldg(F1 + B2 + x - sj) - __ldg(F2 + B1 + x) - __ldg(F2 + B1 + x - 1));
        };
        auto e1 = [&](long long x) -> FT {
            x = kchk(d, x, N, CHK_ZONE_CT); kchk(d, x - sk, N, CHK_ZONE_CT); kchk(d, x - sj, N, CHK_ZONE_CT);
            return (FT)0.25 * (__ldg(F2 + B3 + x) + __ldg(F2 + B3 + x - sk) - __ldg(F3 + B2 + x) - __ldg(F3 + B2 + x - sj));
        };
        auto e2 = [&](long long x) -> FT {
            x = kchk(d, x, N, CHK_ZONE_CT); kchk(d, x - 1, N, CHK_ZONE_CT); kchk(d, x - sk, N, CHK_ZONE_CT);
            return (FT)0.25 * (__ldg(F3 + B1 + x) + __ldg(F3 + B1 + x - 1) - __ldg(F1 + B3 + x) - __ldg(F1 + B3 + x - sk));
        };
        const bool d3 = d.ndim > 2;
        // X1 faces i (lo) and i+1 (hi)
        fb[0][0][0] = 0.; fb[0][0][1] = 0.;
        fb[0][1][0] = (double)((FT)0.5 * (e3(c) + e3(c + sj)));
        fb[0][1][1] = (double)((FT)0.5 * (e3(c + 1) + e3(c + 1 + sj)));
        fb[0][2][0] = d3 ? (double)((FT)-0.5 * (e2(c) + e2(c + sk))) : ldf(F1, B3 + c);
        fb[0][2][1] = d3 ? (double)((FT)-0.5 * (e2(c + 1) + e2(c + 1 + sk))) : ldf(F1, B3 + c + 1);
        // X2 faces j, j+1
        fb[1][0][0] = (double)((FT)-0.5 * (e3(c) + e3(c + 1)));
        fb[1][0][1] = (double)((FT)-0.5 * (e3(c + sj) + e3(c + sj + 1)));
        fb[1][1][0] = 0.; fb[1][1][1] = 0.;
        fb[1][2][0] = d3 ? (double)((FT)0.5 * (e1(c) + e1(c + sk))) : ldf(F2, B3 + c);
        fb[1][2][1] = d3 ? (double)((FT)0.5 * (e1(c + sj) + e1(c + sj + sk))) : ldf(F2, B3 + c + sj);
        // KBoundaries zero_polar_flux after flux-CT (boundaries.cpp:672-684)
        if (ph.zero_polar_flux) {
            if (j == d.js && phys_face(d.bc[2])) { fb[1][0][0] = 0.; fb[1][1][0] = 0.; fb[1][2][0] = 0.; }
            if (j == d.je && phys_face(d.bc[3])) { fb[1][0][1] = 0.; fb[1][1][1] = 0.; fb[1][2][1] = 0.; }
        }
        if (d3) {
            fb[2][0][0] = (double)((FT)0.5 * (e2(c) + e2(c + 1)));
            fb[2][0][1] = (double)((FT)0.5 * (e2(c + sk) + e2(c + sk + 1)));
            fb[2][1][0] = (double)((FT)-0.5 * (e1(c) + e1(c + sj)));
            fb[2][1][1] = (double)((FT)-0.5 * (e1(c + sk) + e1(c + sk + sj)));
            fb[2][2][0] = 0.; fb[2][2][1] = 0.;
        }
    } else {
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            fb[0][v][0] = ldf(F1, (5 + v)*N + c);
            fb[0][v][1] = ldf(F1, (5 + v)*N + c + 1);
        }
    }
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        double du = (a1 * fb[0][v][1] - a1 * fb[0][v][0]);
        if (d.ndim >= 2) du += a2 * fb[1][v][1] - a2 * fb[1][v][0];
        if (d.ndim == 3) du += a3 * fb[2][v][1] - a3 * fb[2][v][0];
        dudt_b[v] = -du / vol;
    }
}

// B_CT::BlockUtoP for one zone (b_ct.cpp:172-181): the zone B^i as the average of its two faces'
// B^i = Bf / sqrt(-g)(face); along an inactive direction the single face's value
__device__ __forceinline__ void ct_zone_b(const Dims& d, const DevGeom& g, const double* const Bf[3], long long c,
                                          int j, int i, double Bp[3])
{
    const long long gi = (long long)j*g.G1 + i;
    Bp[0] = (__ldg(Bf[0] + c) / __ldg(g.gdet[0] + gi) + __ldg(Bf[0] + c + 1) / __ldg(g.gdet[0] + gi + 1)) / 2;
    Bp[1] = (d.ndim > 1) ? (__ldg(Bf[1] + c) / __ldg(g.gdet[1] + gi) + __ldg(Bf[1] + c + d.sj) / __ldg(g.gdet[1] + gi + g.G1)) / 2
                         : __ldg(Bf[1] + c) / __ldg(g.gdet[1] + gi);
    Bp[2] = (d.ndim > 2) ? (__ldg(Bf[2] + c) / __ldg(g.gdet[2] + gi) + __ldg(Bf[2] + c + d.sk) / __ldg(g.gdet[2] + gi)) / 2
                         : __ldg(Bf[2] + c) / __ldg(g.gdet[2] + gi);
}

// ct_zone_b for any zone of the block: the last layer of a direction (i = n1-1, j = n2-1, k = n3-1)
// takes its lower face alone, as k_ghost_ptou does
__device__ __forceinline__ void ct_zone_b_edge(const Dims& d, const DevGeom& g, const double* const Bf[3], long long c,
                                               int j, int i, int k, double Bp[3])
{
    const long long gi = (long long)j*g.G1 + i;
    Bp[0] = (i == d.n1 - 1) ? __ldg(Bf[0] + c) / __ldg(g.gdet[0] + gi)
                            : (__ldg(Bf[0] + c) / __ldg(g.gdet[0] + gi) + __ldg(Bf[0] + c + 1) / __ldg(g.gdet[0] + gi + 1)) / 2;
    Bp[1] = (d.ndim > 1 && j < d.n2 - 1) ? (__ldg(Bf[1] + c) / __ldg(g.gdet[1] + gi) + __ldg(Bf[1] + c + d.sj) / __ldg(g.gdet[1] + gi + g.G1)) / 2
                                         : __ldg(Bf[1] + c) / __ldg(g.gdet[1] + gi);
    Bp[2] = (d.ndim > 2 && k < d.n3 - 1) ? (__ldg(Bf[2] + c) / __ldg(g.gdet[2] + gi) + __ldg(Bf[2] + c + d.sk) / __ldg(g.gdet[2] + gi)) / 2
                                         : __ldg(Bf[2] + c) / __ldg(g.gdet[2] + gi);
}

// The geometric source of one zone (flux.cpp:413-441): new_du[lam] = sum over mu, nu of
// T^mu_nu gdet Gamma^nu_lam mu for the UU and U1-U3 components, from the zone's primitives Ps
template <int NV>
__device__ __forceinline__ void geo_source(const Dims& d, const DevGeom& g, const ZoneGeom& G, double gam,
                                           const double* Ps, int j, int i, double new_du[4])
{
    FourVec<double> D;
    const double gcon0[4] = {G.gcon[0][0], G.gcon[0][1], G.gcon[0][2], G.gcon[0][3]};
    calc_4vecs<double, (NV > 5)>(G.gcov, G.gcon[0][0], gcon0, Ps, D);
#pragma unroll
    for (int lam = 0; lam < 4; ++lam) new_du[lam] = 0.;
    const long long cg = (long long)j*g.n1 + i, cs = (long long)(d.n2)*g.n1;
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
        double Tmu[4];
        calc_tensor<double, (NV > 5)>(Ps[0], Ps[1], (gam - 1) * Ps[1], D, mu, Tmu);
#pragma unroll
        for (int nu = 0; nu < 4; ++nu)
#pragma unroll
            for (int lam = 0; lam < 4; ++lam)
                new_du[lam] += Tmu[nu] * __ldg(g.gdet_conn + ((nu*4 + lam)*4 + mu)*cs + cg);
    }
}

// MODE: compile-time mask of M_* steps (0: take the mask from the arguments at run time).  The
// CFL reduction (M_DT) is always a run-time choice.
// One zone of the zone pass; returns the zone's timestep for the CFL minimum (DBL_MAX if none)
template <int NV, typename FT, int MODE>
__device__ __forceinline__ double zone_body(const Dims& d, const DevGeom& g, const Phys& ph, const ZoneArgs<FT>& a,
                                            int i, int j, int k)
{
    const int mode = MODE ? (MODE | (a.mode & M_DT)) : a.mode;
    double ndt_zone = 1.7976931348623157e308;
    {
        const long long c = kchk(d, ((long long)k*d.n2 + j)*d.n1 + i, d.N, CHK_ZONE_FLUX);
        const long long N = d.N, sj = d.sj, sk = d.sk;
        const double gam = ph.gam;
        kchk(d, c + 1, N, CHK_ZONE_FLUX);
        if (d.ndim >= 2) kchk(d, c + sj, N, CHK_ZONE_FLUX);
        if (d.ndim == 3) kchk(d, c + sk, N, CHK_ZONE_FLUX);
        kchk(d, (long long)j*g.G1 + i, g.gs, CHK_GEOM);
        ZoneGeom G;
        load_zone_geom<(sizeof(FT) == 4)>(g, j, i, G);

        double U[NV], P[NV];
        if (mode & M_UPDATE) {
            // ---- flux divergence (Parthenon FluxDivHelper) with flux-CT B fluxes
            const double a1 = ph.dx2*ph.dx3, a2 = ph.dx1*ph.dx3, a3 = ph.dx1*ph.dx2;
            const double vol = ph.dx1*ph.dx2*ph.dx3;
            const FT* F1 = a.F[0]; const FT* F2 = a.F[1]; const FT* F3 = a.F[2];
            // the zone's own values come from DRAM: start them towards L2 before the register-bound
            // loads below (no registers held, results unchanged)
#pragma unroll
            for (int p = 0; p < NV; ++p) {
                prefetch_l2(a.Us.v[p] + c);
                prefetch_l2(a.U0.v[p] + c);
                prefetch_l2(F1 + p*N + c);
                if (d.ndim >= 2) prefetch_l2(F2 + p*N + c);
                if (d.ndim == 3) prefetch_l2(F3 + p*N + c);
                if (!ph.cart_minkowski) prefetch_l2(a.Ps.v[p] + c);
                if (sizeof(FT) == 8) {
                    // FP64 fluxes: the upper x2/x3 faces too (measured 0.5% off the FP64 step; the FP32
                    // form, whose flux lines are half as many, loses 4% with them)
                    if (d.ndim >= 2) prefetch_l2(F2 + p*N + c + sj);
                    if (d.ndim == 3) prefetch_l2(F3 + p*N + c + sk);
                }
            }
            double dudt[NV];
            constexpr int NH = 5;
#pragma unroll
            for (int p = 0; p < NH; ++p) {
                double du = (a1 * ldf(F1, p*N + c + 1) - a1 * ldf(F1, p*N + c));
                if (d.ndim >= 2) du += a2 * ldf(F2, p*N + c + sj) - a2 * ldf(F2, p*N + c);
                if (d.ndim == 3) du += a3 * ldf(F3, p*N + c + sk) - a3 * ldf(F3, p*N + c);
                dudt[p] = -du / vol;
            }
            if (NV > 5) {
                double dudt_b[3] = {0., 0., 0.};
                // with B_CT the zone B follows the faces (below) and has no flux divergence
                if (!(mode & M_BCT)) ct_divergence<FT>(d, ph, F1, F2, F3, c, j, dudt_b);
#pragma unroll
                for (int v = 0; v < 3; ++v) dudt[5 + v] = dudt_b[v];
            }
            // ---- geometric source, flux.cpp:395-444
            if (!ph.cart_minkowski) {
                double Ps[NV];
#pragma unroll
                for (int p = 0; p < NV; ++p) Ps[p] = __ldg(a.Ps.v[p] + c);
                double new_du[4];
                geo_source<NV>(d, g, G, gam, Ps, j, i, new_du);
                dudt[1] += new_du[0];
                dudt[2] += new_du[1];
                dudt[3] += new_du[2];
                dudt[4] += new_du[3];
            }
            // ---- RK combination (Parthenon WeightedSumData twice, kharma_driver.cpp:339-387)
            const double bdt = a.dt_dev ? a.beta * __ldg(a.dt_dev) : a.bdt;
#pragma unroll
            for (int p = 0; p < NV; ++p) {
                double x = a.g0 * __ldg(a.Us.v[p] + c) + a.g1 * __ldg(a.U0.v[p] + c);
                U[p] = 1.0 * x + bdt * dudt[p];
            }
            if (NV > 5 && (mode & M_BCT)) {
                // B_CT::BlockUtoP on the updated faces: sqrt(-g) B^i at the zone centre
                double Bp[3];
                ct_zone_b(d, g, a.Bf, c, j, i, Bp);
#pragma unroll
                for (int v = 0; v < 3; ++v) U[5 + v] = Bp[v] * G.gdet;
            }
        } else {
#pragma unroll
            for (int p = 0; p < NV; ++p) U[p] = a.Us.v[p][c];
            if (NV > 5 && (MODE & M_GHOSTB) && (mode & M_BCT)) {
                // B_CT::BlockUtoP over the entire block before the inversion (b_ct.cpp:160-188)
                double Bp[3];
                ct_zone_b_edge(d, g, a.Bf, c, j, i, k, Bp);
#pragma unroll
                for (int v = 0; v < 3; ++v) U[5 + v] = Bp[v] * G.gdet;
            }
        }

        int pflag = 0, fflag = 0;
        FourVec<double> D;
        bool have_D = false;
#pragma unroll
        for (int p = 0; p < NV; ++p) P[p] = a.Ps.v[p][c];
        if (mode & M_UTOP) {
            // inverter.cpp:163-181 then b_flux_ct.cpp:196-217
            const int pf = (mode & M_KASTAUN) ? u_to_p_kastaun<NV>(G, gam, floors_at(ph, g, j, i), U, P, ph.iter_max, ph.err_tol)
                                              : u_to_p_onedw<NV, (sizeof(FT) == 4)>(G, gam, U, P, ph.iter_max, ph.err_tol);
            pflag = pf % FF_GEOM_RHO;
            fflag = (pf / FF_GEOM_RHO) * FF_GEOM_RHO;
            if (NV > 5) {
                if (mode & M_BCT) {
                    double Bp[3];
                    if (MODE & M_GHOSTB) ct_zone_b_edge(d, g, a.Bf, c, j, i, k, Bp);
                    else ct_zone_b(d, g, a.Bf, c, j, i, Bp);
#pragma unroll
                    for (int v = 0; v < 3; ++v) P[5 + v] = Bp[v];
                } else {
#pragma unroll
                    for (int v = 0; v < 3; ++v) P[5 + v] = U[5 + v] / G.gdet;
                }
            }
        } else {
            pflag = a.pflag[c];
            fflag = a.fflag[c];
        }
        if ((mode & M_UTOP) && (mode & (M_FLOORS | M_PTOU))) {
            // reload the metric for floors and P->U instead of holding it through the inversion
            // (the compiler barrier keeps the reload; measured 0.4% / 1.3% off the FP64 / FP32 step)
            asm volatile("" ::: "memory");
            load_zone_geom<(sizeof(FT) == 4)>(g, j, i, G);
        }
        if ((mode & M_FLOORS) && ph.floors_on) {
            // floors.cpp:215-229 and floors_impl.hpp:77-125
            double rf, uf;
            const long long cg = (long long)j*g.n1 + i;
            const Prescription& fl = floors_at(ph, g, j, i);
            fflag |= determine_floors<NV>(G, fl, __ldg(g.floor_rho + cg), __ldg(g.floor_u + cg), gam, P, rf, uf, D);
            if (fflag) {
                // mixed frames (floors_impl.hpp:84-106): by radius, or by min(rho, u)/b^2 of the
                // state before the floors
                int frame = ph.frame;
                if (frame == KHB_FRAME_MIXED_FLUID_NORMAL) {
                    frame = (__ldg(g.rcen + cg) > ph.frame_switch_r) ? KHB_FRAME_FLUID : KHB_FRAME_NORMAL;
                } else if (frame == KHB_FRAME_MIXED_NORMAL_DRIFT) {
                    const double mag_switch = kmin(P[0], P[1]) / dot4(D.bcon, D.bcov);
                    frame = (mag_switch < ph.frame_switch_beta) ? KHB_FRAME_DRIFT : KHB_FRAME_NORMAL;
                }
                const int pl = apply_floors_frame<NV>(G, frame, gam, P, U, rf, uf, 8, &D);
                if (pl) pflag = pl;
                apply_ceilings(G, fl, gam, P);
                // the fluid part of U(P) after the floors; the lock-step P->U below computes the same
                // values from the same P, so it is formed here only when that step is not part of the pass
                if (!(mode & M_PTOU)) {
                    double Ut[NV];
                    p_to_u_zone<NV>(G, gam, P, Ut);
#pragma unroll
                    for (int p = 0; p < 5; ++p) U[p] = Ut[p];
                }
            } else {
                have_D = true;   // P is unchanged: its 4-vectors serve the P->U below
            }
        }
        if (mode & M_PTOU) {
            if (have_D) prim_to_flux<double, NV>(P, D, gam, G.gdet, 0, U);
            else p_to_u_zone<NV>(G, gam, P, U);
        }

        if (mode & (M_UPDATE | M_FLOORS | M_PTOU)) {
#pragma unroll
            for (int p = 0; p < NV; ++p) a.Uout.v[p][c] = U[p];
        }
        if (mode & (M_UTOP | M_FLOORS)) {
#pragma unroll
            for (int p = 0; p < NV; ++p) a.Pout.v[p][c] = P[p];
            a.pflag[c] = pflag;
            a.fflag[c] = fflag;
        }
        if ((mode & M_FAILLIST) && pflag > 0) {
            const int slot = atomicAdd(a.fail_count, 1);
            a.fail_list[slot] = (int)c;
        }
        if (mode & M_DT) {
            // grmhd.cpp:313-328
            const double c1 = kmax((double)a.ctop[0][c], 0.0), c2 = kmax((double)a.ctop[1][c], 0.0);
            const double c3 = kmax((double)a.ctop[2][c], 0.0);
            const double z = 1.0 / (1 / (ph.dx1 / c1) + 1 / (ph.dx2 / c2) + 1 / (ph.dx3 * 1 / c3));
            if (!isnan(z)) ndt_zone = z;
        }
    }
    return ndt_zone;
}

// Block minimum of the zone timesteps by warp shuffles, then one atomic per block on the bit
// pattern (values >= 0).  Every thread of the 128-thread block must call it.
__device__ __forceinline__ void block_min_ndt(double v, unsigned long long* word)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    __shared__ double wmin[4];
    if ((threadIdx.x & 31) == 0) wmin[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = wmin[0];
        for (int w = 1; w < 4; ++w) m = fmin(m, wmin[w]);
        if (m >= 0.0) atomicMin(word, (unsigned long long)__double_as_longlong(m));
    }
}

template <int NV, typename FT, int MODE>
__global__ void __launch_bounds__(128, ZoneMinBlocks<MODE, FT>::value)
k_zone(Dims d, DevGeom g, Phys ph, ZoneArgs<FT> a, Box bx)
{
    int i, j, k;
    double ndt_zone = 1.7976931348623157e308;
    if (box_cell(bx, blockIdx.x, i, j, k)) ndt_zone = zone_body<NV, FT, MODE>(d, g, ph, a, i, j, k);
    if (a.mode & M_DT) block_min_ndt(ndt_zone, a.ndt_word);
}

// ===================================================================================== FOFC
// First-order flux correction (flux/fofc.cpp:45-226, driver/kharma_driver.cpp:292-337), between the
// flux calculation and the flux fixes.  The guess update of each zone uses the raw face fluxes as
// they stand (faces outside the flux calculation's range hold zeros or earlier corrections, as in the
// reference), starts its inversion from P_s, and flags zones that would hit floors or lie within
// fofc_r_mark of the centre (event horizon plus buffer).
template <int NV, typename FT, bool KAST>
__global__ void __launch_bounds__(128) k_fofc_guess(Dims d, DevGeom g, Phys ph, khb_fields Ps, khb_fields Us,
                                                    khb_fields U0, const FT* F1, const FT* F2, const FT* F3,
                                                    double g0, double g1, double bdt_host, const double* dt_dev,
                                                    double beta, int32_t* flag, Box bx)
{
    int i, j, k;
    if (!box_cell(bx, blockIdx.x, i, j, k)) return;
    const double bdt = dt_dev ? beta * __ldg(dt_dev) : bdt_host;
    const long long c = ((long long)k*d.n2 + j)*d.n1 + i;
    const long long N = d.N, sj = d.sj, sk = d.sk;
    const double a1 = ph.dx2*ph.dx3, a2 = ph.dx1*ph.dx3, a3 = ph.dx1*ph.dx2;
    const double vol = ph.dx1*ph.dx2*ph.dx3;
    ZoneGeom G;
    load_zone_geom(g, j, i, G);
    double Ug[NV], Pg[NV], dudt[NV];
#pragma unroll
    for (int p = 0; p < NV; ++p) {
        double du = (a1 * ldf(F1, p*N + c + 1) - a1 * ldf(F1, p*N + c));
        if (d.ndim >= 2) du += a2 * ldf(F2, p*N + c + sj) - a2 * ldf(F2, p*N + c);
        if (d.ndim == 3) du += a3 * ldf(F3, p*N + c + sk) - a3 * ldf(F3, p*N + c);
        dudt[p] = -du / vol;
        Pg[p] = Ps.v[p][c];
    }
    // fofc/use_source_term: the guess also takes the geometric source of P_s (kharma_driver.cpp:308-312)
    if (ph.fofc_source && !ph.cart_minkowski) {
        double new_du[4];
        geo_source<NV>(d, g, G, ph.gam, Pg, j, i, new_du);
#pragma unroll
        for (int v = 0; v < 4; ++v) dudt[1 + v] += new_du[v];
    }
#pragma unroll
    for (int p = 0; p < NV; ++p) {
        const double x = g0 * Us.v[p][c] + g1 * U0.v[p][c];
        Ug[p] = 1.0 * x + bdt * dudt[p];
    }
    if (NV > 5) {
#pragma unroll
        for (int v = 0; v < 3; ++v) Pg[5 + v] = Ug[5 + v] / G.gdet;
    }
    const int pf = KAST ? u_to_p_kastaun<NV>(G, ph.gam, floors_at(ph, g, j, i), Ug, Pg, ph.iter_max, ph.err_tol)
                        : u_to_p_onedw<NV>(G, ph.gam, Ug, Pg, ph.iter_max, ph.err_tol);
    int ff = (pf / FF_GEOM_RHO) * FF_GEOM_RHO;
    if (ph.floors_on) {
        const long long cg = (long long)j*g.n1 + i;
        double rf, uf;
        FourVec<double> D;
        ff |= determine_floors<NV>(G, floors_at(ph, g, j, i), __ldg(g.floor_rho + cg), __ldg(g.floor_u + cg), ph.gam, Pg, rf, uf, D);
    }
    const bool eh = ph.spherical && __ldg(g.rcen + (long long)j*g.n1 + i) < ph.fofc_r_mark;
    flag[c] = (ff != 0 || eh) ? 1 : 0;
}
// Rows [j0, j1] of every (k, i) flagged (fofc/polar_cells next to a physical X2 face)
static __global__ void k_fofc_rows(Dims d, int j0, int j1, int32_t* flag)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long rows = (long long)(j1 - j0 + 1) * d.n1;
    if (t >= rows * d.n3) return;
    const int k = (int)(t / rows);
    const long long r = t - (long long)k * rows;
    const int j = j0 + (int)(r / d.n1), i = (int)(r % d.n1);
    flag[((long long)k*d.n2 + j)*d.n1 + i] = 1;
}
// Flags of zones outside the interior in periodic directions from their images (the flag's sync)
static __global__ void k_fofc_periodic(Dims d, int pmask, int32_t* flag)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= d.N) return;
    int k, j, i;
    zone_kji(d, t, k, j, i);
    int ii = i, jj = j, kk = k;
    bool any = false;
    if ((pmask & 1) && (i < d.is || i > d.ie)) { ii += (i < d.is) ? d.nx1 : -d.nx1; any = true; }
    if ((pmask & 2) && (j < d.js || j > d.je)) { jj += (j < d.js) ? d.nx2 : -d.nx2; any = true; }
    if ((pmask & 4) && (k < d.ks || k > d.ke)) { kk += (k < d.ks) ? d.nx3 : -d.nx3; any = true; }
    if (!any) return;
    flag[t] = flag[((long long)kk*d.n2 + jj)*d.n1 + ii];
}
// Donor-cell LLF flux (all variables) on each face of the box bordering a flagged zone (fofc.cpp:159-219)
template <int DIR, int NV, typename R, typename FT>
__global__ void __launch_bounds__(128) k_fofc_replace(Dims d, DevGeom g, Phys ph, khb_fields P, FT* __restrict__ F,
                                                      FT* __restrict__ ctop, const int32_t* __restrict__ flag, Box bx)
{
    int i, j, k;
    if (!box_cell(bx, blockIdx.x, i, j, k)) return;
    const long long c = ((long long)k*d.n2 + j)*d.n1 + i;
    const long long st = (DIR == 1) ? 1 : ((DIR == 2) ? d.sj : d.sk);
    if (!(flag[c] || flag[c - st])) return;
    const int loc = DIR - 1;
    const R gam = (R)ph.gam;
    const long long gi = (long long)j*g.G1 + i;
    const auto* tcov = FaceTables<R>::gcov(g, loc);
    const auto* tcon = FaceTables<R>::gcon(g, loc);
    R gcov[4][4], gcon0[4];
#pragma unroll
    for (int m = 0; m < 16; ++m) gcov[m/4][m%4] = (R)__ldg(tcov + m*g.gs + gi);
#pragma unroll
    for (int m = 0; m < 4; ++m) gcon0[m] = (R)__ldg(tcon + m*g.gs + gi);
    const R gcondd = (R)__ldg(tcon + (DIR*4 + DIR)*g.gs + gi);
    const R gdet = (R)__ldg(FaceTables<R>::gdet(g, loc) + gi);
    R Pl[NV], Pr[NV];
#pragma unroll
    for (int p = 0; p < NV; ++p) { Pl[p] = (R)P.v[p][c - st]; Pr[p] = (R)P.v[p][c]; }
    constexpr bool HAS_B = NV > 5;
    FourVec<R> D;
    R Ul[NV], Fl[NV], Ur[NV], Fr[NV], cmaxL, cminL, cmaxR, cminR;
    calc_4vecs<R, HAS_B>(gcov, gcon0[0], gcon0, Pl, D);
    prim_to_flux<R, NV>(Pl, D, gam, gdet, 0, Ul);
    prim_to_flux<R, NV>(Pl, D, gam, gdet, DIR, Fl);
    vchar<R, HAS_B>(Pl, D, gam, gcon0[0], gcon0[DIR], gcondd, DIR, cmaxL, cminL);
    calc_4vecs<R, HAS_B>(gcov, gcon0[0], gcon0, Pr, D);
    prim_to_flux<R, NV>(Pr, D, gam, gdet, 0, Ur);
    prim_to_flux<R, NV>(Pr, D, gam, gdet, DIR, Fr);
    vchar<R, HAS_B>(Pr, D, gam, gcon0[0], gcon0[DIR], gcondd, DIR, cmaxR, cminR);
    // fofc/use_glf: the speed-of-light Lax-Friedrichs speeds (fofc.cpp:200-205)
    const R cmax = ph.fofc_glf ? R(1) : kmax(kmax(R(0), cmaxL), cmaxR);
    const R cmin = ph.fofc_glf ? R(1) : -kmin(kmin(R(0), cminL), cminR);
    const R ctp = kmax(cmax, cmin);
#pragma unroll
    for (int p = 0; p < NV; ++p) F[p*d.N + c] = (FT)(R(0.5) * (Fl[p] + Fr[p] - ctp * (Ur[p] - Ul[p])));
    ctop[c] = (FT)ctp;
}

// ===================================================================================== fixups
// fixup.cpp:47-156.  Neighbours in periodic directions wrap; across exchanged x3 faces they are
// read from the ghost planes; in other directions they must be interior.  Failed zones never read each other, so one pass over the list is race-free.
template <int NV>
__device__ __forceinline__ void fixup_zone(const Dims& d, const DevGeom& g, const Phys& ph, const khb_fields& P,
                                           const khb_fields& U, const int32_t* pflag, long long c)
{
    {
        int k, j, i;
        zone_kji(d, c, k, j, i);
        // the list holds interior zones only; anything else is skipped, since its neighbours across an
        // exchange face would lie outside the block
        if (c < 0 || c >= d.N || i < d.is || i > d.ie || j < d.js || j > d.je || k < d.ks || k > d.ke) return;
        double wsum = 0., sum[5] = {0., 0., 0., 0., 0.};
        if (ph.fix_avg) {
            for (int nn = -1; nn <= 1; nn++) for (int m = -1; m <= 1; m++) for (int l = -1; l <= 1; l++) {
                int ii = i + l, jj = j + m, kk = k + nn;
                // exchanged faces hold the neighbouring block's values in the ghost zones;
                // periodic directions wrap; other faces end the neighbourhood
                if (ii < d.is || ii > d.ie) {
                    const int bc = d.bc[(ii < d.is) ? 0 : 1];
                    if (bc == KHB_BC_PERIODIC) ii += (ii < d.is) ? d.nx1 : -d.nx1;
                    else if (bc != KHB_BC_EXCHANGE) continue;
                }
                if (jj < d.js || jj > d.je) {
                    const int bc = d.bc[(jj < d.js) ? 2 : 3];
                    if (d.ndim < 2) continue;
                    if (bc == KHB_BC_PERIODIC) jj += (jj < d.js) ? d.nx2 : -d.nx2;
                    else if (bc != KHB_BC_EXCHANGE) continue;
                }
                if (kk < d.ks || kk > d.ke) {
                    const int bc = d.bc[(kk < d.ks) ? 4 : 5];
                    if (d.ndim < 3) continue;
                    if (bc == KHB_BC_PERIODIC) kk += (kk < d.ks) ? d.nx3 : -d.nx3;
                    else if (bc != KHB_BC_EXCHANGE) continue;
                }
                const long long cn = kchk(d, ((long long)kk*d.n2 + jj)*d.n1 + ii, d.N, CHK_FIXUP);
                if (!(pflag[cn] > 0)) {
                    const double w = 1./(abs(l) + abs(m) + abs(nn) + 1);
                    wsum += w;
#pragma unroll
                    for (int p = 0; p < 5; ++p) sum[p] += w * P.v[p][cn];
                }
            }
        }
        double Pz[NV], Uz[NV];
#pragma unroll
        for (int p = 0; p < 5; ++p) Pz[p] = (wsum < 1.e-10) ? 0. : sum[p]/wsum;
#pragma unroll
        for (int p = 5; p < NV; ++p) Pz[p] = P.v[p][c];
        const double rf = g.floor_rho[(long long)j*g.n1 + i], uf = g.floor_u[(long long)j*g.n1 + i];
        Pz[0] += kmax(0., rf - Pz[0]);
        Pz[1] += kmax(0., uf - Pz[1]);
        ZoneGeom G;
        load_zone_geom(g, j, i, G);
        p_to_u_zone<NV>(G, ph.gam, Pz, Uz);
#pragma unroll
        for (int p = 0; p < 5; ++p) P.v[p][c] = Pz[p];
#pragma unroll
        for (int p = 0; p < NV; ++p) U.v[p][c] = Uz[p];
    }
}

template <int NV>
__global__ void k_fixup(Dims d, DevGeom g, Phys ph, khb_fields P, khb_fields U, const int32_t* pflag,
                        const int* fail_count, const int* fail_list)
{
    const int n = *fail_count;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
        fixup_zone<NV>(d, g, ph, P, U, pflag, fail_list[t]);
}

// KBoundaries::check_inflow (boundaries.hpp:101-136) on a ghost zone's u^i (u[0..2]): where the
// flow enters the domain, the 3-velocity is reset to the normal observer's radial drift and the
// Lorentz factor rebuilt.  R: double, or Dual<double> for its Jacobian (gcov in R).
template <typename R>
__device__ __forceinline__ void inflow_fix(const ZoneGeom& G, const R gcov[4][4], R* u, bool inner)
{
    R uvec[3] = {u[0], u[1], u[2]};
    R gamma = lorentz(gcov, uvec[0], uvec[1], uvec[2]);
    const double alpha = 1. / sqrt(-G.gcon[0][0]);
    const R ucon1 = uvec[0] - gamma * R(alpha) * R(G.gcon[0][1]);
    if (((ucon1 > R(0.)) && inner) || ((ucon1 < R(0.)) && !inner)) {
#pragma unroll
        for (int v = 0; v < 3; ++v) uvec[v] = uvec[v] / gamma;
        const double beta1 = G.gcon[0][1] * alpha * alpha;
        uvec[0] = R(beta1 / alpha);
        const R vsq = gcov[1][1] * uvec[0] * uvec[0] + gcov[2][2] * uvec[1] * uvec[1] +
                      gcov[3][3] * uvec[2] * uvec[2] +
                      R(2.) * (gcov[1][2] * uvec[0] * uvec[1] + gcov[1][3] * uvec[0] * uvec[2] +
                               gcov[2][3] * uvec[1] * uvec[2]);
        gamma = R(1.) / dsqrt(R(1.) - vsq);
#pragma unroll
        for (int v = 0; v < 3; ++v) u[v] = uvec[v] * gamma;
    }
}

// ===================================================================================== boundaries
// Parthenon's outflow/reflecting functions (unvendored) as KHARMA applies them: fluid primitives
// and the conserved field; then the inflow check (boundaries.hpp:101-136).  NV = 10: the EMHD state,
// whose scalar primitives q~, dP~ (slots 8, 9) are copied as the density is.
// One zone (thread t of the face's ng x cnt_a x cnt_k enumeration) of k_bc
template <int NV>
__device__ __forceinline__ void bc_zone(const Dims& d, const DevGeom& g, const Phys& ph, const khb_fields& P,
                                        const khb_fields& U, int face, int lo_a, int cnt_a, int lo_k, int cnt_k,
                                        long long t)
{
    const int bdir = face / 2 + 1;
    const bool inner = (face % 2) == 0;
    const int ng = (bdir == 1) ? d.is : ((bdir == 2) ? d.js : d.ks);
    if (t >= (long long)ng*cnt_a*cnt_k) return;
    const int gidx = (int)(t % ng);
    const long long r = t / ng;
    const int aidx = lo_a + (int)(r % cnt_a);
    int i, j, k, ref;
    if (bdir == 1) {
        j = aidx;
        k = lo_k + (int)(r / cnt_a);
        ref = inner ? d.is : d.ie;
        i = inner ? gidx : d.ie + 1 + gidx;
    } else if (bdir == 2) {
        i = aidx;
        k = lo_k + (int)(r / cnt_a);
        ref = inner ? d.js : d.je;
        j = inner ? gidx : d.je + 1 + gidx;
    } else {
        // X3 faces: a runs over the whole (j, i) plane
        j = aidx / d.n1;
        i = aidx - j * d.n1;
        ref = inner ? d.ks : d.ke;
        k = inner ? gidx : d.ke + 1 + gidx;
    }
    const int type = d.bc[face];
    const int offset = 2 * ref + (inner ? -1 : 1);
    const bool transmit = type == KHB_BC_TRANSMITTING;
    int ii = i, jj = j, kk = k;
    if (bdir == 1)      ii = (type == KHB_BC_OUTFLOW) ? ref : offset - i;
    else if (bdir == 2) jj = (type == KHB_BC_OUTFLOW) ? ref : offset - j;
    else                kk = (type == KHB_BC_OUTFLOW) ? ref : offset - k;
    // transmitting: the mirrored zone half-way round in x3 (one_block_transmit.cpp:116-134)
    if (transmit) kk = ((k - d.ks + d.nx3 / 2) % d.nx3) + d.ks;
    const long long c = kchk(d, ((long long)k*d.n2 + j)*d.n1 + i, d.N, CHK_BC);
    const long long s = kchk(d, ((long long)kk*d.n2 + jj)*d.n1 + ii, d.N, CHK_BC);
    double Pz[5];
#pragma unroll
    for (int p = 0; p < 5; ++p) {
        const bool flip = ((type == KHB_BC_REFLECTING) && (p == 1 + bdir)) || (transmit && (p == 3 || p == 4));
        Pz[p] = (flip ? -1.0 : 1.0) * P.v[p][s];
    }
    if (NV == 10) {                          // slots that are not evolved may be NULL
        if (P.v[8]) P.v[8][c] = P.v[8][s];
        if (P.v[9]) P.v[9][c] = P.v[9][s];
    }
    if (NV > 5) {
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            const bool flip = ((type == KHB_BC_REFLECTING) && (v == bdir - 1)) || (transmit && v >= 1);
            U.v[5 + v][c] = (flip ? -1.0 : 1.0) * U.v[5 + v][s];
        }
    }
    const bool inflow = (face == 0 && ph.check_inflow_in) || (face == 1 && ph.check_inflow_out);
    if (inflow) {
        ZoneGeom G;
        load_zone_geom(g, j, i, G);
        inflow_fix<double>(G, G.gcov, Pz + 2, inner);
    }
#pragma unroll
    for (int p = 0; p < 5; ++p) P.v[p][c] = Pz[p];
}
template <int NV>
__global__ void k_bc(Dims d, DevGeom g, Phys ph, khb_fields P, khb_fields U, int face,
                     int lo_a, int cnt_a, int lo_k, int cnt_k)
{
    bc_zone<NV>(d, g, ph, P, U, face, lo_a, cnt_a, lo_k, cnt_k, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

// Ghost zones of one (j, i) plane, enumerated without the interior: the rows below js, the zones
// left and right of the interior in rows js..je, the rows above je.  Returns false past the end.
__device__ __forceinline__ bool plane_ghost(const Dims& d, unsigned t, int& j, int& i)
{
    const unsigned n1 = d.n1, side = n1 - (unsigned)(d.ie - d.is + 1);
    const unsigned below = (unsigned)d.js * n1, rows = (unsigned)(d.je - d.js + 1);
    const unsigned mid = rows * side, above = (unsigned)(d.n2 - 1 - d.je) * n1;
    if (t < below) { j = (int)(t / n1); i = (int)(t - (unsigned)j * n1); return true; }
    t -= below;
    if (t < mid) {
        const unsigned r = t / side, q = t - r * side;
        j = d.js + (int)r;
        i = (q < (unsigned)d.is) ? (int)q : (int)q + (d.ie - d.is + 1);
        return true;
    }
    t -= mid;
    if (t < above) { const unsigned r = t / n1; j = d.je + 1 + (int)r; i = (int)(t - r * n1); return true; }
    return false;
}
__host__ __device__ inline unsigned plane_ghost_count(const Dims& d)
{
    return (unsigned)(d.n1 * d.n2) - (unsigned)((d.ie - d.is + 1) * (d.je - d.js + 1));
}

// B_P = B_U/gdet and U = U(P) on the X1/X2 ghost zones of the interior k range.  B_CT blocks with
// physical faces (Bf.v[0] set): a zone outside the interior only along directions in ct_mask (bit
// 0: X1, bit 1: X2, bit 2: X3) takes B from its faces (B_CT::BlockUtoP over the boundary domain, b_ct.cpp:
// 160-188); the last ghost layer of a direction has its lower face only (the face array stops
// there) and takes B from that face alone.
// kplanes: the ghost planes of physical X3 faces instead (whole (j, i) planes below ks and above ke).
// pfaces (nonzero): a zone is taken only if it lies past a face whose bit is set (the boundary
// domains inner_x1 ... outer_x3 of those faces; the exchanged ghost zones keep their values)
template <int NV>
__device__ __forceinline__ void ghost_ptou_zone(const Dims& d, const DevGeom& g, const Phys& ph, const khb_fields& P,
                                                const khb_fields& U, const khb_fields& Bf, int ct_mask, int kplanes,
                                                int pfaces, unsigned t)
{
    int j, i, k;
    if (kplanes) {
        const unsigned plane = (unsigned)(d.n1 * d.n2);
        const unsigned kp = t / plane, r = t - kp * plane;
        const unsigned below = (kplanes & 1) ? (unsigned)d.ks : 0u;
        const unsigned above = (kplanes & 2) ? (unsigned)(d.n3 - 1 - d.ke) : 0u;
        if (kp >= below + above) return;
        k = (kp < below) ? (int)kp : d.ke + 1 + (int)(kp - below);
        j = (int)(r / (unsigned)d.n1);
        i = (int)(r - (unsigned)j * (unsigned)d.n1);
    } else {
        const unsigned per = plane_ghost_count(d);
        const unsigned kk = t / per;
        if (kk >= (unsigned)(d.ke - d.ks + 1)) return;
        if (!plane_ghost(d, t - kk * per, j, i)) return;
        k = d.ks + (int)kk;
    }
    if (pfaces && !(((pfaces & 1) && i < d.is) || ((pfaces & 2) && i > d.ie) || ((pfaces & 4) && j < d.js) ||
                    ((pfaces & 8) && j > d.je) || ((pfaces & 16) && k < d.ks) || ((pfaces & 32) && k > d.ke)))
        return;
    const long long c = ((long long)k*d.n2 + j)*d.n1 + i;
    ZoneGeom G;
    load_zone_geom(g, j, i, G);
    double Pz[NV], Uz[NV];
#pragma unroll
    for (int p = 0; p < 5; ++p) Pz[p] = P.v[p][c];
    const bool gi = i < d.is || i > d.ie, gj = j < d.js || j > d.je, gk = k < d.ks || k > d.ke;
    const bool from_faces = NV > 5 && Bf.v[0] && !(gi && !(ct_mask & 1)) && !(gj && !(ct_mask & 2)) &&
                            !(gk && !(ct_mask & 4));
    if (from_faces) {
        const long long gi0 = (long long)j*g.G1 + i;
        const double* F1 = Bf.v[0]; const double* F2 = Bf.v[1]; const double* F3 = Bf.v[2];
        Pz[5] = (i == d.n1 - 1) ? F1[c] / __ldg(g.gdet[0] + gi0)
                                : (F1[c] / __ldg(g.gdet[0] + gi0) + F1[c + 1] / __ldg(g.gdet[0] + gi0 + 1)) / 2;
        Pz[6] = (d.ndim > 1 && j < d.n2 - 1) ? (F2[c] / __ldg(g.gdet[1] + gi0) + F2[c + d.sj] / __ldg(g.gdet[1] + gi0 + g.G1)) / 2
                                             : F2[c] / __ldg(g.gdet[1] + gi0);
        Pz[7] = (d.ndim > 2 && k < d.n3 - 1) ? (F3[c] / __ldg(g.gdet[2] + gi0) + F3[c + d.sk] / __ldg(g.gdet[2] + gi0)) / 2
                                             : F3[c] / __ldg(g.gdet[2] + gi0);
#pragma unroll
        for (int v = 0; v < 3; ++v) P.v[5 + v][c] = Pz[5 + v];
    } else if (NV > 5) {
#pragma unroll
        for (int v = 0; v < 3; ++v) { Pz[5 + v] = U.v[5 + v][c] / G.gdet; P.v[5 + v][c] = Pz[5 + v]; }
    }
    p_to_u_zone<NV>(G, ph.gam, Pz, Uz);
#pragma unroll
    for (int p = 0; p < NV; ++p) U.v[p][c] = Uz[p];
}
template <int NV>
__global__ void k_ghost_ptou(Dims d, DevGeom g, Phys ph, khb_fields P, khb_fields U, khb_fields Bf, int ct_mask,
                             int kplanes, int pfaces)
{
    ghost_ptou_zone<NV>(d, g, ph, P, U, Bf, ct_mask, kplanes, pfaces, blockIdx.x * blockDim.x + threadIdx.x);
}

// Periodic images: every zone outside the interior in a periodic direction copies all variables
// of P and U from its image (wrapping only the periodic directions).
// Launched over the zones outside the interior only: the k ghost planes whole, then the X1/X2
// ghost zones of each interior plane.
template <int NV>
__device__ __forceinline__ void periodic_zone(const Dims& d, const khb_fields& P, const khb_fields& U, int pmask,
                                              unsigned u)
{
    const unsigned plane = (unsigned)(d.n1 * d.n2);
    const unsigned kg = (unsigned)(d.n3 - (d.ke - d.ks + 1));     // k ghost planes
    int k, j, i;
    if (u < kg * plane) {
        const unsigned kp = u / plane, r = u - kp * plane;
        k = (kp < (unsigned)d.ks) ? (int)kp : d.ke + 1 + (int)(kp - (unsigned)d.ks);
        j = (int)(r / (unsigned)d.n1);
        i = (int)(r - (unsigned)j * (unsigned)d.n1);
    } else {
        u -= kg * plane;
        const unsigned per = plane_ghost_count(d);
        if (per == 0) return;
        const unsigned kk = u / per;
        if (kk >= (unsigned)(d.ke - d.ks + 1)) return;
        if (!plane_ghost(d, u - kk * per, j, i)) return;
        k = d.ks + (int)kk;
    }
    const long long t = ((long long)k*d.n2 + j)*d.n1 + i;
    int ii = i, jj = j, kk = k;
    bool any = false;
    if ((pmask & 1) && (i < d.is || i > d.ie)) { ii += (i < d.is) ? d.nx1 : -d.nx1; any = true; }
    if ((pmask & 2) && (j < d.js || j > d.je)) { jj += (j < d.js) ? d.nx2 : -d.nx2; any = true; }
    if ((pmask & 4) && (k < d.ks || k > d.ke)) { kk += (k < d.ks) ? d.nx3 : -d.nx3; any = true; }
    if (!any) return;
    const long long s = kchk(d, ((long long)kk*d.n2 + jj)*d.n1 + ii, d.N, CHK_PERIODIC);
#pragma unroll
    for (int p = 0; p < NV; ++p) {
        if (NV > 8 && !P.v[p]) continue;       // EMHD slots that are not evolved
        P.v[p][t] = P.v[p][s]; U.v[p][t] = U.v[p][s];
    }
}
template <int NV>
__global__ void k_periodic(Dims d, khb_fields P, khb_fields U, int pmask)
{
    periodic_zone<NV>(d, P, U, pmask, blockIdx.x * blockDim.x + threadIdx.x);
}

// The boundary work of many blocks, one launch per phase of launch_boundaries: blockIdx.y picks the
// task (one block's face, ghost P->U pass or periodic images), blockIdx.x * blockDim.x + threadIdx.x
// the zone of its enumeration; the tasks of one phase are different blocks' or disjoint regions
template <int NV>
__global__ void __launch_bounds__(128) k_bound_tasks(const BoundTask* __restrict__ tasks)
{
    const BoundTask& T = tasks[blockIdx.y];
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T.count) return;
    if (T.kind == BOUND_BC) bc_zone<NV>(T.d, T.g, T.ph, T.P, T.U, T.face, T.lo_a, T.cnt_a, T.lo_k, T.cnt_k, t);
    else if (T.kind == BOUND_GHOST_PTOU) ghost_ptou_zone<NV>(T.d, T.g, T.ph, T.P, T.U, T.Bf, 0, T.kplanes, T.pfaces, (unsigned)t);
    else periodic_zone<NV>(T.d, T.P, T.U, T.pmask, (unsigned)t);
}

// The ghost shell (every zone outside the interior) of a stage's input copied to its output: the
// stage's copy of P_s into P_{s+1} as the inversion guess (kharma_driver.cpp:380-384) and U = U(P)
// there, as they stand before the caller's boundary exchange replaces them.  Needed only for blocks
// with exchange faces; physical and periodic faces are filled afterwards by the boundary kernels.
__device__ __forceinline__ bool shell_zone(const Dims& d, unsigned u, long long& c)
{
    const unsigned plane = (unsigned)(d.n1 * d.n2);
    const unsigned kg = (unsigned)(d.n3 - (d.ke - d.ks + 1));
    int k, j, i;
    if (u < kg * plane) {
        const unsigned kp = u / plane, r = u - kp * plane;
        k = (kp < (unsigned)d.ks) ? (int)kp : d.ke + 1 + (int)(kp - (unsigned)d.ks);
        j = (int)(r / (unsigned)d.n1);
        i = (int)(r - (unsigned)j * (unsigned)d.n1);
    } else {
        u -= kg * plane;
        const unsigned per = plane_ghost_count(d);
        if (per == 0) return false;
        const unsigned kk = u / per;
        if (kk >= (unsigned)(d.ke - d.ks + 1)) return false;
        if (!plane_ghost(d, u - kk * per, j, i)) return false;
        k = d.ks + (int)kk;
    }
    c = ((long long)k*d.n2 + j)*d.n1 + i;
    return true;
}
template <int NV>
__device__ __forceinline__ void copy_zone(const khb_fields& Pin, const khb_fields& Uin, const khb_fields& Pout,
                                          const khb_fields& Uout, long long c)
{
#pragma unroll
    for (int p = 0; p < NV; ++p) { Pout.v[p][c] = Pin.v[p][c]; Uout.v[p][c] = Uin.v[p][c]; }
}
template <int NV>
__global__ void k_ghost_copy(Dims d, khb_fields Pin, khb_fields Uin, khb_fields Pout, khb_fields Uout)
{
    long long c;
    if (shell_zone(d, blockIdx.x * blockDim.x + threadIdx.x, c)) copy_zone<NV>(Pin, Uin, Pout, Uout, c);
}
// One row of CTAs per block (blockIdx.y), grid-striding over that block's shell
template <int NV>
__global__ void k_batch_ghost_copy(const FixupBlock* __restrict__ blocks, int stage)
{
    const FixupBlock& B = blocks[blockIdx.y];
    if (!B.exch) return;
    const int s = stage - 1;
    const unsigned n = (unsigned)(B.d.N - (long long)(B.d.ie - B.d.is + 1)*(B.d.je - B.d.js + 1)*(B.d.ke - B.d.ks + 1));
    for (unsigned u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
        long long c;
        if (shell_zone(B.d, u, c)) copy_zone<NV>(B.Pin[s], B.Uin[s], B.P[s], B.U[s], c);
    }
}

// Whole-block P->U (Flux::MeshPtoU)
template <int NV>
__global__ void k_ptou(Dims d, DevGeom g, Phys ph, khb_fields P, khb_fields U)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= d.N) return;
    int k, j, i;
    zone_kji(d, t, k, j, i);
    ZoneGeom G;
    load_zone_geom(g, j, i, G);
    double Pz[NV], Uz[NV];
#pragma unroll
    for (int p = 0; p < NV; ++p) Pz[p] = P.v[p][t];
    p_to_u_zone<NV>(G, ph.gam, Pz, Uz);
#pragma unroll
    for (int p = 0; p < NV; ++p) U.v[p][t] = Uz[p];
}

// Materialize flux-CT into the B flux scratch (b_flux_ct.cpp:307-370), for khb_flux_ct.
// Reads raw fluxes from Fr (a copy) and writes the rewritten B fluxes into F.
template <typename FT>
__global__ void k_emf(Dims d, const FT* F1, const FT* F2, const FT* F3, FT* E)
{
    // corner EMFs on [ks, ke+1(3D)] x [js, je+1] x [is, ie+1]
    const int ci = d.ie - d.is + 2, cj = d.je - d.js + 2, ck = (d.ndim > 2) ? d.ke - d.ks + 2 : 1;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)ci*cj*ck) return;
    const int i = d.is + (int)(t % ci);
    const int j = d.js + (int)((t / ci) % cj);
    const int k = d.ks + (int)(t / ((long long)ci*cj));
    const long long c = ((long long)k*d.n2 + j)*d.n1 + i, N = d.N, sj = d.sj, sk = d.sk;
    if (d.ndim > 2) {
        E[c]     = (FT)0.25 * (F2[7*N + c] + F2[7*N + c - sk] - F3[6*N + c] - F3[6*N + c - sj]);
        E[N + c] = (FT)0.25 * (F3[5*N + c] + F3[5*N + c - 1] - F1[7*N + c] - F1[7*N + c - sk]);
    }
    E[2*N + c] = (FT)0.25 * (F1[6*N + c] + F1[6*N + c - sj] - F2[5*N + c] - F2[5*N + c - 1]);
}
template <typename FT>
__global__ void k_ct_apply(Dims d, FT* F1, FT* F2, FT* F3, const FT* E)
{
    // each thread owns one (k,j,i) in [ks, ke+1] x [js, je+1] x [is, ie+1] and writes the faces there
    const int ci = d.ie - d.is + 2, cj = d.je - d.js + 2, ck = (d.ndim > 2) ? d.ke - d.ks + 2 : 1;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)ci*cj*ck) return;
    const int i = d.is + (int)(t % ci);
    const int j = d.js + (int)((t / ci) % cj);
    const int k = d.ks + (int)(t / ((long long)ci*cj));
    const long long c = ((long long)k*d.n2 + j)*d.n1 + i, N = d.N, sj = d.sj, sk = d.sk;
    const FT* e1 = E; const FT* e2 = E + N; const FT* e3 = E + 2*N;
    const bool d3 = d.ndim > 2;
    const bool kin = k <= d.ke, jin = j <= d.je, iin = i <= d.ie;
    if (kin && jin) {
        F1[5*N + c] = (FT)0.0;
        F1[6*N + c] = (FT)0.5 * (e3[c] + e3[c + sj]);
        if (d3) F1[7*N + c] = (FT)-0.5 * (e2[c] + e2[c + sk]);
    }
    if (kin && iin) {
        F2[5*N + c] = (FT)-0.5 * (e3[c] + e3[c + 1]);
        F2[6*N + c] = (FT)0.0;
        if (d3) F2[7*N + c] = (FT)0.5 * (e1[c] + e1[c + sk]);
    }
    if (d3 && jin && iin) {
        F3[5*N + c] = (FT)0.5 * (e2[c] + e2[c + 1]);
        F3[6*N + c] = (FT)-0.5 * (e1[c] + e1[c + sj]);
        F3[7*N + c] = (FT)0.0;
    }
}

// Copy scratch fluxes out as doubles
template <typename FT>
__global__ void k_copy_flux(long long N, int nv, const FT* F, const FT* ctop, khb_fields out, double* ctop_out)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N) return;
    for (int p = 0; p < nv; ++p) if (out.v[p]) out.v[p][t] = (double)F[p*N + t];
    if (ctop_out) ctop_out[t] = (double)ctop[t];
}

// |corner divB| at corner (k,j,i) of the conserved field (b_flux_ct_functions.hpp:52-75)
__device__ __forceinline__ double corner_divb(const Dims& d, const Phys& ph, const khb_fields& U,
                                              int k, int j, int i)
{
    const long long c = ((long long)k*d.n2 + j)*d.n1 + i, sj = d.sj, sk = d.sk;
    const double* B1 = U.v[5]; const double* B2 = U.v[6]; const double* B3 = U.v[7];
    const bool do3 = d.ndim > 2;
    const double norm = do3 ? 0.25 : 0.5;
    double term1 = B1[c] - B1[c-1] + B1[c-sj] - B1[c-sj-1];
    double term2 = B2[c] - B2[c-sj] + B2[c-1] - B2[c-sj-1];
    double term3 = 0.;
    if (do3) {
        term1 += B1[c-sk] + B1[c-sk-sj] - B1[c-sk-1] - B1[c-sk-sj-1];
        term2 += B2[c-sk] + B2[c-sk-1] - B2[c-sk-sj] - B2[c-sk-sj-1];
        term3 = B3[c] + B3[c-sj] + B3[c-1] + B3[c-sj-1] - B3[c-sk] - B3[c-sk-sj] - B3[c-sk-1] - B3[c-sk-sj-1];
    }
    return fabs(norm*term1/ph.dx1 + norm*term2/ph.dx2 + norm*term3/ph.dx3);
}

// Maximum over the 256 threads of a block (blockDim.x == 256)
__device__ __forceinline__ double block_max256(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    __shared__ double wmax[8];
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = v;
    __syncthreads();
    double m = wmax[0];
    for (int w = 1; w < 8; ++w) m = fmax(m, wmax[w]);
    return m;
}

// One corner per thread over [ks, ke+1(3D)] x [js, je+1] x [i_lo, i_hi]
__device__ __forceinline__ double divb_of_thread(const Dims& d, const Phys& ph, const khb_fields& U,
                                                 int i_lo, int i_hi)
{
    const int ci = i_hi - i_lo + 1, cj = d.je - d.js + 2, ck = (d.ndim > 2) ? d.ke - d.ks + 2 : 1;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)ci*cj*ck) return 0.;
    const int i = i_lo + (int)(t % ci);
    const int j = d.js + (int)((t / ci) % cj);
    const int k = d.ks + (int)(t / ((long long)ci*cj));
    return corner_divb(d, ph, U, k, j, i);
}

#ifdef KHB_COMMON_KERNELS
// B_FluxCT::MaxDivB (b_flux_ct.cpp:566-607): block max, then one atomicMax on the bit pattern
__global__ void __launch_bounds__(256) k_divb(Dims d, Phys ph, khb_fields U, int i_lo, int i_hi, unsigned long long* word)
{
    const double m = block_max256(divb_of_thread(d, ph, U, i_lo, i_hi));
    if (threadIdx.x == 0) atomicMax(word, (unsigned long long)__double_as_longlong(m));
}
#endif

// ===================================================================================== batches
// Every meshblock of a batch in one launch per kernel: a CTA takes tiles (128-thread boxes of one
// block) from the tile table, stages that block's descriptor in shared memory and runs the same
// per-face / per-zone code as the single-block kernels on it.  With a persistent grid each CTA
// walks the table with a stride of gridDim.x.
template <typename T>
__device__ __forceinline__ void stage_desc(T& dst, const T* __restrict__ src)
{
    static_assert(sizeof(T) % 8 == 0, "descriptor size must be a multiple of 8 bytes");
    const unsigned long long* s = reinterpret_cast<const unsigned long long*>(src);
    unsigned long long* o = reinterpret_cast<unsigned long long*>(&dst);
    for (unsigned x = threadIdx.x; x < sizeof(T) / 8; x += blockDim.x) o[x] = __ldg(s + x);
}

template <int DIR, int RECON, int NV, typename R, typename FT>
__global__ void __launch_bounds__(128, FluxMinBlocks<R, DIR>::value)
k_batch_flux(const BatchBlock<FT>* __restrict__ blocks, const int* __restrict__ tiles, unsigned ntiles, int stage)
{
    __shared__ __align__(16) BatchBlock<FT> sb;
    int cur = -1;
    for (unsigned t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int b = __ldg(tiles + t);
        if (b != cur) {
            __syncthreads();
            stage_desc(sb, blocks + b);
            __syncthreads();
            cur = b;
        }
        int i, j, k;
        if (box_cell(sb.fbox[DIR - 1], t - sb.tile0[DIR - 1], i, j, k))
            flux_face<DIR, RECON, NV, R, FT>(sb.d, sb.g, sb.ph, sb.Pin[stage - 1], sb.F[DIR - 1], sb.ctop[DIR - 1],
                                            i, j, k);
    }
}

template <int NV, typename FT, int MODE>
__global__ void __launch_bounds__(128, ZoneMinBlocks<MODE, FT>::value)
k_batch_zone(const BatchBlock<FT>* __restrict__ blocks, const int* __restrict__ tiles, unsigned ntiles, int stage,
             int dtm, double beta, const double* __restrict__ dt)
{
    __shared__ __align__(16) BatchBlock<FT> sb;
    const int s = stage - 1;
    int cur = -1;
    for (unsigned t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int b = __ldg(tiles + t);
        if (b != cur) {
            __syncthreads();
            stage_desc(sb, blocks + b);
            __syncthreads();                          // the whole descriptor is in place before the patch
            if (threadIdx.x == 0) {
                sb.za[s].bdt = beta * __ldg(dt);      // as the single-block path forms beta * dt
                sb.za[s].mode = dtm;
                // the cell half inverts the state the update half wrote (the fused pass keeps it in registers)
                if ((MODE & M_UTOP) && !(MODE & M_UPDATE)) sb.za[s].Us = sb.za[s].Uout;
            }
            __syncthreads();
            cur = b;
        }
        int i, j, k;
        double ndt_zone = 1.7976931348623157e308;
        if (box_cell(sb.zbox, t - sb.tile0[3], i, j, k)) ndt_zone = zone_body<NV, FT, MODE>(sb.d, sb.g, sb.ph, sb.za[s], i, j, k);
        if (dtm & M_DT) {
            block_min_ndt(ndt_zone, sb.za[s].ndt_word);
            __syncthreads();          // wmin is reused by the next tile of this CTA
        }
    }
}

// The cell half of the zone pass (inversion from the seed, floors, U = U(P)) on the ghost zones of a
// mesh's exchange entries, after the kharma driver's exchange: MeshUtoP and MeshApplyFloors over the
// entire block (kharma_step.cpp:233-236).  Stage s's arguments of the destination block, its updated
// U as the state to invert; standalone (an exchange outside a stage): the seeds are the block's
// state primitives, which the zone also writes.  No timestep and no failed-zone list: FixUtoP works
// on the interior.
template <int NV, typename FT, int MODE>
__global__ void __launch_bounds__(128) k_mesh_ghost_cell(const BatchBlock<FT>* __restrict__ blocks,
                                                         const int* __restrict__ table, long long n, int s,
                                                         int standalone)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int* t = table + 6 * e;
    const BatchBlock<FT>& B = blocks[__ldg(t)];
    ZoneArgs<FT> a = B.za[s];
    a.Us = a.Uout;
    if (standalone) a.Ps = B.za[0].Ps;
    a.mode = 0;
    int k, j, i;
    zone_kji(B.d, __ldg(t + 1), k, j, i);
    zone_body<NV, FT, MODE>(B.d, B.g, B.ph, a, i, j, k);
}

// The fused plan's first launch of a stage (Launch<FT>::batch_flux_all): the faces of all directions
// of every block and the ghost-shell copies of blocks with exchange faces, one table of 128-wide
// tiles; CTA 0 first resets the failed-zone counters and the timestep minimum the zone pass fills.
// The launch bound is the x3 faces' (the largest register need of the three directions).
#ifndef KHB_BATCH_FLUXALL_MINB
#define KHB_BATCH_FLUXALL_MINB KHB_FLUX64_X3_MINB
#endif
template <typename R> struct FluxAllMinBlocks { static constexpr int value = KHB_FLUX32_MINB; };
template <> struct FluxAllMinBlocks<double> { static constexpr int value = KHB_BATCH_FLUXALL_MINB; };
template <int RECON, int NV, typename R, typename FT>
__global__ void __launch_bounds__(128, FluxAllMinBlocks<R>::value)
k_batch_flux_all(const BatchBlock<FT>* __restrict__ blocks, const int* __restrict__ tiles, unsigned ntiles, int stage,
                 int* const* __restrict__ counts, int nblocks, unsigned long long* word)
{
    __shared__ __align__(16) BatchBlock<FT> sb;
    if (blockIdx.x == 0) {
        for (int x = threadIdx.x; x < nblocks; x += blockDim.x) *counts[x] = 0;
        if (threadIdx.x == 0 && word) *word = 0x7FEFFFFFFFFFFFFFull;     // bit pattern of DBL_MAX
    }
    const int s = stage - 1;
    int cur = -1;
    for (unsigned t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int e = __ldg(tiles + t);
        const int b = e & 0x0fffffff, kind = (e >> 28) & 3;
        if (b != cur) {
            __syncthreads();
            stage_desc(sb, blocks + b);
            __syncthreads();
            cur = b;
        }
        const unsigned lt = t - sb.tile0c[kind];
        int i, j, k;
        if (kind == 3) {
            long long c;
            if (shell_zone(sb.d, lt * 128u + threadIdx.x, c))
                copy_zone<NV>(sb.za[s].Ps, sb.za[s].Us, sb.za[s].Pout, sb.za[s].Uout, c);
        } else if (kind == 0) {
            if (box_cell(sb.fbox[0], lt, i, j, k))
                flux_face<1, RECON, NV, R, FT>(sb.d, sb.g, sb.ph, sb.Pin[s], sb.F[0], sb.ctop[0], i, j, k);
        } else if (kind == 1) {
            if (box_cell(sb.fbox[1], lt, i, j, k))
                flux_face<2, RECON, NV, R, FT>(sb.d, sb.g, sb.ph, sb.Pin[s], sb.F[1], sb.ctop[1], i, j, k);
        } else {
            if (box_cell(sb.fbox[2], lt, i, j, k))
                flux_face<3, RECON, NV, R, FT>(sb.d, sb.g, sb.ph, sb.Pin[s], sb.F[2], sb.ctop[2], i, j, k);
        }
    }
}

// ===================================================================================== SMR
// Flux correction (Parthenon's flux-correction messages, kharma_step.cpp:183-195): each entry
// replaces a coarse face's fluxes by the average of the 2^(ndim-1) fine fluxes through it.  Entry:
// {coarse block, direction, coarse face, fine block, fine face of lowest index, -}.
template <typename FT>
__global__ void __launch_bounds__(128) k_mesh_flux(const BatchBlock<FT>* __restrict__ blocks,
                                                   const int* __restrict__ table, long long n, int nv)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int* t = table + 6 * e;
    const BatchBlock<FT>& C = blocks[__ldg(t)];
    const BatchBlock<FT>& F = blocks[__ldg(t + 3)];
    const int dir = __ldg(t + 1);
    const long long cc = __ldg(t + 2), fc = __ldg(t + 4);
    FT* Fc = C.F[dir - 1];
    const FT* Ff = F.F[dir - 1];
    const Dims& df = F.d;
    // tangential strides in the fine block
    const long long t1 = (dir == 1) ? df.sj : 1;
    const long long t2 = (dir == 3) ? df.sj : df.sk;
    const bool two = df.ndim > 2;
    for (int p = 0; p < nv; ++p) {
        const FT* f = Ff + p * df.N + fc;
        FT v;
        if (two) v = ((f[0] + f[t1]) + (f[t2] + f[t1 + t2])) * (FT)0.25;
        else v = (f[0] + f[t1]) * (FT)0.5;
        Fc[p * C.d.N + cc] = v;
    }
}

#ifdef KHB_COMMON_KERNELS
// SMR ghost zones (Parthenon's cell-centred refinement operators on a uniform grid): entries
// {dst block, dst zone, op, src block, src zone, aux} fill the stage output's primitives of a ghost
// zone by a copy, the average of the 2^ndim fine zones (restriction), or the coarse value plus a
// minmod-limited slope times +-1/4 per active direction (prolongation; aux bit d: + side along
// d+1), then set its conserved variables U = U(P).  Prolongations run in a second launch: they read
// coarse ghost zones that copies and restrictions fill.
__device__ __forceinline__ double minmod2(double a, double b)
{
    return (a * b > 0.) ? ((fabs(a) < fabs(b)) ? a : b) : 0.;
}
// One variable of a ghost entry: op 0 copy, 1 restriction, 2 prolongation (q: the source array)
__device__ __forceinline__ double mesh_op(const double* q, long long cs, int op, int aux, const Dims& ds)
{
    if (op == 0) return q[cs];
    if (op == 1) {
        double r = (q[cs] + q[cs + 1]);
        if (ds.ndim > 1) r = r + (q[cs + ds.sj] + q[cs + ds.sj + 1]);
        if (ds.ndim > 2) r = r + ((q[cs + ds.sk] + q[cs + ds.sk + 1]) + (q[cs + ds.sk + ds.sj] + q[cs + ds.sk + ds.sj + 1]));
        return r * ((ds.ndim > 2) ? 0.125 : (ds.ndim > 1) ? 0.25 : 0.5);
    }
    const double uc = q[cs];
    double v = uc;
    const long long st[3] = {1, ds.sj, ds.sk};
    for (int d = 0; d < ds.ndim; ++d) {
        const double sl = minmod2(uc - q[cs - st[d]], q[cs + st[d]] - uc);
        v += ((aux >> d) & 1) ? 0.25 * sl : -0.25 * sl;
    }
    return v;
}
template <int NV>
__global__ void __launch_bounds__(128) k_mesh_ghost(const FixupBlock* __restrict__ blocks, const int* __restrict__ table,
                                                    long long begin, long long end, int stage)
{
    const long long e = begin + (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= end) return;
    const int s = stage - 1;
    const int* t = table + 6 * e;
    const FixupBlock& D = blocks[__ldg(t)];
    const FixupBlock& S = blocks[__ldg(t + 3)];
    const long long cd = __ldg(t + 1), cs = __ldg(t + 4);
    const int op = __ldg(t + 2), aux = __ldg(t + 5);
    const khb_fields& Ps = S.P[s];
    double P[NV];
#pragma unroll
    for (int p = 0; p < NV; ++p) P[p] = mesh_op(Ps.v[p], cs, op, aux, S.d);
    const khb_fields& Pd = D.P[s];
    const khb_fields& Ud = D.U[s];
#pragma unroll
    for (int p = 0; p < NV; ++p) Pd.v[p][cd] = P[p];
    int k, j, i;
    zone_kji(D.d, cd, k, j, i);
    ZoneGeom G;
    load_zone_geom(D.g, j, i, G);
    double U[NV];
    p_to_u_zone<NV>(G, D.ph.gam, P, U);
#pragma unroll
    for (int p = 0; p < NV; ++p) Ud.v[p][cd] = U[p];
}

// The kharma driver's exchange (sync_prims false, kharma_driver.cpp:109-118): the conserved variables
// by the entry's operator, and the fluid primitives too as the seed of the ghost zone's inversion
// (GRMHD sync_utop_seed, grmhd.cpp:159-165).  Runs between the update and the inversion: the
// updated U of stage s sits in U[u_sel], the seeds (the stage's input primitives) in Pin[seed_sel];
// the ghost zone's values go to the same arrays, where later phases and the inversion read them.
template <int NV>
__global__ void __launch_bounds__(128) k_mesh_ghost_cons(const FixupBlock* __restrict__ blocks,
                                                         const int* __restrict__ table, long long begin,
                                                         long long end, int seed_sel, int u_sel)
{
    const long long e = begin + (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= end) return;
    const int* t = table + 6 * e;
    const FixupBlock& D = blocks[__ldg(t)];
    const FixupBlock& S = blocks[__ldg(t + 3)];
    const long long cd = __ldg(t + 1), cs = __ldg(t + 4);
    const int op = __ldg(t + 2), aux = __ldg(t + 5);
    double P[NV], U[NV];
#pragma unroll
    for (int p = 0; p < NV; ++p) {
        P[p] = mesh_op(S.Pin[seed_sel].v[p], cs, op, aux, S.d);
        U[p] = mesh_op(S.U[u_sel].v[p], cs, op, aux, S.d);
    }
#pragma unroll
    for (int p = 0; p < NV; ++p) {
        D.Pin[seed_sel].v[p][cd] = P[p];
        D.U[u_sel].v[p][cd] = U[p];
    }
}
#endif

#ifdef KHB_COMMON_KERNELS
// One row of CTAs per block (blockIdx.y), each walking that block's failed-zone list
template <int NV>
__global__ void k_batch_fixup(const FixupBlock* __restrict__ blocks, int stage)
{
    const FixupBlock& B = blocks[blockIdx.y];
    if (!B.ph.fix_avg && !B.ph.fix_atmo) return;
    const int s = stage - 1;
    const int n = *B.fail_count;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
        fixup_zone<NV>(B.d, B.g, B.ph, B.P[s], B.U[s], B.pflag, B.fail_list[t]);
}
__global__ void k_stage_reset(int* count, unsigned long long* word)
{
    *count = 0;
    if (word) *word = 0x7FEFFFFFFFFFFFFFull;     // bit pattern of DBL_MAX
}
// GRMHD::EstimateTimestep: clip(cfl * min_ndt, dt_min, max_dt_increase * dt_last); then
// KHARMADriver::SetGlobalTimeStep: min(2 dt_last, that) (grmhd.cpp:320-339, kharma_driver.cpp:439-460)
__global__ void k_next_dt(const unsigned long long* ndt_word, double* state, double cfl, double dt_min,
                          double max_dt_increase)
{
    const double mn = __longlong_as_double((long long)*ndt_word);
    const double dt = state[0];
    const double ndt = kmin(kmax(mn * cfl, dt_min), max_dt_increase * dt);
    state[1] += dt;
    state[2] = dt;
    state[0] = kmin(2.0 * dt, ndt);
}
__global__ void k_batch_reset(int* const* counts, int nblocks, unsigned long long* word)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nblocks) *counts[t] = 0;
    if (t == 0 && word) *word = 0x7FEFFFFFFFFFFFFFull;     // bit pattern of DBL_MAX
}
#endif

// ===================================================================================== launchers
template <int DIR, int NV, typename FT>
static void flux_dir_recon(int recon, const Dims& d, const DevGeom& g, const Phys& ph, const khb_fields& P,
                           FT* F, FT* ctop, const int lo[3], const int cnt[3], cudaStream_t st)
{
    const Box bx = make_box(lo[0], lo[1], lo[2], cnt[0], cnt[1], cnt[2]);
    const unsigned nb = box_blocks(bx);
    switch (recon) {
    case RECON_DONOR: k_flux<DIR, RECON_DONOR, NV, FT, FT><<<nb, 128, 0, st>>>(d, g, ph, P, F, ctop, bx); break;
    case RECON_MC:    k_flux<DIR, RECON_MC, NV, FT, FT><<<nb, 128, 0, st>>>(d, g, ph, P, F, ctop, bx); break;
    case RECON_WENO5: k_flux<DIR, RECON_WENO5, NV, FT, FT><<<nb, 128, 0, st>>>(d, g, ph, P, F, ctop, bx); break;
    case RECON_PPM:   k_flux<DIR, RECON_PPM, NV, FT, FT><<<nb, 128, 0, st>>>(d, g, ph, P, F, ctop, bx); break;
    case RECON_WENO5X: k_flux<DIR, RECON_WENO5X, NV, FT, FT><<<nb, 128, 0, st>>>(d, g, ph, P, F, ctop, bx); break;
    default:          k_flux<DIR, RECON_EXTRA, NV, FT, FT><<<nb, 128, 0, st>>>(d, g, ph, P, F, ctop, bx); break;
    }
}

template <int NV, typename FT>
static void flux_nv(int recon, int dir, const Dims& d, const DevGeom& g, const Phys& ph, const khb_fields& P,
                    FT* F, FT* ctop, const int lo[3], const int cnt[3], cudaStream_t st)
{
    if (dir == 1) flux_dir_recon<1, NV, FT>(recon, d, g, ph, P, F, ctop, lo, cnt, st);
    else if (dir == 2) flux_dir_recon<2, NV, FT>(recon, d, g, ph, P, F, ctop, lo, cnt, st);
    else flux_dir_recon<3, NV, FT>(recon, d, g, ph, P, F, ctop, lo, cnt, st);
}

template <typename FT>
void Launch<FT>::flux(int recon, int nv, int dir, const Dims& d, const DevGeom& g, const Phys& ph,
                      const khb_fields& P, FT* F, FT* ctop, const int lo[3], const int cnt[3], cudaStream_t st)
{
    // the kernel variant: KHB_RECON_* 0-3 as they are, 4-7 through RECON_EXTRA, WENO5 with lowering
    // or the floor fallback through RECON_WENO5X
    const int kr = (recon > RECON_PPM) ? RECON_EXTRA
                 : ((recon == RECON_WENO5 && (ph.weno_lower || ph.recon_fallback)) ? RECON_WENO5X : recon);
    if (nv == 8) flux_nv<8, FT>(kr, dir, d, g, ph, P, F, ctop, lo, cnt, st);
    else flux_nv<5, FT>(kr, dir, d, g, ph, P, F, ctop, lo, cnt, st);
}

template <typename FT>
void Launch<FT>::fix_flux_x2(int nv, const Dims& d, const Phys& ph, FT* F1, FT* F2, FT* F3, int inner, cudaStream_t st)
{
    const int ni = d.ie - d.is + 3, nk = (d.ndim > 2) ? d.ke - d.ks + 3 : 1;
    const unsigned nb = blocks_for((long long)ni*nk, 128);
    if (nv == 10) k_fix_flux_x2<10, FT><<<nb, 128, 0, st>>>(d, ph, F1, F2, F3, inner);
    else if (nv == 8) k_fix_flux_x2<8, FT><<<nb, 128, 0, st>>>(d, ph, F1, F2, F3, inner);
    else k_fix_flux_x2<5, FT><<<nb, 128, 0, st>>>(d, ph, F1, F2, F3, inner);
}

template <typename FT>
void Launch<FT>::fix_tasks(int nv, const FixTask<FT>* tasks, int ntasks, int max_count, cudaStream_t st)
{
    if (ntasks <= 0 || max_count <= 0) return;
    const dim3 grid(blocks_for(max_count, 128), (unsigned)ntasks);
    if (nv == 8) k_fix_tasks<8, FT><<<grid, 128, 0, st>>>(tasks);
    else k_fix_tasks<5, FT><<<grid, 128, 0, st>>>(tasks);
}

template <typename FT>
void Launch<FT>::fix_flux_x1(const Dims& d, FT* F1, int inner, cudaStream_t st)
{
    const int nj = (d.ndim > 1) ? d.je - d.js + 3 : 1, nk = (d.ndim > 2) ? d.ke - d.ks + 3 : 1;
    k_fix_flux_x1<FT><<<blocks_for((long long)nj*nk, 128), 128, 0, st>>>(d, F1, inner);
}

template <int NV, typename FT>
static void zone_nv(const Dims& d, const DevGeom& g, const Phys& ph, const ZoneArgs<FT>& a, cudaStream_t st)
{
    const Box bx = make_box(d.is, d.js, d.ks, d.ie - d.is + 1, d.je - d.js + 1, d.ke - d.ks + 1);
    const unsigned nb = box_blocks(bx);
    const int m = a.mode & ~M_DT;
    switch (m) {
    case M_ZONE_FUSED: k_zone<NV, FT, M_ZONE_FUSED><<<nb, 128, 0, st>>>(d, g, ph, a, bx); break;
    case M_ZONE_FUSED | M_KASTAUN: k_zone<NV, FT, M_ZONE_FUSED | M_KASTAUN><<<nb, 128, 0, st>>>(d, g, ph, a, bx); break;
    case M_UPDATE: k_zone<NV, FT, M_UPDATE><<<nb, 128, 0, st>>>(d, g, ph, a, bx); break;
    case M_ZONE_CELL: k_zone<NV, FT, M_ZONE_CELL><<<nb, 128, 0, st>>>(d, g, ph, a, bx); break;
    case M_ZONE_CELL | M_KASTAUN: k_zone<NV, FT, M_ZONE_CELL | M_KASTAUN><<<nb, 128, 0, st>>>(d, g, ph, a, bx); break;
    case M_UTOP: k_zone<NV, FT, M_UTOP><<<nb, 128, 0, st>>>(d, g, ph, a, bx); break;
    case M_UTOP | M_KASTAUN: k_zone<NV, FT, M_UTOP | M_KASTAUN><<<nb, 128, 0, st>>>(d, g, ph, a, bx); break;
    case M_ZONE_FLOORS: k_zone<NV, FT, M_ZONE_FLOORS><<<nb, 128, 0, st>>>(d, g, ph, a, bx); break;
    default: k_zone<NV, FT, 0><<<nb, 128, 0, st>>>(d, g, ph, a, bx); break;
    }
}

template <typename FT>
void Launch<FT>::zone(int nv, const Dims& d, const DevGeom& g, const Phys& ph, const ZoneArgs<FT>& a, cudaStream_t st)
{
    if (nv == 8) zone_nv<8, FT>(d, g, ph, a, st);
    else zone_nv<5, FT>(d, g, ph, a, st);
}

template <typename FT>
void Launch<FT>::flux_ct(const Dims& d, FT* F1, FT* F2, FT* F3, FT* emf, cudaStream_t st)
{
    const long long tot = (long long)(d.ie - d.is + 2)*(d.je - d.js + 2)*((d.ndim > 2) ? d.ke - d.ks + 2 : 1);
    k_emf<FT><<<blocks_for(tot, 128), 128, 0, st>>>(d, F1, F2, F3, emf);
    k_ct_apply<FT><<<blocks_for(tot, 128), 128, 0, st>>>(d, F1, F2, F3, emf);
}

template <typename FT>
void Launch<FT>::copy_flux(long long N, int nv, const FT* F, const FT* ctop, const khb_fields& out, double* ctop_out,
                           cudaStream_t st)
{
    k_copy_flux<FT><<<blocks_for(N, 256), 256, 0, st>>>(N, nv, F, ctop, out, ctop_out);
}

template <int NV, typename FT>
static void fofc_nv(const Dims& d, const DevGeom& g, const Phys& ph, const khb_fields& Ps, const khb_fields& Us,
                    const khb_fields& U0, FT* const F[3], FT* const ctop[3], double g0, double g1, double bdt,
                    const double* dt_dev, double beta, int32_t* flag, cudaStream_t st)
{
    // flags are read over the interior +-2 (+-0 along periodic directions, filled from the images)
    const int p1 = d.bc[0] == KHB_BC_PERIODIC, p2 = d.bc[2] == KHB_BC_PERIODIC, p3 = d.bc[4] == KHB_BC_PERIODIC;
    const int h2 = d.ndim > 1, h3 = d.ndim > 2;
    const int i0 = d.is - (p1 ? 0 : 2), i1 = d.ie + (p1 ? 0 : 2);
    const int j0 = d.js - (p2 ? 0 : 2*h2), j1 = d.je + (p2 ? 0 : 2*h2);
    const int k0 = d.ks - (p3 ? 0 : 2*h3), k1 = d.ke + (p3 ? 0 : 2*h3);
    cudaMemsetAsync(flag, 0, sizeof(int32_t) * d.N, st);
    const Box gb = make_box(i0, j0, k0, i1 - i0 + 1, j1 - j0 + 1, k1 - k0 + 1);
    if (ph.inverter == KHB_INVERTER_KASTAUN)
        k_fofc_guess<NV, FT, true><<<box_blocks(gb), 128, 0, st>>>(d, g, ph, Ps, Us, U0, F[0], F[1], F[2], g0, g1, bdt, dt_dev, beta, flag, gb);
    else
        k_fofc_guess<NV, FT, false><<<box_blocks(gb), 128, 0, st>>>(d, g, ph, Ps, Us, U0, F[0], F[1], F[2], g0, g1, bdt, dt_dev, beta, flag, gb);
    if (ph.spherical && ph.fofc_polar_cells > 0 && d.ndim > 1) {
        for (int face = 2; face <= 3; ++face) {
            if (!phys_face(d.bc[face])) continue;
            const int ja = (face == 2) ? d.js : d.je - ph.fofc_polar_cells + 1;
            const int jb = (face == 2) ? d.js + ph.fofc_polar_cells - 1 : d.je;
            const long long n = (long long)(jb - ja + 1) * d.n1 * d.n3;
            k_fofc_rows<<<blocks_for(n, 128), 128, 0, st>>>(d, ja, jb, flag);
        }
    }
    const int pmask = (p1 ? 1 : 0) | ((h2 && p2) ? 2 : 0) | ((h3 && p3) ? 4 : 0);
    if (pmask) k_fofc_periodic<<<blocks_for(d.N, 256), 256, 0, st>>>(d, pmask, flag);
    // faces over the interior +-1 (one more along the face direction), with a left neighbour in range
    for (int dir = 1; dir <= d.ndim; ++dir) {
        const int lo_i = max(d.is - 1, dir == 1 ? 1 : 0), hi_i = min(d.ie + 1 + (dir == 1), d.n1 - 1);
        const int lo_j = h2 ? max(d.js - 1, dir == 2 ? 1 : 0) : d.js, hi_j = h2 ? min(d.je + 1 + (dir == 2), d.n2 - 1) : d.je;
        const int lo_k = h3 ? max(d.ks - 1, dir == 3 ? 1 : 0) : d.ks, hi_k = h3 ? min(d.ke + 1 + (dir == 3), d.n3 - 1) : d.ke;
        const Box fb = make_box(lo_i, lo_j, lo_k, hi_i - lo_i + 1, hi_j - lo_j + 1, hi_k - lo_k + 1);
        const unsigned nb = box_blocks(fb);
        if (dir == 1) k_fofc_replace<1, NV, FT, FT><<<nb, 128, 0, st>>>(d, g, ph, Ps, F[0], ctop[0], flag, fb);
        else if (dir == 2) k_fofc_replace<2, NV, FT, FT><<<nb, 128, 0, st>>>(d, g, ph, Ps, F[1], ctop[1], flag, fb);
        else k_fofc_replace<3, NV, FT, FT><<<nb, 128, 0, st>>>(d, g, ph, Ps, F[2], ctop[2], flag, fb);
    }
}
template <typename FT>
void Launch<FT>::fofc(int nv, const Dims& d, const DevGeom& g, const Phys& ph, const khb_fields& Ps,
                      const khb_fields& Us, const khb_fields& U0, FT* const F[3], FT* const ctop[3], double g0,
                      double g1, double bdt, const double* dt_dev, double beta, int32_t* flag, cudaStream_t st)
{
    if (nv == 8) fofc_nv<8, FT>(d, g, ph, Ps, Us, U0, F, ctop, g0, g1, bdt, dt_dev, beta, flag, st);
    else fofc_nv<5, FT>(d, g, ph, Ps, Us, U0, F, ctop, g0, g1, bdt, dt_dev, beta, flag, st);
}

// Batched flux launch; ntiles == 0 returns the resident CTAs per SM of the kernel
template <int DIR, int NV, typename FT>
static int batch_flux_dir(int recon, const BatchBlock<FT>* blocks, const int* tiles, unsigned ntiles, unsigned grid,
                          int stage, cudaStream_t st)
{
    const void* fn;
    switch (recon) {
    case RECON_DONOR: fn = (const void*)k_batch_flux<DIR, RECON_DONOR, NV, FT, FT>; break;
    case RECON_MC:    fn = (const void*)k_batch_flux<DIR, RECON_MC, NV, FT, FT>; break;
    case RECON_WENO5: fn = (const void*)k_batch_flux<DIR, RECON_WENO5, NV, FT, FT>; break;
    default:          fn = (const void*)k_batch_flux<DIR, RECON_PPM, NV, FT, FT>; break;
    }
    if (ntiles == 0) {
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 128, 0);
        return occ;
    }
    const unsigned nb = grid ? grid : ntiles;
    switch (recon) {
    case RECON_DONOR: k_batch_flux<DIR, RECON_DONOR, NV, FT, FT><<<nb, 128, 0, st>>>(blocks, tiles, ntiles, stage); break;
    case RECON_MC:    k_batch_flux<DIR, RECON_MC, NV, FT, FT><<<nb, 128, 0, st>>>(blocks, tiles, ntiles, stage); break;
    case RECON_WENO5: k_batch_flux<DIR, RECON_WENO5, NV, FT, FT><<<nb, 128, 0, st>>>(blocks, tiles, ntiles, stage); break;
    default:          k_batch_flux<DIR, RECON_PPM, NV, FT, FT><<<nb, 128, 0, st>>>(blocks, tiles, ntiles, stage); break;
    }
    return 0;
}
template <int NV, typename FT>
static int batch_flux_nv(int recon, int dir, const BatchBlock<FT>* blocks, const int* tiles, unsigned ntiles,
                         unsigned grid, int stage, cudaStream_t st)
{
    if (dir == 1) return batch_flux_dir<1, NV, FT>(recon, blocks, tiles, ntiles, grid, stage, st);
    if (dir == 2) return batch_flux_dir<2, NV, FT>(recon, blocks, tiles, ntiles, grid, stage, st);
    return batch_flux_dir<3, NV, FT>(recon, blocks, tiles, ntiles, grid, stage, st);
}
template <typename FT>
int Launch<FT>::batch_flux(int recon, int nv, int dir, const BatchBlock<FT>* blocks, const int* tiles, unsigned ntiles,
                           unsigned grid, int stage, cudaStream_t st)
{
    return (nv == 8) ? batch_flux_nv<8, FT>(recon, dir, blocks, tiles, ntiles, grid, stage, st)
                     : batch_flux_nv<5, FT>(recon, dir, blocks, tiles, ntiles, grid, stage, st);
}

template <int NV, typename FT>
static int batch_flux_all_nv(int recon, const BatchBlock<FT>* blocks, const int* tiles, unsigned ntiles, unsigned grid,
                             int stage, int* const* counts, int nblocks, unsigned long long* word, cudaStream_t st)
{
    const void* fn;
    switch (recon) {
    case RECON_DONOR: fn = (const void*)k_batch_flux_all<RECON_DONOR, NV, FT, FT>; break;
    case RECON_MC:    fn = (const void*)k_batch_flux_all<RECON_MC, NV, FT, FT>; break;
    case RECON_WENO5: fn = (const void*)k_batch_flux_all<RECON_WENO5, NV, FT, FT>; break;
    default:          fn = (const void*)k_batch_flux_all<RECON_PPM, NV, FT, FT>; break;
    }
    if (ntiles == 0) {
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, 128, 0);
        return occ;
    }
    const unsigned nb = grid ? grid : ntiles;
    switch (recon) {
    case RECON_DONOR: k_batch_flux_all<RECON_DONOR, NV, FT, FT><<<nb, 128, 0, st>>>(blocks, tiles, ntiles, stage, counts, nblocks, word); break;
    case RECON_MC:    k_batch_flux_all<RECON_MC, NV, FT, FT><<<nb, 128, 0, st>>>(blocks, tiles, ntiles, stage, counts, nblocks, word); break;
    case RECON_WENO5: k_batch_flux_all<RECON_WENO5, NV, FT, FT><<<nb, 128, 0, st>>>(blocks, tiles, ntiles, stage, counts, nblocks, word); break;
    default:          k_batch_flux_all<RECON_PPM, NV, FT, FT><<<nb, 128, 0, st>>>(blocks, tiles, ntiles, stage, counts, nblocks, word); break;
    }
    return 0;
}
template <typename FT>
int Launch<FT>::batch_flux_all(int recon, int nv, const BatchBlock<FT>* blocks, const int* tiles, unsigned ntiles,
                               unsigned grid, int stage, int* const* counts, int nblocks, unsigned long long* word,
                               cudaStream_t st)
{
    return (nv == 8) ? batch_flux_all_nv<8, FT>(recon, blocks, tiles, ntiles, grid, stage, counts, nblocks, word, st)
                     : batch_flux_all_nv<5, FT>(recon, blocks, tiles, ntiles, grid, stage, counts, nblocks, word, st);
}

template <int NV, typename FT, int MODE>
static int batch_zone_mode(const BatchBlock<FT>* blocks, const int* tiles, unsigned ntiles, unsigned grid, int stage,
                           int dtm, double beta, const double* dt, cudaStream_t st)
{
    if (ntiles == 0) {
        int occ = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, (const void*)k_batch_zone<NV, FT, MODE>, 128, 0);
        return occ;
    }
    k_batch_zone<NV, FT, MODE><<<grid ? grid : ntiles, 128, 0, st>>>(blocks, tiles, ntiles, stage, dtm, beta, dt);
    return 0;
}
template <typename FT>
int Launch<FT>::batch_zone(int nv, int mode, const BatchBlock<FT>* blocks, const int* tiles, unsigned ntiles,
                           unsigned grid, int stage, int dtm, double beta, const double* dt, cudaStream_t st)
{
    if ((mode & ~M_KASTAUN) == M_ZONE_FUSED) {
        // the fused plan: update and cell halves in one pass
        const bool kast = mode & M_KASTAUN;
        if (nv == 8) return kast ? batch_zone_mode<8, FT, M_ZONE_FUSED | M_KASTAUN>(blocks, tiles, ntiles, grid, stage, dtm, beta, dt, st)
                                 : batch_zone_mode<8, FT, M_ZONE_FUSED>(blocks, tiles, ntiles, grid, stage, dtm, beta, dt, st);
        return kast ? batch_zone_mode<5, FT, M_ZONE_FUSED | M_KASTAUN>(blocks, tiles, ntiles, grid, stage, dtm, beta, dt, st)
                    : batch_zone_mode<5, FT, M_ZONE_FUSED>(blocks, tiles, ntiles, grid, stage, dtm, beta, dt, st);
    }
    if (nv == 8) {
        if (mode == M_UPDATE) return batch_zone_mode<8, FT, M_UPDATE>(blocks, tiles, ntiles, grid, stage, dtm, beta, dt, st);
        if (mode & M_KASTAUN)
            return batch_zone_mode<8, FT, M_ZONE_CELL | M_KASTAUN>(blocks, tiles, ntiles, grid, stage, dtm, beta, dt, st);
        return batch_zone_mode<8, FT, M_ZONE_CELL>(blocks, tiles, ntiles, grid, stage, dtm, beta, dt, st);
    }
    if (mode == M_UPDATE) return batch_zone_mode<5, FT, M_UPDATE>(blocks, tiles, ntiles, grid, stage, dtm, beta, dt, st);
    if (mode & M_KASTAUN)
        return batch_zone_mode<5, FT, M_ZONE_CELL | M_KASTAUN>(blocks, tiles, ntiles, grid, stage, dtm, beta, dt, st);
    return batch_zone_mode<5, FT, M_ZONE_CELL>(blocks, tiles, ntiles, grid, stage, dtm, beta, dt, st);
}

template <typename FT>
void Launch<FT>::mesh_flux(int nv, const BatchBlock<FT>* blocks, const int* table, long long n, cudaStream_t st)
{
    if (n > 0) k_mesh_flux<FT><<<blocks_for(n, 128), 128, 0, st>>>(blocks, table, n, nv);
}

template <typename FT>
void Launch<FT>::mesh_ghost_cell(int nv, bool kastaun, const BatchBlock<FT>* blocks, const int* table, long long n,
                                 int s, int standalone, cudaStream_t st)
{
    if (n <= 0) return;
    constexpr int C = M_UTOP | M_FLOORS | M_PTOU;
    const unsigned nb = blocks_for(n, 128);
    if (nv == 8) {
        if (kastaun) k_mesh_ghost_cell<8, FT, C | M_KASTAUN><<<nb, 128, 0, st>>>(blocks, table, n, s, standalone);
        else k_mesh_ghost_cell<8, FT, C><<<nb, 128, 0, st>>>(blocks, table, n, s, standalone);
    } else {
        if (kastaun) k_mesh_ghost_cell<5, FT, C | M_KASTAUN><<<nb, 128, 0, st>>>(blocks, table, n, s, standalone);
        else k_mesh_ghost_cell<5, FT, C><<<nb, 128, 0, st>>>(blocks, table, n, s, standalone);
    }
}

#ifdef KHB_COMMON_KERNELS
void LaunchCommon::mesh_ghost(int nv, const FixupBlock* blocks, const int* table, long long begin, long long end,
                              int stage, cudaStream_t st)
{
    if (end <= begin) return;
    if (nv == 8) k_mesh_ghost<8><<<blocks_for(end - begin, 128), 128, 0, st>>>(blocks, table, begin, end, stage);
    else k_mesh_ghost<5><<<blocks_for(end - begin, 128), 128, 0, st>>>(blocks, table, begin, end, stage);
}

void LaunchCommon::mesh_ghost_cons(int nv, const FixupBlock* blocks, const int* table, long long begin,
                                   long long end, int seed_sel, int u_sel, cudaStream_t st)
{
    if (end <= begin) return;
    if (nv == 8) k_mesh_ghost_cons<8><<<blocks_for(end - begin, 128), 128, 0, st>>>(blocks, table, begin, end, seed_sel, u_sel);
    else k_mesh_ghost_cons<5><<<blocks_for(end - begin, 128), 128, 0, st>>>(blocks, table, begin, end, seed_sel, u_sel);
}

void LaunchCommon::batch_fixup(int nv, const FixupBlock* blocks, int nblocks, int stage, cudaStream_t st)
{
    const dim3 grid(4, nblocks);
    if (nv == 8) k_batch_fixup<8><<<grid, 128, 0, st>>>(blocks, stage);
    else k_batch_fixup<5><<<grid, 128, 0, st>>>(blocks, stage);
}

void LaunchCommon::batch_reset(int* const* counts, int nblocks, unsigned long long* word, cudaStream_t st)
{
    k_batch_reset<<<blocks_for(nblocks, 128), 128, 0, st>>>(counts, nblocks, word);
}

void LaunchCommon::stage_reset(int* count, unsigned long long* word, cudaStream_t st)
{
    k_stage_reset<<<1, 1, 0, st>>>(count, word);
}

void LaunchCommon::next_dt(const unsigned long long* ndt_word, double* state, double cfl, double dt_min,
                           double max_dt_increase, cudaStream_t st)
{
    k_next_dt<<<1, 1, 0, st>>>(ndt_word, state, cfl, dt_min, max_dt_increase);
}

void LaunchCommon::fixup(int nv, const Dims& d, const DevGeom& g, const Phys& ph, const khb_fields& P,
                         const khb_fields& U, const int32_t* pflag, const int* fail_count, const int* fail_list,
                         cudaStream_t st)
{
    const unsigned nb = 4 * 148;
    if (nv == 8) k_fixup<8><<<nb, 128, 0, st>>>(d, g, ph, P, U, pflag, fail_count, fail_list);
    else k_fixup<5><<<nb, 128, 0, st>>>(d, g, ph, P, U, pflag, fail_count, fail_list);
}

void LaunchCommon::bc(int nv, const Dims& d, const DevGeom& g, const Phys& ph, const khb_fields& P, const khb_fields& U,
                      int face, int lo_a, int cnt_a, int lo_k, int cnt_k, cudaStream_t st)
{
    const int ng = (face < 2) ? d.is : ((face < 4) ? d.js : d.ks);
    const unsigned nb = blocks_for((long long)ng*cnt_a*cnt_k, 128);
    if (nv == 10) k_bc<10><<<nb, 128, 0, st>>>(d, g, ph, P, U, face, lo_a, cnt_a, lo_k, cnt_k);
    else if (nv == 8) k_bc<8><<<nb, 128, 0, st>>>(d, g, ph, P, U, face, lo_a, cnt_a, lo_k, cnt_k);
    else k_bc<5><<<nb, 128, 0, st>>>(d, g, ph, P, U, face, lo_a, cnt_a, lo_k, cnt_k);
}

void LaunchCommon::ghost_ptou(int nv, const Dims& d, const DevGeom& g, const Phys& ph, const khb_fields& P,
                              const khb_fields& U, cudaStream_t st, const khb_fields* Bf, int ct_mask, int kplanes,
                              int pfaces)
{
    const long long plane = (long long)d.n1 * d.n2;
    const long long tot = kplanes ? plane * (((kplanes & 1) ? d.ks : 0) + ((kplanes & 2) ? d.n3 - 1 - d.ke : 0))
                                  : (long long)plane_ghost_count(d)*(d.ke - d.ks + 1);
    if (tot == 0) return;
    khb_fields F;
    for (int x = 0; x < KHB_MAX_VARS; ++x) F.v[x] = nullptr;
    if (Bf) for (int x = 0; x < 3; ++x) F.v[x] = Bf->v[x];
    if (nv == 8) k_ghost_ptou<8><<<blocks_for(tot, 128), 128, 0, st>>>(d, g, ph, P, U, F, ct_mask, kplanes, pfaces);
    else k_ghost_ptou<5><<<blocks_for(tot, 128), 128, 0, st>>>(d, g, ph, P, U, F, ct_mask, kplanes, pfaces);
}

void LaunchCommon::bound_tasks(int nv, const BoundTask* tasks, int ntasks, long long max_count, cudaStream_t st)
{
    if (ntasks <= 0 || max_count <= 0) return;
    const dim3 grid(blocks_for(max_count, 128), (unsigned)ntasks);
    if (nv == 8) k_bound_tasks<8><<<grid, 128, 0, st>>>(tasks);
    else k_bound_tasks<5><<<grid, 128, 0, st>>>(tasks);
}

void LaunchCommon::periodic(int nv, const Dims& d, const khb_fields& P, const khb_fields& U, int pmask, cudaStream_t st)
{
    const long long nint = (long long)(d.ie - d.is + 1)*(d.je - d.js + 1)*(d.ke - d.ks + 1);
    const long long tot = d.N - nint;
    if (tot == 0) return;
    if (nv == 10) k_periodic<10><<<blocks_for(tot, 256), 256, 0, st>>>(d, P, U, pmask);
    else if (nv == 8) k_periodic<8><<<blocks_for(tot, 256), 256, 0, st>>>(d, P, U, pmask);
    else k_periodic<5><<<blocks_for(tot, 256), 256, 0, st>>>(d, P, U, pmask);
}

void LaunchCommon::ghost_copy(int nv, const Dims& d, const khb_fields& Pin, const khb_fields& Uin,
                              const khb_fields& Pout, const khb_fields& Uout, cudaStream_t st)
{
    const long long nint = (long long)(d.ie - d.is + 1)*(d.je - d.js + 1)*(d.ke - d.ks + 1);
    const long long tot = d.N - nint;
    if (tot == 0) return;
    if (nv == 8) k_ghost_copy<8><<<blocks_for(tot, 256), 256, 0, st>>>(d, Pin, Uin, Pout, Uout);
    else k_ghost_copy<5><<<blocks_for(tot, 256), 256, 0, st>>>(d, Pin, Uin, Pout, Uout);
}

void LaunchCommon::batch_ghost_copy(int nv, const FixupBlock* blocks, int nblocks, int stage, cudaStream_t st)
{
    const dim3 grid(16, nblocks);
    if (nv == 8) k_batch_ghost_copy<8><<<grid, 256, 0, st>>>(blocks, stage);
    else k_batch_ghost_copy<5><<<grid, 256, 0, st>>>(blocks, stage);
}

void LaunchCommon::ptou(int nv, const Dims& d, const DevGeom& g, const Phys& ph, const khb_fields& P,
                        const khb_fields& U, cudaStream_t st)
{
    if (nv == 8) k_ptou<8><<<blocks_for(d.N, 128), 128, 0, st>>>(d, g, ph, P, U);
    else k_ptou<5><<<blocks_for(d.N, 128), 128, 0, st>>>(d, g, ph, P, U);
}

void LaunchCommon::divb(const Dims& d, const Phys& ph, const khb_fields& U, int i_lo, int i_hi,
                        unsigned long long* word, cudaStream_t st)
{
    const long long tot = (long long)(i_hi - i_lo + 1)*(d.je - d.js + 2)*((d.ndim > 2) ? d.ke - d.ks + 2 : 1);
    k_divb<<<blocks_for(tot, 256), 256, 0, st>>>(d, ph, U, i_lo, i_hi, word);
}
#endif

} // namespace khb

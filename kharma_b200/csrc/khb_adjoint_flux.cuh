// khb_adjoint_flux.cuh -- the face-flux part of the discrete adjoint (k_adj_flux), shared by
// khb_adjoint.cu (FP64 faces, built without contraction) and khb_adjoint_fp32.cu (the FP32-flux
// form's faces, built with the forward FP32 kernels' contraction and fast divide/square root).
#pragma once

#include "khb_internal.hpp"
#include "khb_dual.cuh"
#include "khb_kernels.cuh"

namespace khb {

// The MC-limited slope mc_lim(dm, dp) dp (reconstruction.hpp:52-56, 107-123)
template <typename R>
__device__ __forceinline__ R mc_slope(R dm, R dp) { return mc_lim<R>(dm, dp) * dp; }
// On dual numbers: the value as the forward forms it, the tangent from the homogeneous form of the
// branch the value takes (0, 2 dm, (1 + r)/2 dp = (dm + dp)/2, or 2 dp), so that the tangent of
// r = dm/dp, which overflows where dp is tiny (a field at the bottom of the double range), is never
// formed.  Ties follow kmin/kmax as the forward's mc_lim resolves them.
template <typename T>
__device__ __forceinline__ Dual<T> mc_slope(Dual<T> dm, Dual<T> dp)
{
    const T v = mc_lim<T>(dm.v, dp.v) * dp.v;
    if (!(fabs(dp.v) > T(0))) return Dual<T>(v, T(1.5) * dp.d);      // r = 2: phi = 3/2
    const T r = dm.v / dp.v;
    const T t2r = T(2) * r, thalf = T(0.5) * (T(1) + r);
    const bool inner_half = thalf < t2r;                    // kmin(2r, (1+r)/2)
    const T inner = inner_half ? thalf : t2r;
    const bool mid_two = !(inner < T(2));                   // kmin(2, inner)
    const T mid = mid_two ? T(2) : inner;
    if (!(T(0) < mid)) return Dual<T>(v, T(0));             // kmax(0, mid) = 0
    if (mid_two) return Dual<T>(v, T(2) * dp.d);
    if (inner_half) return Dual<T>(v, T(0.5) * (dm.d + dp.d));
    return Dual<T>(v, T(2) * dm.d);
}

// MC face values of a zone from its left, centre and right values (reconstruction.hpp:107-123)
template <typename R>
__device__ __forceinline__ R mc_right(R xm, R x0, R xp) { return x0 + R(0.5) * mc_slope(x0 - xm, xp - x0); }
template <typename R>
__device__ __forceinline__ R mc_left(R xm, R x0, R xp) { return x0 - R(0.5) * mc_slope(x0 - xm, xp - x0); }

// One side of a face in arithmetic R: conserved state, flux and signal speeds (get_flux.hpp:219-331)
template <typename R, int NV, int DIR>
__device__ __forceinline__ void face_side(const R gcov[4][4], const R* gcon0, R gcondd, R gdet, R gam, const R* P,
                                          R* U, R* F, R& cmax, R& cmin)
{
    FourVec<R> D;
    calc_4vecs<R, (NV > 5)>(gcov, gcon0[0], gcon0, P, D);
    prim_to_flux<R, NV>(P, D, gam, gdet, 0, U);
    prim_to_flux<R, NV>(P, D, gam, gdet, DIR, F);
    vchar<R, (NV > 5)>(P, D, gam, gcon0[0], gcon0[DIR], gcondd, DIR, cmax, cmin);
}

// ---------------------------------------------------------------------------- face fluxes
// Pbar += (dF/dP)^T Fbar for every face of the box (faces [s, e+1] along DIR, [s-1, e+1] across).
// R: the arithmetic of the forward face kernel (double, or float in the FP32-flux form).
// The hydro components of Fbar are formed here from Ubar_upd (zero outside the interior): the
// transpose of U_upd(c) += bdt (area_d/vol) (F_d(c) - F_d(c+st)) gives Fbar_d(c) = area_d w (Ubar_upd(c) -
// Ubar_upd(c-st)) with w = bdt/vol; the magnetic components (flux-CT) come scattered from k_adj_update
// in Fbar; the objective's seed (scale * weight on the X1 mass flux) is added for DIR = 1.
template <int DIR, int NV, int RECON, typename R>
__global__ void __launch_bounds__(128) k_adj_flux(Dims d, DevGeom g, Phys ph, khb_fields P, const double* Fbar,
                                                  const double* Uupd, double w, double area, const double* seed,
                                                  double seed_scale, khb_fields Pbar, Box bx)
{
    int i, j, k;
    if (!box_cell(bx, blockIdx.x, i, j, k)) return;
    const long long c = ((long long)k*d.n2 + j)*d.n1 + i;
    const long long st = (DIR == 1) ? 1 : ((DIR == 2) ? d.sj : d.sk);
    // KBoundaries::FixFlux zero_polar_flux (boundaries.cpp:672-684): these faces carry no flux
    if (DIR == 2 && ph.zero_polar_flux &&
        ((j == d.js && phys_face(d.bc[2])) || (j == d.je + 1 && phys_face(d.bc[3]))))
        return;
    // B_FluxCT's polar fix zeroes the X2 B1 and B3 fluxes on the polar faces
    const bool polar_b = NV > 5 && DIR == 2 && ph.fix_polar_flux &&
                         ((j == d.js && phys_face(d.bc[2])) || (j == d.je + 1 && phys_face(d.bc[3])));
    double fb[NV];
    bool any = false;
#pragma unroll
    for (int p = 0; p < 5; ++p) {
        const double hi = area * (w * Uupd[p*d.N + c]), lo = -(area * (w * Uupd[p*d.N + c - st]));
        fb[p] = (DIR == 1 && p == 0 && seed) ? (seed_scale * seed[c] + hi) + lo : hi + lo;
        any |= fb[p] != 0.;
    }
#pragma unroll
    for (int p = 5; p < NV; ++p) {
        fb[p] = (polar_b && p != 6) ? 0. : Fbar[p*d.N + c];
        any |= fb[p] != 0.;
    }
    if (!any) return;
    typedef Dual<R> DR;
    const int loc = DIR - 1;
    const long long gi = (long long)j*g.G1 + i;
    // the face tables of the forward kernel's arithmetic (FP32 copies in the FP32-flux form)
    const auto* tcov = FaceTables<R>::gcov(g, loc);
    const auto* tcon = FaceTables<R>::gcon(g, loc);
    R gcov[4][4], gcon0[4];
#pragma unroll
    for (int m = 0; m < 16; ++m) gcov[m/4][m%4] = (R)__ldg(tcov + m*g.gs + gi);
#pragma unroll
    for (int m = 0; m < 4; ++m) gcon0[m] = (R)__ldg(tcon + m*g.gs + gi);
    const R gcondd = (R)__ldg(tcon + (DIR*4 + DIR)*g.gs + gi);
    const R gdet = (R)__ldg(FaceTables<R>::gdet(g, loc) + gi);
    const R gam = (R)ph.gam;
    // stencil c-2 .. c+1 (MC uses zones c-2..c for the left state and c-1..c+1 for the right)
    R x[4][NV];
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
        for (int p = 0; p < NV; ++p) x[s][p] = (R)P.v[p][c + (s - 2)*st];
    R Pl[NV], Pr[NV];
#pragma unroll
    for (int p = 0; p < NV; ++p) {
        if (RECON == RECON_DONOR) { Pl[p] = x[1][p]; Pr[p] = x[2][p]; }
        else { Pl[p] = mc_right<R>(x[0][p], x[1][p], x[2][p]); Pr[p] = mc_left<R>(x[1][p], x[2][p], x[3][p]); }
    }
    // values of both sides
    R Uv[2][NV], Fv[2][NV], cmx[2], cmn[2];
    face_side<R, NV, DIR>(gcov, gcon0, gcondd, gdet, gam, Pl, Uv[0], Fv[0], cmx[0], cmn[0]);
    face_side<R, NV, DIR>(gcov, gcon0, gcondd, gdet, gam, Pr, Uv[1], Fv[1], cmx[1], cmn[1]);
    // KBoundaries::FixFlux inflow checks (boundaries.cpp:611-660): the X1 domain faces' mass flux
    // clipped to outflow; where the clip acted, the flux no longer depends on the state
    if (DIR == 1) {
        const bool in = i == d.is && ph.check_inflow_in && phys_face(d.bc[0]);
        const bool out = i == d.ie + 1 && ph.check_inflow_out && phys_face(d.bc[1]);
        if (in || out) {
            const R cmax = kmax(kmax(R(0), cmx[0]), cmx[1]);
            const R cmin = -kmin(kmin(R(0), cmn[0]), cmn[1]);
            const R ctp = kmax(cmax, cmin);
            const R f0 = R(0.5) * (Fv[0][0] + Fv[1][0] - ctp * (Uv[1][0] - Uv[0][0]));
            if ((in && f0 > R(0)) || (out && f0 < R(0))) fb[0] = 0.;
        }
    }
    // dual geometry
    DR Dgcov[4][4], Dgcon0[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        Dgcon0[a] = DR(gcon0[a]);
#pragma unroll
        for (int b = 0; b < 4; ++b) Dgcov[a][b] = DR(gcov[a][b]);
    }
    const DR Dgcondd(gcondd), Dgdet(gdet), Dgam(gam);
    double Pbar_side[2][NV];
    for (int side = 0; side < 2; ++side) {
        const R* Ps = side ? Pr : Pl;
        for (int q = 0; q < NV; ++q) {
            DR Pd[NV];
#pragma unroll
            for (int p = 0; p < NV; ++p) Pd[p] = DR(Ps[p], (p == q) ? R(1) : R(0));
            DR Ud[NV], Fd[NV], cmaxd, cmind;
            face_side<DR, NV, DIR>(Dgcov, Dgcon0, Dgcondd, Dgdet, Dgam, Pd, Ud, Fd, cmaxd, cmind);
            // LLF of the two sides with this side in duals (flux.hpp:110-121, get_flux.hpp:274-331)
            const DR o_cmax(cmx[1 - side]), o_cmin(cmn[1 - side]);
            const DR cmaxL = side ? o_cmax : cmaxd, cminL = side ? o_cmin : cmind;
            const DR cmaxR = side ? cmaxd : o_cmax, cminR = side ? cmind : o_cmin;
            const DR cmax = kmax(kmax(DR(R(0)), cmaxL), cmaxR);
            const DR cmin = -kmin(kmin(DR(R(0)), cminL), cminR);
            const DR ctp = kmax(cmax, cmin);
            double acc = 0.;
#pragma unroll
            for (int p = 0; p < NV; ++p) {
                const DR FL = side ? DR(Fv[0][p]) : Fd[p], FR = side ? Fd[p] : DR(Fv[1][p]);
                const DR UL = side ? DR(Uv[0][p]) : Ud[p], UR = side ? Ud[p] : DR(Uv[1][p]);
                const DR f = DR(R(0.5)) * (FL + FR - ctp * (UR - UL));
                acc += fb[p] * (double)f.d;
            }
            Pbar_side[side][q] = acc;
        }
    }
    // through the reconstruction to the stencil zones
#pragma unroll
    for (int p = 0; p < NV; ++p) {
        if (RECON == RECON_DONOR) {
            atomicAdd(Pbar.v[p] + c - st, Pbar_side[0][p]);
            atomicAdd(Pbar.v[p] + c, Pbar_side[1][p]);
            continue;
        }
        double gl[3], gr[3];
#pragma unroll
        for (int s = 0; s < 3; ++s) {
            DR a[3];
#pragma unroll
            for (int t = 0; t < 3; ++t) a[t] = DR(x[t][p], (t == s) ? R(1) : R(0));
            gl[s] = (double)mc_right<DR>(a[0], a[1], a[2]).d;
            DR b[3];
#pragma unroll
            for (int t = 0; t < 3; ++t) b[t] = DR(x[t + 1][p], (t == s) ? R(1) : R(0));
            gr[s] = (double)mc_left<DR>(b[0], b[1], b[2]).d;
        }
        // left state from zones c-2, c-1, c; right state from c-1, c, c+1
        atomicAdd(Pbar.v[p] + c - 2*st, Pbar_side[0][p] * gl[0]);
        atomicAdd(Pbar.v[p] + c - st, Pbar_side[0][p] * gl[1] + Pbar_side[1][p] * gr[0]);
        atomicAdd(Pbar.v[p] + c, Pbar_side[0][p] * gl[2] + Pbar_side[1][p] * gr[1]);
        atomicAdd(Pbar.v[p] + c + st, Pbar_side[1][p] * gr[2]);
    }
}

// Launch of k_adj_flux<DIR, NV, RECON, float> over the box (defined in khb_adjoint_fp32.cu for
// RECON_MC and RECON_DONOR, DIR 1-3, NV 5 and 8)
template <int DIR, int NV, int RECON>
void launch_adj_flux_f32(cudaStream_t st, const Dims& d, const DevGeom& g, const Phys& ph, const khb_fields& P,
                         const double* Fbar, const double* Uupd, double w, double area, const double* seed,
                         double seed_scale, const khb_fields& Pbar, const Box& bx);

} // namespace khb

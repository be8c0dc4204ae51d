// khb_adjoint.cu -- discrete adjoint of the explicit RK2 stage (the differentiation form).
//
// For one stage (P_s, U_s, U_0) -> (P_out, U_out) of khb_stage, and given the adjoint of its output
// (Pbar_out, Ubar_out), accumulate the adjoints of its inputs.  The stage is the composition
//   face fluxes F_d(P_s)  (MC or donor-cell reconstruction, prim_to_flux, vchar, LLF)
//   U_upd = g0 U_s + g1 U_0 + beta dt (-div F(flux-CT for B) + S(P_s))   (geometric source S)
//   P_out = inverse of U(P) at U_upd (1D_W / Kastaun), U_out = U(P_out) (the lock-step P -> U)
// whose adjoint, in reverse order, is
//   Ubar_upd = Ubar_out + J(P_out)^-T Pbar_out           (implicit-function adjoint of the inversion;
//                                                           J = dU/dP, so U_out = U_upd to the inverter's
//                                                           tolerance and contributes Ubar_out)
//   Ubar_s += g0 Ubar_upd, Ubar_0 += g1 Ubar_upd,
//   Fbar += transpose of the divergence (and of flux-CT), Pbar_s += beta dt (dS/dP)^T Ubar_upd,
//   Pbar_s += (dF/dP_stencil)^T Fbar                      (per face, scattered with atomics).
// Local Jacobians come from the same templated device functions the forward kernels use, evaluated
// on Dual numbers with one unit tangent per input.  With floors (fluid or drift frame, 1D_W), the
// recompute keeps each stage's inverted primitives before the floors, and a floored zone's adjoint
// passes through the floor map's Jacobian (k_adj_cell); a zone whose inversion failed takes the
// adjoint of its fixup (k_adj_fixup).  Out of scope (rejected): normal-frame and mixed-frame floors,
// reconstruction floors, FOFC, transmitting faces, WENO5/PPM, HLLE.  Periodic ghost zones are
// copies of their images, so their adjoints are folded into the images; exchange ghost zones are
// the caller's constants and their adjoints are dropped.  The timestep is taken as given (the
// forward run's sequence).
#include "khb_adjoint_flux.cuh"

#include <cstring>
#include <string>

namespace khb {

// ---------------------------------------------------------------------------- update
// Adjoint of U_upd = g0 U_s + g1 U_0 + bdt (-div F + S(P_s)) over the interior: Fbar (atomics),
// Pbar_s (own zone), Ubar_s and Ubar_0 (own zone; they may be the same array).
template <int NV>
__global__ void __launch_bounds__(128) k_adj_update(Dims d, DevGeom g, Phys ph, const double* Ubar_upd, khb_fields Ps,
                                                    double g0, double g1, double bdt, double* F1b, double* F2b,
                                                    double* F3b, khb_fields Pbar_s, khb_fields Ubar_s,
                                                    khb_fields Ubar_0, Box bx)
{
    int i, j, k;
    if (!box_cell(bx, blockIdx.x, i, j, k)) return;
    const long long c = ((long long)k*d.n2 + j)*d.n1 + i;
    const long long N = d.N, sj = d.sj, sk = d.sk;
    double ub[NV];
    bool any = false;
#pragma unroll
    for (int p = 0; p < NV; ++p) { ub[p] = Ubar_upd[p*N + c]; any |= ub[p] != 0.; }
    if (!any) return;
#pragma unroll
    for (int p = 0; p < NV; ++p) {
        Ubar_s.v[p][c] += g0 * ub[p];
        Ubar_0.v[p][c] += g1 * ub[p];
    }
    const double a1 = ph.dx2*ph.dx3, a2 = ph.dx1*ph.dx3, a3 = ph.dx1*ph.dx2;
    const double w = bdt / (ph.dx1*ph.dx2*ph.dx3);
    // the hydro divergence's transpose is gathered per face by k_adj_flux
    if (NV > 5) {
        // flux-CT (b_flux_ct.cpp:307-370) as ct_divergence forms it: face B fluxes from corner EMFs,
        // EMFs from the raw B fluxes; transposed term by term
        const long long B1 = 5*N, B2 = 6*N, B3 = 7*N;
        const bool d3 = d.ndim > 2;
        auto e3 = [&](long long x, double v) {      // e3 = 0.25 (F1[B2](x) + F1[B2](x-sj) - F2[B1](x) - F2[B1](x-1))
            atomicAdd(F1b + B2 + x, 0.25 * v); atomicAdd(F1b + B2 + x - sj, 0.25 * v);
            atomicAdd(F2b + B1 + x, -0.25 * v); atomicAdd(F2b + B1 + x - 1, -0.25 * v);
        };
        auto e1 = [&](long long x, double v) {      // e1 = 0.25 (F2[B3](x) + F2[B3](x-sk) - F3[B2](x) - F3[B2](x-sj))
            atomicAdd(F2b + B3 + x, 0.25 * v); atomicAdd(F2b + B3 + x - sk, 0.25 * v);
            atomicAdd(F3b + B2 + x, -0.25 * v); atomicAdd(F3b + B2 + x - sj, -0.25 * v);
        };
        auto e2 = [&](long long x, double v) {      // e2 = 0.25 (F3[B1](x) + F3[B1](x-1) - F1[B3](x) - F1[B3](x-sk))
            atomicAdd(F3b + B1 + x, 0.25 * v); atomicAdd(F3b + B1 + x - 1, 0.25 * v);
            atomicAdd(F1b + B3 + x, -0.25 * v); atomicAdd(F1b + B3 + x - sk, -0.25 * v);
        };
        // adjoints of the face B fluxes: U_B[v] += -bdt (a_d (fb[d][v][hi] - fb[d][v][lo]))/vol
        double fbb[3][3][2];
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            const double u = w * ub[5 + v];
            fbb[0][v][1] = -a1 * u; fbb[0][v][0] = a1 * u;
            fbb[1][v][1] = (d.ndim >= 2) ? -a2 * u : 0.; fbb[1][v][0] = (d.ndim >= 2) ? a2 * u : 0.;
            fbb[2][v][1] = (d.ndim == 3) ? -a3 * u : 0.; fbb[2][v][0] = (d.ndim == 3) ? a3 * u : 0.;
        }
        if (d.ndim >= 2) {
            if (ph.zero_polar_flux) {
                if (j == d.js && phys_face(d.bc[2])) { fbb[1][0][0] = 0.; fbb[1][1][0] = 0.; fbb[1][2][0] = 0.; }
                if (j == d.je && phys_face(d.bc[3])) { fbb[1][0][1] = 0.; fbb[1][1][1] = 0.; fbb[1][2][1] = 0.; }
            }
            // X1 faces: fb[0][1] = 0.5 (e3 + e3), fb[0][2] = -0.5 (e2 + e2) or raw F1[B3]
            e3(c, 0.5 * fbb[0][1][0]); e3(c + sj, 0.5 * fbb[0][1][0]);
            e3(c + 1, 0.5 * fbb[0][1][1]); e3(c + 1 + sj, 0.5 * fbb[0][1][1]);
            if (d3) {
                e2(c, -0.5 * fbb[0][2][0]); e2(c + sk, -0.5 * fbb[0][2][0]);
                e2(c + 1, -0.5 * fbb[0][2][1]); e2(c + 1 + sk, -0.5 * fbb[0][2][1]);
            } else {
                atomicAdd(F1b + B3 + c, fbb[0][2][0]); atomicAdd(F1b + B3 + c + 1, fbb[0][2][1]);
            }
            // X2 faces: fb[1][0] = -0.5 (e3 + e3), fb[1][2] = 0.5 (e1 + e1) or raw F2[B3]
            e3(c, -0.5 * fbb[1][0][0]); e3(c + 1, -0.5 * fbb[1][0][0]);
            e3(c + sj, -0.5 * fbb[1][0][1]); e3(c + sj + 1, -0.5 * fbb[1][0][1]);
            if (d3) {
                e1(c, 0.5 * fbb[1][2][0]); e1(c + sk, 0.5 * fbb[1][2][0]);
                e1(c + sj, 0.5 * fbb[1][2][1]); e1(c + sj + sk, 0.5 * fbb[1][2][1]);
                // X3 faces: fb[2][0] = 0.5 (e2 + e2), fb[2][1] = -0.5 (e1 + e1)
                e2(c, 0.5 * fbb[2][0][0]); e2(c + 1, 0.5 * fbb[2][0][0]);
                e2(c + sk, 0.5 * fbb[2][0][1]); e2(c + sk + 1, 0.5 * fbb[2][0][1]);
                e1(c, -0.5 * fbb[2][1][0]); e1(c + sj, -0.5 * fbb[2][1][0]);
                e1(c + sk, -0.5 * fbb[2][1][1]); e1(c + sk + sj, -0.5 * fbb[2][1][1]);
            } else {
                atomicAdd(F2b + B3 + c, fbb[1][2][0]); atomicAdd(F2b + B3 + c + sj, fbb[1][2][1]);
            }
        } else {
#pragma unroll
            for (int v = 0; v < 3; ++v) {
                atomicAdd(F1b + (5 + v)*N + c, fbb[0][v][0]);
                atomicAdd(F1b + (5 + v)*N + c + 1, fbb[0][v][1]);
            }
        }
    }
    // geometric source (flux.cpp:395-444): Pbar_s += bdt (dS/dP)^T Ubar[1..4]
    if (!ph.cart_minkowski) {
        typedef Dual<double> DD;
        ZoneGeom G;
        load_zone_geom(g, j, i, G);
        DD gcov[4][4], gcon0[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            gcon0[a] = DD(G.gcon[0][a]);
#pragma unroll
            for (int b = 0; b < 4; ++b) gcov[a][b] = DD(G.gcov[a][b]);
        }
        const long long cg = (long long)j*g.n1 + i, cs = (long long)(d.n2)*g.n1;
        // S_lam = sum_{mu,nu} T^mu_nu gdet Gamma^nu_{lam mu}, so sum_lam Ubar[1+lam] dS_lam/dP_q =
        // sum_{mu,nu} dT^mu_nu/dP_q W[mu][nu] with W[mu][nu] = sum_lam Ubar[1+lam] gdet Gamma^nu_{lam mu}
        double W[4][4];
#pragma unroll
        for (int mu = 0; mu < 4; ++mu)
#pragma unroll
            for (int nu = 0; nu < 4; ++nu) {
                double s = 0.;
#pragma unroll
                for (int lam = 0; lam < 4; ++lam) s += ub[1 + lam] * __ldg(g.gdet_conn + ((nu*4 + lam)*4 + mu)*cs + cg);
                W[mu][nu] = s;
            }
        double P0[NV];
#pragma unroll
        for (int p = 0; p < NV; ++p) P0[p] = Ps.v[p][c];
        for (int q = 0; q < NV; ++q) {
            DD P[NV];
#pragma unroll
            for (int p = 0; p < NV; ++p) P[p] = DD(P0[p], (p == q) ? 1. : 0.);
            FourVec<DD> D;
            calc_4vecs<DD, (NV > 5)>(gcov, gcon0[0], gcon0, P, D);
            double acc = 0.;
#pragma unroll
            for (int mu = 0; mu < 4; ++mu) {
                DD Tmu[4];
                calc_tensor<DD, (NV > 5)>(P[0], P[1], DD(ph.gam - 1) * P[1], D, mu, Tmu);
#pragma unroll
                for (int nu = 0; nu < 4; ++nu) acc += Tmu[nu].d * W[mu][nu];
            }
            Pbar_s.v[q][c] += bdt * acc;
        }
    }
}

// ---------------------------------------------------------------------------- inversion + P -> U
// J = dU/dP at P (conserved from primitives, flux_functions.hpp:343-352) by NV dual evaluations
template <int NV>
__device__ __forceinline__ void ptou_jacobian(const ZoneGeom& G, double gam, const double* P0, double J[NV][NV])
{
    typedef Dual<double> DD;
    DD gcov[4][4], gcon0[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        gcon0[a] = DD(G.gcon[0][a]);
#pragma unroll
        for (int b = 0; b < 4; ++b) gcov[a][b] = DD(G.gcov[a][b]);
    }
    for (int q = 0; q < NV; ++q) {
        DD P[NV], U[NV];
#pragma unroll
        for (int p = 0; p < NV; ++p) P[p] = DD(P0[p], (p == q) ? 1. : 0.);
        FourVec<DD> D;
        calc_4vecs<DD, (NV > 5)>(gcov, gcon0[0], gcon0, P, D);
        prim_to_flux<DD, NV>(P, D, DD(gam), DD(G.gdet), 0, U);
#pragma unroll
        for (int p = 0; p < NV; ++p) J[p][q] = U[p].d;
    }
}

// Solve A^T y = b in place (b <- y) by Gaussian elimination with partial pivoting on A^T
template <int N>
__device__ __forceinline__ void solve_transposed(double A[N][N], double b[N])
{
    double M[N][N];
#pragma unroll
    for (int r = 0; r < N; ++r)
#pragma unroll
        for (int s = 0; s < N; ++s) M[r][s] = A[s][r];
    for (int col = 0; col < N; ++col) {
        int piv = col;
        double best = fabs(M[col][col]);
        for (int r = col + 1; r < N; ++r) if (fabs(M[r][col]) > best) { best = fabs(M[r][col]); piv = r; }
        if (piv != col) {
            for (int s = 0; s < N; ++s) { const double t = M[col][s]; M[col][s] = M[piv][s]; M[piv][s] = t; }
            const double t = b[col]; b[col] = b[piv]; b[piv] = t;
        }
        const double inv = 1.0 / M[col][col];
        for (int r = col + 1; r < N; ++r) {
            const double f = M[r][col] * inv;
            for (int s = col; s < N; ++s) M[r][s] -= f * M[col][s];
            b[r] -= f * b[col];
        }
    }
    for (int r = N - 1; r >= 0; --r) {
        double s = b[r];
        for (int t = r + 1; t < N; ++t) s -= M[r][t] * b[t];
        b[r] = s / M[r][r];
    }
}

// ---------------------------------------------------------------------------- floors
// The floors of one zone on dual numbers: the operations of determine_floors, apply_floors_frame
// (fluid and drift frames) and apply_ceilings (floors_functions.hpp:50-252, floors_impl.hpp:77-125)
// in the same order, every branch taken by the value as the forward evaluation takes it.  Called
// only for zones the forward run floored (fflag != 0), as the forward applies the frame and the
// ceilings only there.  P: rho, u, u1-u3 (and B1-B3); the fluid primitives are replaced.
template <int NV>
__device__ void floors_dual(const ZoneGeom& G, const Prescription& f, double rhoflr_geom, double uflr_geom,
                            double gam, int frame, Dual<double>* P)
{
    typedef Dual<double> DD;
    DD gcov[4][4], gcon0[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        gcon0[a] = DD(G.gcon[0][a]);
#pragma unroll
        for (int b = 0; b < 4; ++b) gcov[a][b] = DD(G.gcov[a][b]);
    }
    // determine_floors: the floor values
    FourVec<DD> D;
    calc_4vecs<DD, (NV > 5)>(gcov, gcon0[0], gcon0, P, D);
    const DD bsq = dot4(D.bcon, D.bcov);
    const DD rhoflr_b = bsq / DD(f.bsq_over_rho_max);
    const DD uflr_b = bsq / DD(f.bsq_over_u_max);
    const DD uflr_max = kmax(DD(uflr_geom), uflr_b);
    DD rhoflr_max;
    if (!f.temp_adjust_u) {
        const DD rhoflr_temp = kmax(P[1], uflr_max) / DD(f.u_over_rho_max);
        rhoflr_max = kmax(kmax(DD(rhoflr_geom), rhoflr_b), rhoflr_temp);
    } else {
        rhoflr_max = kmax(DD(rhoflr_geom), rhoflr_b);
    }
    // apply_floors_frame
    if (frame == KHB_FRAME_FLUID) {
        P[0] += kmax(DD(0.), rhoflr_max - P[0]);
        P[1] += kmax(DD(0.), uflr_max - P[1]);
    } else {
        const double lapse2 = 1. / (-G.gcon[0][0]);
        double beta[4] = {0., 0., 0., 0.};
        beta[1] = lapse2 * G.gcon[0][1];
        beta[2] = lapse2 * G.gcon[0][2];
        beta[3] = lapse2 * G.gcon[0][3];
        const DD rho = P[0], uu = P[1];
        const DD pg = DD(gam - 1.) * uu;
        const DD w_old = kmax(rho + uu + pg, DD(1e-20));
        DD Bcon[4] = {DD(0.), DD(0.), DD(0.), DD(0.)}, Bcov[4] = {DD(0.), DD(0.), DD(0.), DD(0.)};
        if (NV > 5) { Bcon[1] = P[5]; Bcon[2] = P[6]; Bcon[3] = P[7]; }
#pragma unroll
        for (int mu = 0; mu < 4; ++mu)
#pragma unroll
            for (int nu = 0; nu < 4; ++nu) Bcov[mu] += gcov[mu][nu] * Bcon[nu];
        const DD Bsq = kmax(dot4(Bcon, Bcov), DD(1e-20));
        const DD B_mag = dsqrt(Bsq);
        DD Qcov[4];
        Qcov[0] = w_old * D.ucon[0] * D.ucov[0] + pg;
        Qcov[1] = w_old * D.ucon[0] * D.ucov[1];
        Qcov[2] = w_old * D.ucon[0] * D.ucov[2];
        Qcov[3] = w_old * D.ucon[0] * D.ucov[3];
        const DD QdotB = dot4(Bcon, Qcov);
        DD vpar = QdotB / (B_mag * w_old * D.ucon[0] * D.ucon[0]);
        DD ucon_dr[4] = {DD(0.), DD(0.), DD(0.), DD(0.)};
        ucon_dr[0] = DD(1.) / dsqrt(DD(1.) / (D.ucon[0] * D.ucon[0]) + vpar * vpar);
#pragma unroll
        for (int mu = 0; mu < 4; ++mu)
            ucon_dr[mu] = D.ucon[mu] * (ucon_dr[0] / D.ucon[0]) - (vpar * Bcon[mu] * ucon_dr[0] / B_mag);
        P[0] = kmax(rho, rhoflr_max);
        P[1] = kmax(uu, uflr_max);
        const DD pg_new = DD(gam - 1.) * P[1];
        const DD w_new = P[0] + P[1] + pg_new;
        const DD x = (DD(2.) * QdotB) / (B_mag * w_new * ucon_dr[0]);
        vpar = x / (DD(1.) + dsqrt(DD(1.) + x * x)) * (DD(1.) / ucon_dr[0]);
        DD uc[4];
        uc[0] = DD(1.) / dsqrt(DD(1.) / (ucon_dr[0] * ucon_dr[0]) - vpar * vpar);
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) uc[mu] = ucon_dr[mu] * (uc[0] / ucon_dr[0]) + (vpar * Bcon[mu] * uc[0] / B_mag);
        P[2] = uc[1] + (DD(beta[1]) * uc[0]);
        P[3] = uc[2] + (DD(beta[2]) * uc[0]);
        P[4] = uc[3] + (DD(beta[3]) * uc[0]);
    }
    // apply_ceilings
    const DD gamma = lorentz(gcov, P[2], P[3], P[4]);
    if (gamma.v > f.gamma_max) {
        const DD fr = dsqrt(DD(f.gamma_max * f.gamma_max - 1.) / (gamma * gamma - DD(1.)));
#pragma unroll
        for (int v = 0; v < 3; ++v) P[2 + v] *= fr;
    }
    if (ktot_above(gam, P[0].v, P[1].v, f.ktot_max)) {
        // d pow(rho, gam) = gam pow(rho, gam) / rho d rho
        const double pw = pow(P[0].v, gam);
        const DD rg(pw, gam * pw / P[0].v * P[0].d);
        const DD ktot = DD(gam - 1.) * P[1] / rg;
        P[1] = DD(f.ktot_max) / ktot * P[1];
    }
    if (f.temp_adjust_u && P[1].v / P[0].v > f.u_over_rho_max) P[1] = DD(f.u_over_rho_max) * P[0];
}

// Adjoint of FixUtoP (fixup.cpp:47-156 as fixup_zone runs it): a failed zone (pflag > 0) takes the
// 1/(Manhattan + 1)-weighted average of its good neighbours' fluid primitives (the neighbourhood of
// fixup_zone: periodic directions wrap, exchange faces reach the caller's ghost zones, physical
// faces end it), raised to the geometric floors, keeps the B of its own update (B_P = U_B/sqrt(-g))
// and forms U = U(P).  With t = Pbar_out + J(P_fix)^T Ubar_out, its adjoint goes to the good interior
// neighbours' Pbar_out (fluid, by weight; a neighbour across an exchange face is the caller's
// constant), and to its own updated B (Ubar_upd_B = t_B / sqrt(-g)); its fluid update is discarded.
// Runs before k_adj_cell, which then sees the neighbours' complete Pbar_out and skips failed zones.
template <int NV>
__global__ void __launch_bounds__(128) k_adj_fixup(Dims d, DevGeom g, Phys ph, khb_fields Pout, khb_fields Pbar_out,
                                                   khb_fields Ubar_out, const int32_t* pflag, double* Ubar_upd,
                                                   Box bx)
{
    int i, j, k;
    if (!box_cell(bx, blockIdx.x, i, j, k)) return;
    const long long c = ((long long)k*d.n2 + j)*d.n1 + i;
    if (!(pflag[c] > 0)) return;
    double P[NV], J[NV][NV], t[NV];
#pragma unroll
    for (int p = 0; p < NV; ++p) P[p] = Pout.v[p][c];
    ZoneGeom G;
    load_zone_geom(g, j, i, G);
    ptou_jacobian<NV>(G, ph.gam, P, J);
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double s = Pbar_out.v[q][c];
#pragma unroll
        for (int p = 0; p < NV; ++p) s += J[p][q] * Ubar_out.v[p][c];
        t[q] = s;
    }
    // B: from the zone's own update
#pragma unroll
    for (int v = 5; v < NV; ++v) Ubar_upd[v*d.N + c] = t[v] / G.gdet;
    if (!ph.fix_avg) return;             // the atmosphere values depend on the geometry alone
    // a good neighbour of fixup_zone's neighbourhood: x the zone it reads, inside whether x is an
    // interior zone (else a ghost zone across an exchange face)
    auto neighbour = [&](int l, int m, int nn, long long& x, bool& inside) -> bool {
        int ii = i + l, jj = j + m, kk = k + nn;
        inside = true;
        if (ii < d.is || ii > d.ie) {
            const int bc = d.bc[(ii < d.is) ? 0 : 1];
            if (bc == KHB_BC_PERIODIC) ii += (ii < d.is) ? d.nx1 : -d.nx1;
            else if (bc != KHB_BC_EXCHANGE) return false;
            else inside = false;
        }
        if (jj < d.js || jj > d.je) {
            const int bc = d.bc[(jj < d.js) ? 2 : 3];
            if (d.ndim < 2) return false;
            if (bc == KHB_BC_PERIODIC) jj += (jj < d.js) ? d.nx2 : -d.nx2;
            else if (bc != KHB_BC_EXCHANGE) return false;
            else inside = false;
        }
        if (kk < d.ks || kk > d.ke) {
            const int bc = d.bc[(kk < d.ks) ? 4 : 5];
            if (d.ndim < 3) return false;
            if (bc == KHB_BC_PERIODIC) kk += (kk < d.ks) ? d.nx3 : -d.nx3;
            else if (bc != KHB_BC_EXCHANGE) return false;
            else inside = false;
        }
        x = ((long long)kk*d.n2 + jj)*d.n1 + ii;
        return !(pflag[x] > 0);
    };
    double wsum = 0., sum[2] = {0., 0.};
    for (int nn = -1; nn <= 1; nn++) for (int m = -1; m <= 1; m++) for (int l = -1; l <= 1; l++) {
        long long x;
        bool inside;
        if (!neighbour(l, m, nn, x, inside)) continue;
        const double w = 1./(abs(l) + abs(m) + abs(nn) + 1);
        wsum += w;
        sum[0] += w * Pout.v[0][x];
        sum[1] += w * Pout.v[1][x];
    }
    if (wsum < 1.e-10) return;
    // the geometric floors of the average: where one raised it, that component is a constant
    const long long cg = (long long)j*g.n1 + i;
    const double rf = g.floor_rho[cg], uf = g.floor_u[cg];
    double tf[5];
#pragma unroll
    for (int p = 0; p < 5; ++p) tf[p] = t[p] / wsum;
    if (0. < rf - sum[0]/wsum) tf[0] = 0.;
    if (0. < uf - sum[1]/wsum) tf[1] = 0.;
    for (int nn = -1; nn <= 1; nn++) for (int m = -1; m <= 1; m++) for (int l = -1; l <= 1; l++) {
        long long x;
        bool inside;
        if (!neighbour(l, m, nn, x, inside) || !inside) continue;
        const double w = 1./(abs(l) + abs(m) + abs(nn) + 1);
#pragma unroll
        for (int p = 0; p < 5; ++p) atomicAdd(Pbar_out.v[p] + x, w * tf[p]);
    }
}

// Ubar_upd = Ubar_out + J(P_out)^-T Pbar_out over the interior (zero elsewhere).  With floors (fflag
// set, Pinv the stage's inverted fluid primitives before the floors, [5][N]), a floored zone has
// P_out = Floors(P_inv) and U_out = U(P_out), so there
//   Ubar_upd = J(P_inv)^-T DFloors(P_inv)^T (Pbar_out + J(P_out)^T Ubar_out)
// (the floor Jacobian by one dual evaluation per input); zones the floors left alone keep the first
// form.
template <int NV>
__global__ void __launch_bounds__(128) k_adj_cell(Dims d, DevGeom g, Phys ph, khb_fields Pout, khb_fields Pbar_out,
                                                  khb_fields Ubar_out, double* Ubar_upd, const double* Pinv,
                                                  const int32_t* fflag, const int32_t* pflag, Box bx)
{
    int i, j, k;
    if (!box_cell(bx, blockIdx.x, i, j, k)) return;
    const long long c = ((long long)k*d.n2 + j)*d.n1 + i;
    if (pflag && pflag[c] > 0) return;    // a failed zone: k_adj_fixup
    double P[NV], J[NV][NV], y[NV], ubo[NV];
    bool any = false;
#pragma unroll
    for (int p = 0; p < NV; ++p) { y[p] = Pbar_out.v[p][c]; ubo[p] = Ubar_out.v[p][c]; any |= (y[p] != 0.) | (ubo[p] != 0.); }
    if (!any) return;                     // Ubar_upd stays zero (cleared before the launch)
    ZoneGeom G;
    load_zone_geom(g, j, i, G);
#pragma unroll
    for (int p = 0; p < NV; ++p) P[p] = Pout.v[p][c];
    if (fflag && fflag[c]) {
        // Pbar_out + J(P_out)^T Ubar_out
        ptou_jacobian<NV>(G, ph.gam, P, J);
        double t[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            double s = y[q];
#pragma unroll
            for (int p = 0; p < NV; ++p) s += J[p][q] * ubo[p];
            t[q] = s;
        }
        // the inverted state; B is not changed by the floors
        double Pi[NV];
#pragma unroll
        for (int p = 0; p < 5; ++p) Pi[p] = Pinv[p*d.N + c];
#pragma unroll
        for (int p = 5; p < NV; ++p) Pi[p] = P[p];
        const long long cg = (long long)j*g.n1 + i;
        const Prescription& fl = floors_at(ph, g, j, i);
        const double rfg = __ldg(g.floor_rho + cg), ufg = __ldg(g.floor_u + cg);
        // s = DFloors^T t: column q of DFloors from the tangent seeded on input q
        double s[NV];
        for (int q = 0; q < NV; ++q) {
            Dual<double> X[NV];
#pragma unroll
            for (int p = 0; p < NV; ++p) X[p] = Dual<double>(Pi[p], (p == q) ? 1. : 0.);
            floors_dual<NV>(G, fl, rfg, ufg, ph.gam, ph.frame, X);
            double acc = 0.;
#pragma unroll
            for (int p = 0; p < NV; ++p) acc += X[p].d * t[p];
            s[q] = acc;
        }
        ptou_jacobian<NV>(G, ph.gam, Pi, J);
        solve_transposed<NV>(J, s);
#pragma unroll
        for (int p = 0; p < NV; ++p) Ubar_upd[p*d.N + c] = s[p];
        return;
    }
    ptou_jacobian<NV>(G, ph.gam, P, J);
    solve_transposed<NV>(J, y);
#pragma unroll
    for (int p = 0; p < NV; ++p) Ubar_upd[p*d.N + c] = ubo[p] + y[p];
}

// Pbar += J(P)^T Ubar over the whole block (the adjoint of U = U(P) of an initial state)
template <int NV>
__global__ void __launch_bounds__(128) k_adj_ptou(Dims d, DevGeom g, Phys ph, khb_fields P, khb_fields Ubar,
                                                  khb_fields Pbar)
{
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= d.N) return;
    int k, j, i;
    zone_kji(d, c, k, j, i);
    ZoneGeom G;
    load_zone_geom(g, j, i, G);
    double Pz[NV], J[NV][NV];
#pragma unroll
    for (int p = 0; p < NV; ++p) Pz[p] = P.v[p][c];
    ptou_jacobian<NV>(G, ph.gam, Pz, J);
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double s = 0.;
#pragma unroll
        for (int p = 0; p < NV; ++p) s += J[p][q] * Ubar.v[p][c];
        Pbar.v[q][c] += s;
    }
}

// Ghost-zone adjoints: a zone outside the interior along a periodic direction is a copy of its
// image, so its adjoint is added to the image (first); a zone of a physical face's ghost layers is
// a function of its source zone (k_adj_bc, next); any other ghost zone is the caller's constant.  All
// ghost adjoints are zeroed afterwards.
template <int NV>
__global__ void k_adj_fold(Dims d, khb_fields A, int pmask)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= d.N) return;
    int k, j, i;
    zone_kji(d, t, k, j, i);
    // k_periodic copies every zone outside the interior along a periodic direction from its image,
    // wrapping the periodic directions only (the image may lie in another direction's ghost zones)
    const bool gi = (pmask & 1) && (i < d.is || i > d.ie), gj = (pmask & 2) && (j < d.js || j > d.je);
    const bool gk = (pmask & 4) && (k < d.ks || k > d.ke);
    if (!(gi || gj || gk)) return;
    const int ii = gi ? i + ((i < d.is) ? d.nx1 : -d.nx1) : i;
    const int jj = gj ? j + ((j < d.js) ? d.nx2 : -d.nx2) : j;
    const int kk = gk ? k + ((k < d.ks) ? d.nx3 : -d.nx3) : k;
    const long long s = ((long long)kk*d.n2 + jj)*d.n1 + ii;
    // a periodic ghost zone is never an image, so zeroing it here races with nothing; the physical
    // faces' adjoint then sees only what their own fills contributed
#pragma unroll
    for (int p = 0; p < NV; ++p) { atomicAdd(A.v[p] + s, A.v[p][t]); A.v[p][t] = 0.; }
}
template <int NV>
__global__ void k_adj_clear_ghosts(Dims d, khb_fields A)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= d.N) return;
    int k, j, i;
    zone_kji(d, t, k, j, i);
    const bool interior = i >= d.is && i <= d.ie && j >= d.js && j <= d.je && k >= d.ks && k <= d.ke;
    if (interior) return;
#pragma unroll
    for (int p = 0; p < NV; ++p) A.v[p][t] = 0.;
}

// Adjoint of one physical face's ghost fill k_bc: the ghost zone's fluid primitives are its
// source zone's, the normal velocity inverted on reflecting faces, and on X1 faces with inflow checks
// the velocity passed through inflow_fix (its Jacobian by three dual evaluations).  Pbar(source) +=
// J^T Pbar(ghost), then Pbar(ghost) = 0.  Same thread layout and index logic as k_bc.
template <int NV>
__global__ void k_adj_bc(Dims d, DevGeom g, Phys ph, khb_fields P, khb_fields Pbar, khb_fields Ubar, int face,
                         int lo_a, int cnt_a, int lo_k, int cnt_k)
{
    const int bdir = face / 2 + 1;
    const bool inner = (face % 2) == 0;
    const int ng = (bdir == 1) ? d.is : d.js;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)ng*cnt_a*cnt_k) return;
    const int gidx = (int)(t % ng);
    const long long r = t / ng;
    const int aidx = lo_a + (int)(r % cnt_a);
    const int k = lo_k + (int)(r / cnt_a);
    int i, j, ref;
    if (bdir == 1) { j = aidx; ref = inner ? d.is : d.ie; i = inner ? gidx : d.ie + 1 + gidx; }
    else { i = aidx; ref = inner ? d.js : d.je; j = inner ? gidx : d.je + 1 + gidx; }
    const int type = d.bc[face];
    const int offset = 2 * ref + (inner ? -1 : 1);
    int ii = i, jj = j;
    if (bdir == 1) ii = (type == KHB_BC_OUTFLOW) ? ref : offset - i;
    else           jj = (type == KHB_BC_OUTFLOW) ? ref : offset - j;
    const long long c = ((long long)k*d.n2 + j)*d.n1 + i;
    const long long s = ((long long)k*d.n2 + jj)*d.n1 + ii;
    if (NV > 5) {
        // k_bc's U_B copy (the normal component inverted on reflecting faces); the ghost B_P = U_B/gdet
        // of k_ghost_ptou was moved into Ubar by k_adj_ghost_b before these passes
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            const double ub = Ubar.v[5 + v][c];
            Ubar.v[5 + v][c] = 0.;
            const double fl = ((type == KHB_BC_REFLECTING) && (v == bdir - 1)) ? -1.0 : 1.0;
            if (ub != 0.) atomicAdd(Ubar.v[5 + v] + s, fl * ub);
        }
    }
    double pb[5];
    bool any = false;
#pragma unroll
    for (int p = 0; p < 5; ++p) { pb[p] = Pbar.v[p][c]; Pbar.v[p][c] = 0.; any |= pb[p] != 0.; }
    if (!any) return;
    double sgn[5];
#pragma unroll
    for (int p = 0; p < 5; ++p) sgn[p] = ((type == KHB_BC_REFLECTING) && (p == 1 + bdir)) ? -1.0 : 1.0;
    const bool inflow = (face == 0 && ph.check_inflow_in) || (face == 1 && ph.check_inflow_out);
    if (inflow) {
        typedef Dual<double> DD;
        ZoneGeom G;
        load_zone_geom(g, j, i, G);
        DD gcov[4][4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) gcov[a][b] = DD(G.gcov[a][b]);
        double u0[3];
#pragma unroll
        for (int v = 0; v < 3; ++v) u0[v] = sgn[2 + v] * P.v[2 + v][s];
        double ub[3] = {0., 0., 0.};
        for (int q = 0; q < 3; ++q) {
            DD u[3];
#pragma unroll
            for (int v = 0; v < 3; ++v) u[v] = DD(u0[v], (v == q) ? 1. : 0.);
            inflow_fix<DD>(G, gcov, u, inner);
            double acc = 0.;
#pragma unroll
            for (int v = 0; v < 3; ++v) acc += u[v].d * pb[2 + v];
            ub[q] = acc;
        }
#pragma unroll
        for (int v = 0; v < 3; ++v) pb[2 + v] = ub[v];
    }
#pragma unroll
    for (int p = 0; p < 5; ++p) atomicAdd(Pbar.v[p] + s, sgn[p] * pb[p]);
}

// The adjoint of k_ghost_ptou's B_P = U_B / gdet on the X1/X2 ghost zones of the interior k range of
// the physical directions (Ubar_B += Pbar_B / gdet, Pbar_B = 0); same enumeration as k_ghost_ptou
__global__ void k_adj_ghost_b(Dims d, DevGeom g, khb_fields Pbar, khb_fields Ubar)
{
    const unsigned per = plane_ghost_count(d);
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned kk = t / per;
    if (kk >= (unsigned)(d.ke - d.ks + 1)) return;
    int j, i;
    if (!plane_ghost(d, t - kk * per, j, i)) return;
    const long long c = ((long long)(d.ks + (int)kk)*d.n2 + j)*d.n1 + i;
    const double gdet = __ldg(g.gdet[3] + (long long)j*g.G1 + i);
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        const double pb = Pbar.v[5 + v][c];
        Pbar.v[5 + v][c] = 0.;
        Ubar.v[5 + v][c] += pb / gdet;
    }
}

// The adjoint of B_FluxCT's polar flux fix (k_fix_flux_x2 with fix_polar_flux, b_flux_ct.cpp:372-418):
// the X1 and X3 B2 fluxes of the ghost row beside the polar face are minus those of the first
// interior row, so their adjoints move there with a sign and are cleared.  One thread per (k, i).
__global__ void k_adj_fix_polar(Dims d, double* F1b, double* F3b, int inner)
{
    const int ni = d.ie - d.is + 3;
    const int nk = (d.ndim > 2) ? d.ke - d.ks + 3 : 1;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ni*nk) return;
    const int i = d.is - 1 + t % ni;
    const int k = (d.ndim > 2) ? d.ks - 1 + t / ni : d.ks;
    const int j = inner ? d.js : d.je + 1;
    const long long c = ((long long)k*d.n2 + j)*d.n1 + i, N = d.N;
    const long long gh = inner ? c - d.sj : c, in = inner ? c : c - d.sj;     // written row, read row
    F1b[6*N + in] -= F1b[6*N + gh];
    F1b[6*N + gh] = 0.;
    if (d.ndim > 2) {
        F3b[6*N + in] -= F3b[6*N + gh];
        F3b[6*N + gh] = 0.;
    }
}

// Deterministic sum_f w[f] * F[f] (times scale) added to *out: fixed-size grid of partial sums,
// then one block adds them in order.
constexpr int kDotBlocks = 592, kDotThreads = 256;
template <typename FT>
__global__ void __launch_bounds__(kDotThreads) k_flux_dot_partial(long long N, const FT* F, const double* w,
                                                                  double* partial)
{
    double s = 0.;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x) {
        const double ww = w[t];
        if (ww != 0.) s += ww * (double)F[t];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ double ws[kDotThreads / 32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.;
        for (int i = 0; i < kDotThreads / 32; ++i) t += ws[i];
        partial[blockIdx.x] = t;
    }
}
// one warp: lane l adds partials l, l+32, ... in order, then a fixed butterfly (deterministic)
__global__ void k_flux_dot_final(const double* partial, int n, double scale, double* out)
{
    const int l = threadIdx.x;
    double t = 0.;
    for (int i = l; i < n; i += 32) t += partial[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (l == 0) *out += scale * t;
}

} // namespace khb

using namespace khb;

namespace {

#define KHB_ACUDA(call)                                                                                        \
    do {                                                                                                       \
        cudaError_t e_ = (call);                                                                               \
        if (e_ != cudaSuccess) return set_error(KHB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

int adj_supported(const khb_ctx* ctx, const char* who)
{
    const Dims& d = ctx->d;
    const std::string w(who);
    if (ctx->ph.recon_floors) return set_error(KHB_ERR_UNSUPPORTED, w + ": reconstruction floors are not differentiated");
    if (ctx->ph.floors_on && ctx->ph.frame != KHB_FRAME_FLUID && ctx->ph.frame != KHB_FRAME_DRIFT)
        return set_error(KHB_ERR_UNSUPPORTED, w + ": floors are differentiated in the fluid and drift frames only");
    if (ctx->ph.floors_on && ctx->ph.inverter != KHB_INVERTER_ONEDW)
        return set_error(KHB_ERR_UNSUPPORTED, w + ": floors are differentiated with the 1D_W inverter only");
    if (ctx->ph.fofc) return set_error(KHB_ERR_UNSUPPORTED, w + ": first-order flux correction is not differentiated");
    if (ctx->ph.ct_scheme) return set_error(KHB_ERR_UNSUPPORTED, w + ": B_CT is not differentiated");
    if (ctx->ph.riemann != 0) return set_error(KHB_ERR_UNSUPPORTED, w + ": LLF fluxes only");
    if (ctx->cfg.recon != KHB_RECON_LINEAR_MC && ctx->cfg.recon != KHB_RECON_DONOR_CELL)
        return set_error(KHB_ERR_UNSUPPORTED, w + ": linear MC or donor-cell reconstruction only");
    for (int f = 0; f < 2 * d.ndim; ++f) {
        if (!phys_face(d.bc[f])) continue;
        // outflow / reflecting X1 and X2 faces (their ghost fills, inflow checks and flux fixes,
        // flux-CT's polar B-flux fix included, are differentiated); transmitting faces are not
        if (f >= 4 || (d.bc[f] != KHB_BC_OUTFLOW && d.bc[f] != KHB_BC_REFLECTING))
            return set_error(KHB_ERR_UNSUPPORTED, w + ": physical faces must be outflow or reflecting X1/X2 faces");
    }
    return KHB_OK;
}

int pmask_of(const Dims& d)
{
    int m = 0;
    if (d.bc[0] == KHB_BC_PERIODIC) m |= 1;
    if (d.ndim >= 2 && d.bc[2] == KHB_BC_PERIODIC) m |= 2;
    if (d.ndim >= 3 && d.bc[4] == KHB_BC_PERIODIC) m |= 4;
    return m;
}

khb_fields slice_fields(double* base, long long N, int nv)
{
    khb_fields f;
    std::memset(&f, 0, sizeof(f));
    for (int p = 0; p < nv; ++p) f.v[p] = base + (size_t)p * N;
    return f;
}

// The adjoint of launch_boundaries' ghost fills in reverse order (inner x1 again with fix_corner,
// x2 faces, x1 faces), for a stage input P
template <int NV>
void bc_adjoint(const khb_ctx* ctx, const khb_fields& P, const khb_fields& Pbar, const khb_fields& Ubar,
                cudaStream_t st)
{
    const Dims& d = ctx->d;
    const int cnt_k = d.ke - d.ks + 1;
    if (NV > 5) {
        const long long tot = (long long)plane_ghost_count(d) * cnt_k;
        if (tot) k_adj_ghost_b<<<blocks_for(tot, 128), 128, 0, st>>>(d, ctx->g, Pbar, Ubar);
    }
    auto one = [&](int face, int lo_a, int cnt_a) {
        const int ng = (face < 2) ? d.is : d.js;
        k_adj_bc<NV><<<blocks_for((long long)ng * cnt_a * cnt_k, 128), 128, 0, st>>>(d, ctx->g, ctx->ph, P, Pbar, Ubar,
                                                                                     face, lo_a, cnt_a, d.ks, cnt_k);
    };
    if (d.ndim >= 2 && ctx->cfg.fix_corner_inner && phys_face(d.bc[0]) && phys_face(d.bc[3])) one(0, 0, d.n2);
    if (d.ndim >= 2)
        for (int face = 3; face >= 2; --face)
            if (phys_face(d.bc[face])) one(face, 0, d.n1);
    for (int face = 1; face >= 0; --face)
        if (phys_face(d.bc[face])) one(face, d.js, d.je - d.js + 1);
}

template <int NV>
void fold(const khb_ctx* ctx, const khb_fields& A, cudaStream_t st)
{
    const Dims& d = ctx->d;
    k_adj_fold<NV><<<blocks_for(d.N, 256), 256, 0, st>>>(d, A, pmask_of(d));
    k_adj_clear_ghosts<NV><<<blocks_for(d.N, 256), 256, 0, st>>>(d, A);
}

// The stage input's ghost adjoints: periodic images first, then (physical faces) the ghost fills'
// transposes, which move Pbar (and for MHD the ghost B into Ubar) to the source zones, then cleared
template <int NV>
void fold_input(const khb_ctx* ctx, const khb_fields& P, const khb_fields& Pbar, const khb_fields& Ubar,
                cudaStream_t st)
{
    const Dims& d = ctx->d;
    k_adj_fold<NV><<<blocks_for(d.N, 256), 256, 0, st>>>(d, Pbar, pmask_of(d));
    k_adj_fold<NV><<<blocks_for(d.N, 256), 256, 0, st>>>(d, Ubar, pmask_of(d));
    bool physical = false;
    for (int f = 0; f < 2 * d.ndim; ++f) physical |= phys_face(d.bc[f]);
    if (physical) bc_adjoint<NV>(ctx, P, Pbar, Ubar, st);
    k_adj_clear_ghosts<NV><<<blocks_for(d.N, 256), 256, 0, st>>>(d, Pbar);
    k_adj_clear_ghosts<NV><<<blocks_for(d.N, 256), 256, 0, st>>>(d, Ubar);
}

// what k_adj_flux needs to form the hydro flux adjoints: Ubar_upd, bdt/vol, the objective's seed
struct FluxAdj {
    const double* Uupd;
    double w;
    const double* seed;
    double seed_scale;
};

template <int DIR, int NV, typename R>
void adj_flux_dir(const khb_ctx* ctx, const khb_fields& P, const double* Fb, const FluxAdj& fa, const khb_fields& Pbar,
                  cudaStream_t st)
{
    const Dims& d = ctx->d;
    int lo[3], cnt[3];
    const int s[3] = {d.is, d.js, d.ks}, e[3] = {d.ie, d.je, d.ke};
    for (int a = 0; a < 3; ++a) {
        const bool active = (a + 1) <= d.ndim;
        int hi;
        if (a + 1 == DIR) { lo[a] = s[a]; hi = e[a] + 1; }
        else if (active) { lo[a] = s[a] - 1; hi = e[a] + 1; }
        else { lo[a] = s[a]; hi = e[a]; }
        cnt[a] = hi - lo[a] + 1;
    }
    const Box bx = make_box(lo[0], lo[1], lo[2], cnt[0], cnt[1], cnt[2]);
    const double a = (DIR == 1) ? ctx->ph.dx2 * ctx->ph.dx3 : ((DIR == 2) ? ctx->ph.dx1 * ctx->ph.dx3 : ctx->ph.dx1 * ctx->ph.dx2);
    const bool donor = ctx->cfg.recon == KHB_RECON_DONOR_CELL;
    if (sizeof(R) == 4) {
        if (donor) launch_adj_flux_f32<DIR, NV, RECON_DONOR>(st, d, ctx->g, ctx->ph, P, Fb, fa.Uupd, fa.w, a, fa.seed,
                                                             fa.seed_scale, Pbar, bx);
        else launch_adj_flux_f32<DIR, NV, RECON_MC>(st, d, ctx->g, ctx->ph, P, Fb, fa.Uupd, fa.w, a, fa.seed,
                                                    fa.seed_scale, Pbar, bx);
    } else if (donor) {
        k_adj_flux<DIR, NV, RECON_DONOR, double><<<box_blocks(bx), 128, 0, st>>>(d, ctx->g, ctx->ph, P, Fb, fa.Uupd,
                                                                                 fa.w, a, fa.seed, fa.seed_scale, Pbar, bx);
    } else {
        k_adj_flux<DIR, NV, RECON_MC, double><<<box_blocks(bx), 128, 0, st>>>(d, ctx->g, ctx->ph, P, Fb, fa.Uupd,
                                                                              fa.w, a, fa.seed, fa.seed_scale, Pbar, bx);
    }
}

// Adjoint of one stage.  Pbar_out/Ubar_out are read by the first kernel; with clear_out they are
// zeroed right after, so that they can receive Ubar_0 (stage 2 passes the caller's arrays both ways).
// Launches: memset, cell, [clear], update, ndim flux (the X1 one adds the objective seed), 2-3 folds x 2.
template <int NV>
int adjoint_stage_nv(khb_ctx* ctx, int stage, double dt, const khb_fields& Ps, const khb_fields& Pout,
                     const khb_fields& Pbar_out, const khb_fields& Ubar_out, bool clear_out, const double* weight,
                     double wscale, const khb_fields& Pbar_s, const khb_fields& Ubar_s, const khb_fields& Ubar_0,
                     const double* pinv, const int32_t* fflag, const int32_t* pflag, cudaStream_t st)
{
    const Dims& d = ctx->d;
    const size_t N = (size_t)d.N;
    double* Fb[3] = {ctx->adj_buf, ctx->adj_buf + NV * N, ctx->adj_buf + 2 * NV * N};
    double* Uupd = ctx->adj_buf + 3 * NV * N;
    KHB_ACUDA(cudaMemsetAsync(ctx->adj_buf, 0, sizeof(double) * 4 * NV * N, st));
    const Box zb = make_box(d.is, d.js, d.ks, d.ie - d.is + 1, d.je - d.js + 1, d.ke - d.ks + 1);
    if (pflag) {
        k_adj_fixup<NV><<<box_blocks(zb), 128, 0, st>>>(d, ctx->g, ctx->ph, Pout, Pbar_out, Ubar_out, pflag, Uupd, zb);
        ctx->launches += 1;
    }
    k_adj_cell<NV><<<box_blocks(zb), 128, 0, st>>>(d, ctx->g, ctx->ph, Pout, Pbar_out, Ubar_out, Uupd, pinv, fflag,
                                                   pflag, zb);
    if (clear_out)
        for (int p = 0; p < NV; ++p) {
            KHB_ACUDA(cudaMemsetAsync(Pbar_out.v[p], 0, sizeof(double) * N, st));
            KHB_ACUDA(cudaMemsetAsync(Ubar_out.v[p], 0, sizeof(double) * N, st));
        }
    const int s = stage - 1;
    const double bdt = kRkBeta[s] * dt;
    k_adj_update<NV><<<box_blocks(zb), 128, 0, st>>>(d, ctx->g, ctx->ph, Uupd, Ps, kRkGam0[s], kRkGam1[s],
                                                     bdt, Fb[0], Fb[1], Fb[2], Pbar_s, Ubar_s, Ubar_0, zb);
    if (NV > 5 && d.ndim >= 2 && ctx->ph.fix_polar_flux)
        for (int face = 2; face <= 3; ++face) {
            if (!phys_face(d.bc[face])) continue;
            const int ni = d.ie - d.is + 3, nk = (d.ndim > 2) ? d.ke - d.ks + 3 : 1;
            k_adj_fix_polar<<<blocks_for((long long)ni * nk, 128), 128, 0, st>>>(d, Fb[0], Fb[2], face == 2);
        }
    const FluxAdj fa{Uupd, bdt / (ctx->ph.dx1 * ctx->ph.dx2 * ctx->ph.dx3), weight, wscale};
    for (int dir = 1; dir <= d.ndim; ++dir) {
        if (ctx->fp32) {
            if (dir == 1) adj_flux_dir<1, NV, float>(ctx, Ps, Fb[0], fa, Pbar_s, st);
            else if (dir == 2) adj_flux_dir<2, NV, float>(ctx, Ps, Fb[1], fa, Pbar_s, st);
            else adj_flux_dir<3, NV, float>(ctx, Ps, Fb[2], fa, Pbar_s, st);
        } else {
            if (dir == 1) adj_flux_dir<1, NV, double>(ctx, Ps, Fb[0], fa, Pbar_s, st);
            else if (dir == 2) adj_flux_dir<2, NV, double>(ctx, Ps, Fb[1], fa, Pbar_s, st);
            else adj_flux_dir<3, NV, double>(ctx, Ps, Fb[2], fa, Pbar_s, st);
        }
    }
    fold_input<NV>(ctx, Ps, Pbar_s, Ubar_s, st);
    if (Ubar_0.v[0] != Ubar_s.v[0]) fold<NV>(ctx, Ubar_0, st);
    KHB_ACUDA(cudaGetLastError());
    ctx->launches += 3 + d.ndim + (clear_out ? 2 * NV : 0) + 2 * (Ubar_0.v[0] != Ubar_s.v[0] ? 3 : 2);
    return KHB_OK;
}

// pinv/fflag/pflag: per stage, the inverted fluid primitives before the floors, the floor flags and
// the inversion flags of the recomputed stages (NULL where the stage was not recomputed)
template <int NV>
int adjoint_step_nv(khb_ctx* ctx, double dt, const khb_fields& Pn, const khb_fields& Pstar,
                    const khb_fields& Pnp1, const khb_fields& Pbar, const khb_fields& Ubar, const double* weight,
                    double wscale, const double* const pinv[2], const int32_t* const fflag[2],
                    const int32_t* const pflag[2], cudaStream_t st)
{
    const size_t N = (size_t)ctx->d.N;
    const khb_fields Pbar_star = slice_fields(ctx->adj_buf + 4 * NV * N, ctx->d.N, NV);
    const khb_fields Ubar_star = slice_fields(ctx->adj_buf + 5 * NV * N, ctx->d.N, NV);
    KHB_ACUDA(cudaMemsetAsync(ctx->adj_buf + 4 * NV * N, 0, sizeof(double) * 2 * NV * N, st));
    ctx->launches += 1;
    int rc;
    // stage 2: (P*, U*, U^n) -> (P^{n+1}, U^{n+1}); the caller's arrays turn into the adjoint of U^n
    if ((rc = adjoint_stage_nv<NV>(ctx, 2, dt, Pstar, Pnp1, Pbar, Ubar, true, weight, wscale, Pbar_star, Ubar_star,
                                   Ubar, pinv[1], fflag[1], pflag[1], st)))
        return rc;
    // stage 1: (P^n, U^n, U^n) -> (P*, U*)
    return adjoint_stage_nv<NV>(ctx, 1, dt, Pn, Pstar, Pbar_star, Ubar_star, false, weight, wscale, Pbar, Ubar, Ubar,
                                pinv[0], fflag[0], pflag[0], st);
}

} // namespace

extern "C" {

int khb_adjoint_step(khb_ctx* ctx, double dt, const khb_fields* P_n, const khb_fields* U_n,
                     const khb_fields* P_np1, const khb_fields* Pbar, const khb_fields* Ubar,
                     const double* rho_flux1_weight, double weight_scale, void* stream)
{
    KHB_RANGE("khb_adjoint_step");
    if (!ctx || !ctx->geom_set) return set_error(KHB_ERR_STATE, "khb_adjoint_step: context without geometry");
    if (!P_n || !U_n || !P_np1 || !Pbar || !Ubar) return set_error(KHB_ERR_ARG, "khb_adjoint_step: NULL argument");
    for (int p = 0; p < ctx->nv; ++p)
        if (!P_n->v[p] || !U_n->v[p] || !P_np1->v[p] || !Pbar->v[p] || !Ubar->v[p])
            return set_error(KHB_ERR_ARG, "khb_adjoint_step: NULL variable pointer");
    if (!(dt > 0.)) return set_error(KHB_ERR_ARG, "khb_adjoint_step: dt must be positive");
    int rc;
    if ((rc = adj_supported(ctx, "khb_adjoint_step"))) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const Dims& d = ctx->d;
    if (!ctx->adj_buf) {
        KHB_ACUDA(cudaMalloc((void**)&ctx->adj_buf, sizeof(double) * 6 * ctx->nv * (size_t)d.N));
        KHB_ACUDA(cudaMalloc((void**)&ctx->adj_flags, sizeof(int32_t) * 2 * (size_t)d.N));
        KHB_ACUDA(cudaMemset(ctx->adj_flags, 0, sizeof(int32_t) * 2 * (size_t)d.N));
        KHB_ACUDA(cudaDeviceSynchronize());
    }
    const bool floors = ctx->ph.floors_on;
    if (!ctx->adj_s2) {
        KHB_ACUDA(cudaMalloc((void**)&ctx->adj_s2, sizeof(double) * 2 * ctx->nv * (size_t)d.N));
        KHB_ACUDA(cudaMalloc((void**)&ctx->adj_flags2, sizeof(int32_t) * 2 * (size_t)d.N));
        KHB_ACUDA(cudaMemset(ctx->adj_s2, 0, sizeof(double) * 2 * ctx->nv * (size_t)d.N));
        KHB_ACUDA(cudaMemset(ctx->adj_flags2, 0, sizeof(int32_t) * 2 * (size_t)d.N));
        KHB_ACUDA(cudaDeviceSynchronize());
    }
    if (floors && !ctx->adj_pf) {
        KHB_ACUDA(cudaMalloc((void**)&ctx->adj_pf, sizeof(double) * 10 * (size_t)d.N));
        KHB_ACUDA(cudaMemset(ctx->adj_pf, 0, sizeof(double) * 10 * (size_t)d.N));
        KHB_ACUDA(cudaDeviceSynchronize());
    }
    // recompute both stages: the intermediate state (P*, U*) into the context's stage scratch, and
    // each stage's inversion flags (failed zones take the fixup's adjoint) and, with floors, its
    // inverted primitives before the floors and its floor flags
    struct PrefloorScope {
        khb_ctx* c;
        ~PrefloorScope() { c->prefloor_dst = nullptr; }
    } scope{ctx};
    const khb_fields Pstar = slice_fields(ctx->stageP, d.N, ctx->nv), Ustar = slice_fields(ctx->stageU, d.N, ctx->nv);
    ctx->prefloor_dst = floors ? ctx->adj_pf : nullptr;
    if ((rc = khb_stage(ctx, 1, dt, P_n, U_n, U_n, &Pstar, &Ustar, ctx->adj_flags, ctx->adj_flags + d.N, stream)))
        return rc;
    const khb_fields P2 = slice_fields(ctx->adj_s2, d.N, ctx->nv);
    const khb_fields U2 = slice_fields(ctx->adj_s2 + (size_t)ctx->nv * d.N, d.N, ctx->nv);
    ctx->prefloor_dst = floors ? ctx->adj_pf + 5 * (size_t)d.N : nullptr;
    if ((rc = khb_stage(ctx, 2, dt, &Pstar, &Ustar, U_n, &P2, &U2, ctx->adj_flags2, ctx->adj_flags2 + d.N, stream)))
        return rc;
    ctx->prefloor_dst = nullptr;
    const double* pinv[2] = {nullptr, nullptr};
    const int32_t* ffl[2] = {nullptr, nullptr};
    const int32_t* pfl[2] = {ctx->adj_flags, ctx->adj_flags2};
    if (floors) {
        pinv[0] = ctx->adj_pf; pinv[1] = ctx->adj_pf + 5 * (size_t)d.N;
        ffl[0] = ctx->adj_flags + d.N; ffl[1] = ctx->adj_flags2 + d.N;
    }
    if (ctx->nv == 8)
        return adjoint_step_nv<8>(ctx, dt, *P_n, Pstar, *P_np1, *Pbar, *Ubar, rho_flux1_weight, weight_scale, pinv, ffl,
                                  pfl, st);
    return adjoint_step_nv<5>(ctx, dt, *P_n, Pstar, *P_np1, *Pbar, *Ubar, rho_flux1_weight, weight_scale, pinv, ffl,
                              pfl, st);
}

int khb_flux_dot(khb_ctx* ctx, int dir, int var, const double* weight, double scale, double* out, void* stream)
{
    KHB_RANGE("khb_flux_dot");
    if (!ctx || !weight || !out) return set_error(KHB_ERR_ARG, "khb_flux_dot: NULL argument");
    if (dir < 1 || dir > ctx->d.ndim) return set_error(KHB_ERR_ARG, "khb_flux_dot: inactive direction");
    if (var < 0 || var >= ctx->nv) return set_error(KHB_ERR_ARG, "khb_flux_dot: bad variable");
    cudaStream_t st = (cudaStream_t)stream;
    const long long N = ctx->d.N;
    if (!ctx->adj_red) {
        KHB_ACUDA(cudaMalloc((void**)&ctx->adj_red, sizeof(double) * kDotBlocks));
        KHB_ACUDA(cudaDeviceSynchronize());
    }
    if (ctx->fp32)
        k_flux_dot_partial<float><<<kDotBlocks, kDotThreads, 0, st>>>(N, (const float*)ctx->F[dir - 1] + (size_t)var * N,
                                                                      weight, ctx->adj_red);
    else
        k_flux_dot_partial<double><<<kDotBlocks, kDotThreads, 0, st>>>(N, (const double*)ctx->F[dir - 1] + (size_t)var * N,
                                                                       weight, ctx->adj_red);
    k_flux_dot_final<<<1, 32, 0, st>>>(ctx->adj_red, kDotBlocks, scale, out);
    KHB_ACUDA(cudaGetLastError());
    ctx->launches += 2;
    return KHB_OK;
}

int khb_adjoint_ptou(khb_ctx* ctx, const khb_fields* P, const khb_fields* Ubar, const khb_fields* Pbar, void* stream)
{
    KHB_RANGE("khb_adjoint_ptou");
    if (!ctx || !ctx->geom_set) return set_error(KHB_ERR_STATE, "khb_adjoint_ptou: context without geometry");
    if (!P || !Ubar || !Pbar) return set_error(KHB_ERR_ARG, "khb_adjoint_ptou: NULL argument");
    for (int p = 0; p < ctx->nv; ++p)
        if (!P->v[p] || !Ubar->v[p] || !Pbar->v[p]) return set_error(KHB_ERR_ARG, "khb_adjoint_ptou: NULL variable pointer");
    cudaStream_t st = (cudaStream_t)stream;
    const Dims& d = ctx->d;
    if (ctx->nv == 8) k_adj_ptou<8><<<blocks_for(d.N, 128), 128, 0, st>>>(d, ctx->g, ctx->ph, *P, *Ubar, *Pbar);
    else k_adj_ptou<5><<<blocks_for(d.N, 128), 128, 0, st>>>(d, ctx->g, ctx->ph, *P, *Ubar, *Pbar);
    KHB_ACUDA(cudaGetLastError());
    ctx->launches += 1;
    return KHB_OK;
}

} // extern "C"

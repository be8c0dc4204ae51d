// khb_emhd.cu -- extended GRMHD (EMHD) and the per-zone implicit Newton solve on sm_100a.
//
// Kernels (one thread per zone):
//   k_emhd_ptou        Flux::p_to_u with the EMHD stress tensor and the q, dP conserved variables
//   k_emhd_temps       u_mu and Theta over the interior plus a one-zone halo (EMHD::AddSource temporaries)
//   k_emhd_sources     explicit conduction/viscosity sources, gradients by MC slopes (EMHD::AddSource)
//   k_implicit_iter    one Newton iteration of Implicit::Step: residual, Jacobian (forward differences
//                      as the reference, or the exact tangent), QR with column pivoting (or the LU
//                      path), backtracking, line search, update, residual norm and the block maximum
//   k_implicit_jacobian  residual and Jacobian only (the split "implicit_jacobian" kernel's output)
//   k_fix_solve_avg / k_fix_solve_apply   Implicit::FixSolve neighbour averaging and P->U
//   k_emhd_floors / k_emhd_limits   the floors and the EMHD stability limits of an ImEx stage
//
// The Newton state of a zone stays in registers for a whole iteration; the Jacobian (at most 7x7)
// is never written to memory.  Successive iterations are separate launches that read the previous
// iteration's maximum residual norm from device memory and return at once when the reference's
// loop would have stopped, so the whole solve is launched without a host round trip.
//
// Built with -fmad=false: with the forward-difference Jacobian the results agree bit for bit with
// the oracle's restatement of the reference (the torus closure, which calls exp, excepted).
#include "khb_kernels.cuh"

namespace khb {

static constexpr double SMALL = 1e-20;          // decs.hpp:82

enum { CL_CONSTANT = 0, CL_SOUNDSPEED = 1, CL_KAPPA_ETA = 2, CL_TORUS = 3 };
enum { SOLVE_CONVERGED = 0, SOLVE_FAIL = 1, SOLVE_BEYOND_TOL = 2, SOLVE_BACKTRACK = 3 };

// ------------------------------------------------------------------------------ closures
// EMHD::set_parameters, scalar form (emhd.hpp:179-261); r is the zone-centre radius (torus closure)
__device__ __forceinline__ void set_parameters(const EmhdArgs& E, double gam, double rho, double u, double qtilde,
                                               double dPtilde, double bsq, double r,
                                               double& tau, double& chi_e, double& nu_e)
{
    if (E.closure == CL_CONSTANT) {
        tau = E.tau;
        chi_e = E.conduction_alpha;
        nu_e = E.viscosity_alpha;
    } else if (E.closure == CL_SOUNDSPEED) {
        const double cs2 = (gam * (gam - 1.) * u) / (rho + (gam * u));
        tau = E.tau;
        chi_e = E.conduction_alpha * cs2 * tau;
        nu_e = E.viscosity_alpha * cs2 * tau;
    } else if (E.closure == CL_KAPPA_ETA) {
        tau = E.tau;
        chi_e = E.kappa / kmax(rho, SMALL);
        nu_e = E.eta / kmax(rho, SMALL);
    } else {
        const double tau_dyn = sqrt(r*r*r);
        tau = tau_dyn;
        const double pg = (gam - 1.) * u;
        const double Theta = pg / rho;
        const double cs2 = kmax(SMALL, gam * pg / (rho + (gam * u)));
        const double lambda = 0.01;
        {
            const double q = E.higher_order_terms ? qtilde * sqrt(rho * E.conduction_alpha * cs2 * Theta * Theta) : qtilde;
            const double q_max = E.conduction_alpha * rho * cs2 * sqrt(cs2);
            const double q_ratio = fabs(q) / q_max;
            const double inv_exp_g = exp(-(q_ratio - 1.) / lambda);
            const double f_fmin = inv_exp_g / (inv_exp_g + 1.) + 1.e-5;
            tau = kmin(tau, f_fmin * tau_dyn);
        }
        {
            const double dP = E.higher_order_terms ? dPtilde * sqrt(rho * E.viscosity_alpha * cs2 * Theta) : dPtilde;
            const double dP_comp_ratio = kmax(pg - 2./3. * dP, SMALL) / kmax(pg + 1./3. * dP, SMALL);
            const double dP_max = (dP > 0.) ? kmin(0.5 * bsq * dP_comp_ratio, 1.49 * pg / 1.07)
                                            : kmax(-bsq, -2.99 * pg / 1.07);
            const double dP_ratio = fabs(dP) / (fabs(dP_max) + SMALL);
            const double inv_exp_g = exp((1. - dP_ratio) / lambda);
            const double f_fmin = inv_exp_g / (inv_exp_g + 1.) + 1.e-5;
            tau = kmin(tau, f_fmin * tau_dyn);
        }
        const double max_alpha = (1 - cs2) / (2 * cs2 + 1.e-12);
        chi_e = kmin(max_alpha, E.conduction_alpha) * cs2 * tau;
        nu_e = kmin(max_alpha, E.viscosity_alpha) * cs2 * tau;
    }
}

// EMHD::convert_prims_to_q_dP (emhd.hpp:313-332)
__device__ __forceinline__ void convert_q_dP(const EmhdArgs& E, double qt, double dPt, double rho, double Theta,
                                             double cs2, double& q, double& dP)
{
    q = qt;
    if (E.higher_order_terms) {
        if (E.closure == CL_KAPPA_ETA) q *= sqrt(E.kappa * Theta * Theta / E.tau);
        else                           q *= sqrt(rho * E.conduction_alpha * cs2 * Theta * Theta);
    }
    dP = dPt;
    if (E.higher_order_terms) {
        if (E.closure == CL_KAPPA_ETA) dP *= sqrt(E.eta * Theta / E.tau);
        else                           dP *= sqrt(rho * E.viscosity_alpha * cs2 * Theta);
    }
}

// Row T^dir_mu of the EMHD stress tensor (emhd.hpp:296-309) from the full q and dP
__device__ __forceinline__ void emhd_tensor(double rho, double u, double pgas, double q, double dP,
                                            const FourVec<double>& D, int dir, double T[4])
{
    const double bsq = kmax(dot4(D.bcon, D.bcov), SMALL);
    const double b_mag = sqrt(bsq);
    const double eta = pgas + rho + u + bsq;
    const double ptot = pgas + 0.5 * bsq;
#pragma unroll
    for (int mu = 0; mu < 4; ++mu)
        T[mu] = eta * D.ucon[dir] * D.ucov[mu] + ptot * (double)(dir == mu) - D.bcon[dir] * D.bcov[mu]
              + (q / b_mag) * ((D.ucon[dir] * D.bcov[mu]) + (D.bcon[dir] * D.ucov[mu]))
              - dP * ((D.bcon[dir] * D.bcov[mu] / bsq) - (1./3.) * ((double)(dir == mu) + D.ucon[dir] * D.ucov[mu]));
}

// Zone-centre geometry for the EMHD kernels
struct CenterGeom {
    double gcov[4][4];
    double gcon0[4];          // gcon[0][mu]
    double gdet;
};
__device__ __forceinline__ void load_center(const DevGeom& g, int j, int i, CenterGeom& G)
{
    const long long gi = (long long)j*g.G1 + i;
#pragma unroll
    for (int m = 0; m < 16; ++m) G.gcov[m/4][m%4] = __ldg(g.gcov[3] + m*g.gs + gi);
#pragma unroll
    for (int m = 0; m < 4; ++m) G.gcon0[m] = __ldg(g.gcon[3] + m*g.gs + gi);
    G.gdet = __ldg(g.gdet[3] + gi);
}

// Flux::prim_to_flux (dir = 0) for the 10-slot state: conserved rho u^t, T^t_t + rho u^t, T^t_i, B^i gdet,
// q~ u^t gdet, dP~ u^t gdet (flux_functions.hpp:80-107, 180-232).  P: rho u u1 u2 u3 B1 B2 B3 q dP.
__device__ __forceinline__ void emhd_p_to_u(const EmhdArgs& E, double gam, const CenterGeom& G, const double* P,
                                            double* U)
{
    FourVec<double> D;
    calc_4vecs<double, true>(G.gcov, G.gcon0[0], G.gcon0, P, D);
    const double gdet = G.gdet;
    U[0] = P[0] * D.ucon[0] * gdet;
    double T[4];
    if ((E.conduction || E.viscosity) && E.feedback) {
        const double qt = E.conduction ? P[8] : 0., dPt = E.viscosity ? P[9] : 0.;
        const double Theta = (gam - 1) * P[1] / P[0];
        const double cs2 = gam * (gam - 1) * P[1] / (P[0] + gam * P[1]);
        double q, dP;
        convert_q_dP(E, qt, dPt, P[0], Theta, cs2, q, dP);
        emhd_tensor(P[0], P[1], (gam - 1) * P[1], q, dP, D, 0, T);
    } else {
        calc_tensor<double, true>(P[0], P[1], (gam - 1) * P[1], D, 0, T);
    }
    U[1] = T[0] * gdet + U[0];
    U[2] = T[1] * gdet;
    U[3] = T[2] * gdet;
    U[4] = T[3] * gdet;
#pragma unroll
    for (int v = 0; v < 3; ++v) U[5 + v] = P[5 + v] * gdet;
    if (E.conduction) U[8] = P[8] * D.ucon[0] * gdet;
    if (E.viscosity) U[9] = P[9] * D.ucon[0] * gdet;
}

// Flux::prim_to_flux for the 10-slot state at any location (dir = 0: conserved variables), with the
// EMHD stress tensor when q or dP feed back (flux_functions.hpp:80-107, 180-232).  Inactive EMHD
// slots get 0.
__device__ __forceinline__ void emhd_prim_to_flux(const EmhdArgs& E, double gam, double gdet, const double* P,
                                                  const FourVec<double>& D, int dir, double* flux)
{
    flux[0] = P[0] * D.ucon[dir] * gdet;
    double T[4];
    if ((E.conduction || E.viscosity) && E.feedback) {
        const double qt = E.conduction ? P[8] : 0., dPt = E.viscosity ? P[9] : 0.;
        const double Theta = (gam - 1) * P[1] / P[0];
        const double cs2 = gam * (gam - 1) * P[1] / (P[0] + gam * P[1]);
        double q, dP;
        convert_q_dP(E, qt, dPt, P[0], Theta, cs2, q, dP);
        emhd_tensor(P[0], P[1], (gam - 1) * P[1], q, dP, D, dir, T);
    } else {
        calc_tensor<double, true>(P[0], P[1], (gam - 1) * P[1], D, dir, T);
    }
    flux[1] = T[0] * gdet + flux[0];
    flux[2] = T[1] * gdet;
    flux[3] = T[2] * gdet;
    flux[4] = T[3] * gdet;
    if (dir == 0) {
#pragma unroll
        for (int v = 0; v < 3; ++v) flux[5 + v] = P[5 + v] * gdet;
    } else {
#pragma unroll
        for (int v = 0; v < 3; ++v) flux[5 + v] = (D.bcon[v+1] * D.ucon[dir] - D.bcon[dir] * D.ucon[v+1]) * gdet;
    }
    flux[8] = E.conduction ? P[8] * D.ucon[dir] * gdet : 0.;
    flux[9] = E.viscosity ? P[9] * D.ucon[dir] * gdet : 0.;
}

// vchar with the EMHD-augmented sound speed (flux_functions.hpp:380-403); the closure parameters the
// reference computes there are unused, so they are not formed
__device__ __forceinline__ void emhd_vchar(const EmhdArgs& E, double gam, const double* P, const FourVec<double>& D,
                                           double gcon00, double gcon0d, double gcondd, int dir,
                                           double& cmax, double& cmin)
{
    const double ef  = P[0] + gam * P[1];
    const double cs2 = gam * (gam - 1) * P[1] / ef;
    const double bsq = dot4(D.bcon, D.bcov);
    const double va2 = bsq / (bsq + ef);
    const double ccond2 = E.conduction ? (gam - 1.) * E.conduction_alpha * cs2 : 0.0;
    const double cvis2 = E.viscosity ? (4./3.) / (P[0] + (gam * P[1])) * P[0] * E.viscosity_alpha * cs2 : 0.0;
    const double cs2_emhd = 0.5*(cs2 + ccond2 + sqrt(cs2*cs2 + ccond2*ccond2)) + cvis2;
    const double cms2 = cs2_emhd + va2 - cs2_emhd*va2;
    vchar_speeds<double>(cms2, D, gcon00, gcon0d, gcondd, dir, cmax, cmin);
}

// ------------------------------------------------------------------------------ residual
// Constants of one zone's residual (everything that does not depend on the trial state)
template <int NF>
struct ResidZone {
    CenterGeom G;
    double B[3];                    // B^i primitives (explicit, fixed during the solve)
    double Ui[NF], S[NF];           // initial conserved and explicit dU/dt of the implicit variables
    double tau, chi_e, nu_e;
    double ucov_old[4], Theta_old;
    double cq0, cq[4], cd0, cd[4];  // time-derivative source coefficients (emhd_sources.hpp:103-122)
    double fac_q, fac_d, gq, gd;
    double dUi_q, dUi_d;            // implicit sources of the full-step initial state
    double norm_q, norm_d;          // final residual normalisation (implicit.hpp:190-198)
};

// The velocity-dependent part of the residual at a trial state: 4-vectors, Lorentz factor and
// (EMHD) the time derivative of u_mu and div u.  Columns of the forward-difference Jacobian that
// perturb rho, u, q~ or dP~ reuse the base state's: same inputs, same bits.
struct VelState {
    FourVec<double> D;
    double gamma;
    double dt_ucov[4];
    double div_ucon;
};

// Intermediates of the trial state kept for the exact Jacobian
struct ResidState {
    double Theta, cs2, fq, fd, q, dP;
    double bsq, bmag, eta;
    bool bsq_clamped, theta_clamped;
};

template <bool HQ, bool HD>
struct Imp {
    static constexpr int NF = 5 + HQ + HD;
    static constexpr int IQ = 5;
    static constexpr int ID = 5 + HQ;
    static constexpr bool EM = HQ || HD;
};

// Set up the residual constants (calc_residual's sub-step-state and full-step-state parts,
// implicit.hpp:161-198; emhd_sources.hpp:69-128).  Pf, Ps: 10-slot full-step and sub-step states.
template <bool HQ, bool HD>
__device__ __forceinline__ void setup_zone(const EmhdArgs& E, double gam, double r, const double* Pf, const double* Uf,
                                           const double* Ps, const double* Sz, const double* Psol,
                                           ResidZone<Imp<HQ, HD>::NF>& Z)
{
    using I = Imp<HQ, HD>;
#pragma unroll
    for (int v = 0; v < 3; ++v) Z.B[v] = Psol[5 + v];
#pragma unroll
    for (int p = 0; p < 5; ++p) { Z.Ui[p] = Uf[p]; Z.S[p] = Sz[p]; }
    if (HQ) { Z.Ui[I::IQ] = Uf[8]; Z.S[I::IQ] = Sz[8]; }
    if (HD) { Z.Ui[I::ID] = Uf[9]; Z.S[I::ID] = Sz[9]; }
    if (!I::EM) return;
    const CenterGeom& G = Z.G;
    // EMHD::set_parameters on the sub-step state (emhd.hpp:262-287)
    FourVec<double> Ds;
    calc_4vecs<double, true>(G.gcov, G.gcon0[0], G.gcon0, Ps, Ds);
    const double bsq = kmax(dot4(Ds.bcon, Ds.bcov), SMALL);
    const double qts = HQ ? Ps[8] : 0., dPts = HD ? Ps[9] : 0.;
    set_parameters(E, gam, Ps[0], Ps[1], qts, dPts, bsq, r, Z.tau, Z.chi_e, Z.nu_e);
    const double tau = Z.tau, chi_e = Z.chi_e, nu_e = Z.nu_e;
    // time_derivative_sources constants
    const double mag_b = sqrt(bsq);
    {
        double ucon[4];
        const double gamma = lorentz(G.gcov, Pf[2], Pf[3], Pf[4]);
        const double alpha = 1. / sqrt(-G.gcon0[0]);
        ucon[0] = gamma / alpha;
#pragma unroll
        for (int v = 0; v < 3; ++v) ucon[v+1] = Pf[2 + v] - gamma * alpha * G.gcon0[v+1];
        lower4(G.gcov, ucon, Z.ucov_old);
    }
    Z.Theta_old = kmax((gam-1) * Pf[1] / Pf[0], SMALL);
    const double rho = Ps[0];
    const double Theta = (gam-1) * Ps[1] / Ps[0];
    const double gdet = G.gdet;
    if (HQ) {
        Z.cq0 = -rho * chi_e * (Ds.bcon[0] / mag_b);
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) Z.cq[mu] = rho * chi_e * (Ds.bcon[mu] / mag_b) * Theta * Ds.ucon[0];
        Z.fac_q = (chi_e != 0) ? sqrt(tau / (chi_e * rho * Theta * Theta)) : 0.0;
        Z.gq = gdet * (qts / 2.);
        Z.dUi_q = -gdet * (Pf[8] / tau);
        Z.norm_q = (chi_e != 0) ? sqrt(rho * chi_e * tau * Theta * Theta) / tau : 1.;
    }
    if (HD) {
        Z.cd0 = -rho * nu_e;
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) Z.cd[mu] = 3. * rho * nu_e * (Ds.bcon[0] * Ds.bcon[mu] / bsq);
        Z.fac_d = (nu_e != 0) ? sqrt(tau / (nu_e * rho * Theta)) : 0.0;
        Z.gd = gdet * (dPts / 2.);
        Z.dUi_d = -gdet * (Pf[9] / tau);
        Z.norm_d = (nu_e != 0) ? sqrt(rho * nu_e * tau * Theta) / tau : 1.;
    }
}

// GRMHD::calc_4vecs of the trial state (grmhd_functions.hpp:225-246) and, for EMHD, the
// time-derivative pieces of EMHD::time_derivative_sources (emhd_sources.hpp:84-93)
template <bool HQ, bool HD>
__device__ __forceinline__ void velocity_part(double dt, const ResidZone<Imp<HQ, HD>::NF>& Z, const double* x,
                                              VelState& V)
{
    using I = Imp<HQ, HD>;
    const CenterGeom& G = Z.G;
    FourVec<double>& D = V.D;
    V.gamma = lorentz(G.gcov, x[2], x[3], x[4]);
    const double alpha = 1. / sqrt(-G.gcon0[0]);
    D.ucon[0] = V.gamma / alpha;
#pragma unroll
    for (int v = 0; v < 3; ++v) D.ucon[v+1] = x[2 + v] - V.gamma * alpha * G.gcon0[v+1];
    lower4(G.gcov, D.ucon, D.ucov);
    double b0 = 0.;
#pragma unroll
    for (int v = 0; v < 3; ++v) b0 += Z.B[v] * D.ucov[v+1];
    D.bcon[0] = b0;
#pragma unroll
    for (int v = 0; v < 3; ++v) D.bcon[v+1] = (Z.B[v] + b0 * D.ucon[v+1]) / D.ucon[0];
    lower4(G.gcov, D.bcon, D.bcov);
    if (I::EM) {
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) V.dt_ucov[mu] = (D.ucov[mu] - Z.ucov_old[mu]) / dt;
        double div_ucon = 0.;
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) div_ucon += G.gcon0[mu] * V.dt_ucov[mu];
        V.div_ucon = div_ucon;
    }
}

// Implicit::calc_residual (implicit.hpp:139-200) at the trial implicit variables x (rho, u, u1-u3[, q~][, dP~])
// given their velocity part V
template <bool HQ, bool HD>
__device__ __forceinline__ void residual_with(const EmhdArgs& E, double gam, double dt,
                                              const ResidZone<Imp<HQ, HD>::NF>& Z, const double* x,
                                              const VelState& V, double* res, ResidState& S)
{
    using I = Imp<HQ, HD>;
    const CenterGeom& G = Z.G;
    const FourVec<double>& D = V.D;
    const double gdet = G.gdet;
    double U[I::NF];
    U[0] = x[0] * D.ucon[0] * gdet;
    double T[4];
    const double pgas = (gam - 1) * x[1];
    if (I::EM && E.feedback) {
        const double qt = HQ ? x[I::IQ] : 0., dPt = HD ? x[I::ID] : 0.;
        S.Theta = (gam - 1) * x[1] / x[0];
        S.cs2 = gam * (gam - 1) * x[1] / (x[0] + gam * x[1]);
        convert_q_dP(E, qt, dPt, x[0], S.Theta, S.cs2, S.q, S.dP);
        const double dot = dot4(D.bcon, D.bcov);
        S.bsq_clamped = dot < SMALL;
        S.bsq = kmax(dot, SMALL);
        S.bmag = sqrt(S.bsq);
        S.eta = pgas + x[0] + x[1] + S.bsq;
        const double ptot = pgas + 0.5 * S.bsq;
#pragma unroll
        for (int mu = 0; mu < 4; ++mu)
            T[mu] = S.eta * D.ucon[0] * D.ucov[mu] + ptot * (double)(0 == mu) - D.bcon[0] * D.bcov[mu]
                  + (S.q / S.bmag) * ((D.ucon[0] * D.bcov[mu]) + (D.bcon[0] * D.ucov[mu]))
                  - S.dP * ((D.bcon[0] * D.bcov[mu] / S.bsq) - (1./3.) * ((double)(0 == mu) + D.ucon[0] * D.ucov[mu]));
    } else {
        S.bsq = dot4(D.bcon, D.bcov);
        S.bsq_clamped = false;
        S.eta = pgas + x[0] + x[1] + S.bsq;
        calc_tensor<double, true>(x[0], x[1], pgas, D, 0, T);
    }
    U[1] = T[0] * gdet + U[0];
    U[2] = T[1] * gdet;
    U[3] = T[2] * gdet;
    U[4] = T[3] * gdet;
    if (HQ) U[I::IQ] = x[I::IQ] * D.ucon[0] * gdet;
    if (HD) U[I::ID] = x[I::ID] * D.ucon[0] * gdet;
#pragma unroll
    for (int p = 0; p < I::NF; ++p) res[p] = (U[p] - Z.Ui[p]) / dt - Z.S[p];
    if (I::EM) {
        const double tau = Z.tau;
        const double th = (gam-1) * x[1] / x[0];
        S.theta_clamped = th < SMALL;
        const double Theta_new = kmax(th, SMALL);
        const double dt_Theta = (Theta_new - Z.Theta_old) / dt;
        if (HQ) {
            double rq = res[I::IQ];
            const double dUq = -gdet * (x[I::IQ] / tau);
            rq -= 0.5*(dUq + Z.dUi_q);
            double q0 = Z.cq0 * dt_Theta;
#pragma unroll
            for (int mu = 0; mu < 4; ++mu) q0 -= Z.cq[mu] * V.dt_ucov[mu];
            double q0t = q0;
            if (E.higher_order_terms) q0t *= Z.fac_q;
            double dUqt = gdet * (q0t / tau);
            if (E.higher_order_terms) dUqt += Z.gq * V.div_ucon;
            rq -= dUqt;
            rq *= tau;
            if (E.higher_order_terms) rq *= Z.norm_q;
            res[I::IQ] = rq;
        }
        if (HD) {
            double rd = res[I::ID];
            const double dUd = -gdet * (x[I::ID] / tau);
            rd -= 0.5*(dUd + Z.dUi_d);
            double dP0 = Z.cd0 * V.div_ucon;
#pragma unroll
            for (int mu = 0; mu < 4; ++mu) dP0 += Z.cd[mu] * V.dt_ucov[mu];
            double dP0t = dP0;
            if (E.higher_order_terms) dP0t *= Z.fac_d;
            double dUdt_ = gdet * (dP0t / tau);
            if (E.higher_order_terms) dUdt_ += Z.gd * V.div_ucon;
            rd -= dUdt_;
            rd *= tau;
            if (E.higher_order_terms) rd *= Z.norm_d;
            res[I::ID] = rd;
        }
    }
}

template <bool HQ, bool HD>
__device__ __forceinline__ void residual(const EmhdArgs& E, double gam, double dt, const ResidZone<Imp<HQ, HD>::NF>& Z,
                                         const double* x, double* res)
{
    VelState V;
    ResidState S;
    velocity_part<HQ, HD>(dt, Z, x, V);
    residual_with<HQ, HD>(E, gam, dt, Z, x, V, res, S);
}

// Forward-difference Jacobian (Implicit::calc_jacobian, implicit.hpp:208-255).  res: residual at x.
template <bool HQ, bool HD>
__device__ __forceinline__ void jacobian_fd(const EmhdArgs& E, double gam, double dt, double delta,
                                            const ResidZone<Imp<HQ, HD>::NF>& Z, const double* x,
                                            double* res, double (&J)[Imp<HQ, HD>::NF][Imp<HQ, HD>::NF])
{
    constexpr int NF = Imp<HQ, HD>::NF;
    VelState V0;
    ResidState S;
    velocity_part<HQ, HD>(dt, Z, x, V0);
    residual_with<HQ, HD>(E, gam, dt, Z, x, V0, res, S);
#pragma unroll
    for (int col = 0; col < NF; ++col) {
        double xp[NF];
#pragma unroll
        for (int p = 0; p < NF; ++p) xp[p] = x[p];
        if (fabs(x[col]) < (0.5 * delta)) xp[col] = x[col] + delta;
        else xp[col] = (1 + delta) * x[col];
        double rp[NF];
        if (col >= 2 && col <= 4) {
            VelState V;
            velocity_part<HQ, HD>(dt, Z, xp, V);
            residual_with<HQ, HD>(E, gam, dt, Z, xp, V, rp, S);
        } else {
            residual_with<HQ, HD>(E, gam, dt, Z, xp, V0, rp, S);
        }
        const double h = xp[col] - x[col] + SMALL;
#pragma unroll
        for (int row = 0; row < NF; ++row) J[row][col] = (rp[row] - res[row]) / h;
    }
}

// Exact Jacobian of the same residual by a hand-written tangent.  Each column is one seed
// direction, handled by its own code path so that no work is spent on structurally zero terms:
//   rho, u      enter through eta, p_gas and (EMHD) q, dP via Theta and cs2
//   u~1..u~3    enter through u^mu, u_mu, b^mu, b_mu and b^2 (Lorentz factor, lowering, b^0)
//   q~, dP~     enter linearly through q, dP and their conserved forms
// then the product rule through T^t_mu, the conserved variables and the EMHD source terms.  The
// tangent is not bound to the reference's operation order, so divisions are replaced by products
// with reciprocals computed once.
template <bool HQ, bool HD>
__device__ __forceinline__ void jacobian_exact(const EmhdArgs& E, double gam, double dt,
                                               const ResidZone<Imp<HQ, HD>::NF>& Z, const double* x,
                                               double* res, double (&J)[Imp<HQ, HD>::NF][Imp<HQ, HD>::NF])
{
    using I = Imp<HQ, HD>;
    constexpr int NF = I::NF;
    VelState V;
    ResidState S;
    velocity_part<HQ, HD>(dt, Z, x, V);
    residual_with<HQ, HD>(E, gam, dt, Z, x, V, res, S);
    const CenterGeom& G = Z.G;
    const FourVec<double>& D = V.D;
    const double u0 = D.ucon[0], b0 = D.bcon[0];
    const double gdet = G.gdet, rho = x[0], uu = x[1];
    const double inv_dt = 1. / dt, inv_u0 = 1. / u0, inv_rho = 1. / rho;
    const double inv_tau = I::EM ? 1. / Z.tau : 0.;
    const double gdt = gdet * inv_dt;
    const bool emt = I::EM && E.feedback;
    // EMHD tensor pieces: T^t_mu = ... + (q/|b|) X_mu - dP Y_mu
    double X[4], Y[4], qb = 0., fq = 1., fd = 1., inv_bsq = 0., inv_bmag = 0.;
    double dq[2] = {0., 0.}, ddP[2] = {0., 0.};
    if (emt) {
        inv_bsq = 1. / S.bsq;
        inv_bmag = 1. / S.bmag;
        qb = S.q * inv_bmag;
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) {
            X[mu] = u0 * D.bcov[mu] + b0 * D.ucov[mu];
            Y[mu] = b0 * D.bcov[mu] * inv_bsq - ((double)(mu == 0) + u0 * D.ucov[mu]) * (1. / 3.);
        }
        if (E.higher_order_terms) {
            const double Th = S.Theta, cs2 = S.cs2, inv_den = 1. / (rho + gam * uu);
            const double dTh[2] = {-Th * inv_rho, (gam - 1) * inv_rho};
            const double dcs2[2] = {-cs2 * inv_den, (gam * (gam - 1) - gam * cs2) * inv_den};
            const double qt = HQ ? x[I::IQ] : 0., dPt = HD ? x[I::ID] : 0.;
            double sq, sd, dsq[2], dsd[2];
            if (E.closure == CL_KAPPA_ETA) {
                const double kt = E.kappa / E.tau, et = E.eta / E.tau;
                sq = kt * Th * Th;
                sd = et * Th;
#pragma unroll
                for (int a = 0; a < 2; ++a) { dsq[a] = 2. * kt * Th * dTh[a]; dsd[a] = et * dTh[a]; }
            } else {
                const double ac = E.conduction_alpha, av = E.viscosity_alpha;
                sq = rho * ac * cs2 * Th * Th;
                sd = rho * av * cs2 * Th;
#pragma unroll
                for (int a = 0; a < 2; ++a) {
                    const double dr = (a == 0) ? 1. : 0.;
                    dsq[a] = ac * Th * (dr * cs2 * Th + rho * dcs2[a] * Th + 2. * rho * cs2 * dTh[a]);
                    dsd[a] = av * (dr * cs2 * Th + rho * dcs2[a] * Th + rho * cs2 * dTh[a]);
                }
            }
            fq = sqrt(sq);
            fd = sqrt(sd);
            const double hq = (fq > 0.) ? 0.5 * qt / fq : 0., hd = (fd > 0.) ? 0.5 * dPt / fd : 0.;
#pragma unroll
            for (int a = 0; a < 2; ++a) { dq[a] = hq * dsq[a]; ddP[a] = hd * dsd[a]; }
        }
    }
    // Fills column k from the tangent of T^t_mu (dT), of u^t (du0), of dt_Theta and of div u and
    // dt u_mu (velocity columns only)
    auto column = [&](int k, const double* dT, double drho, double du0, double dqt, double ddPt,
                      double ddt_Theta, double ddiv, const double* dtu) {
        double dU[NF];
        dU[0] = (drho * u0 + rho * du0) * gdt;
        dU[1] = dT[0] * gdt + dU[0];
        dU[2] = dT[1] * gdt;
        dU[3] = dT[2] * gdt;
        dU[4] = dT[3] * gdt;
        if (HQ) dU[I::IQ] = (dqt * u0 + x[I::IQ] * du0) * gdt;
        if (HD) dU[I::ID] = (ddPt * u0 + x[I::ID] * du0) * gdt;
#pragma unroll
        for (int row = 0; row < NF; ++row) J[row][k] = dU[row];
        if (HQ) {
            double dq0 = Z.cq0 * ddt_Theta;
            if (dtu) {
#pragma unroll
                for (int mu = 0; mu < 4; ++mu) dq0 -= Z.cq[mu] * dtu[mu];
            }
            if (E.higher_order_terms) dq0 *= Z.fac_q;
            double dsrc = gdet * dq0 * inv_tau;
            if (E.higher_order_terms) dsrc += Z.gq * ddiv;
            double dr = (dU[I::IQ] + 0.5 * gdet * dqt * inv_tau - dsrc) * Z.tau;
            if (E.higher_order_terms) dr *= Z.norm_q;
            J[I::IQ][k] = dr;
        }
        if (HD) {
            double dd0 = Z.cd0 * ddiv;
            if (dtu) {
#pragma unroll
                for (int mu = 0; mu < 4; ++mu) dd0 += Z.cd[mu] * dtu[mu];
            }
            if (E.higher_order_terms) dd0 *= Z.fac_d;
            double dsrc = gdet * dd0 * inv_tau;
            if (E.higher_order_terms) dsrc += Z.gd * ddiv;
            double dr = (dU[I::ID] + 0.5 * gdet * ddPt * inv_tau - dsrc) * Z.tau;
            if (E.higher_order_terms) dr *= Z.norm_d;
            J[I::ID][k] = dr;
        }
    };
    const double dThn = (gam - 1) * inv_dt * inv_rho;
    // rho: d eta = 1
    {
        double dT[4];
        const double a = dq[0] * inv_bmag, c = ddP[0];
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) {
            dT[mu] = u0 * D.ucov[mu];
            if (emt) dT[mu] += a * X[mu] - c * Y[mu];
        }
        column(0, dT, 1., 0., 0., 0., S.theta_clamped ? 0. : -dThn * uu * inv_rho, 0., nullptr);
    }
    // u: d eta = gam, d p_tot = gam - 1
    {
        double dT[4];
        const double a = dq[1] * inv_bmag, c = ddP[1];
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) {
            dT[mu] = gam * u0 * D.ucov[mu] + (gam - 1) * (double)(mu == 0);
            if (emt) dT[mu] += a * X[mu] - c * Y[mu];
        }
        column(1, dT, 0., 0., 0., 0., S.theta_clamped ? 0. : dThn, 0., nullptr);
    }
    // velocities
    const double inv_alpha = sqrt(-G.gcon0[0]), alpha = 1. / inv_alpha, inv_gamma = 1. / V.gamma;
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        double gk = 0.;
#pragma unroll
        for (int w = 0; w < 3; ++w) gk += G.gcov[v+1][w+1] * x[2 + w];
        const double dgam = gk * inv_gamma;
        double du[4], dul[4], db[4], dbl[4];
        du[0] = dgam * inv_alpha;
#pragma unroll
        for (int m = 1; m < 4; ++m) du[m] = (double)(m - 1 == v) - alpha * G.gcon0[m] * dgam;
        lower4(G.gcov, du, dul);
        double d0 = 0.;
#pragma unroll
        for (int w = 0; w < 3; ++w) d0 += Z.B[w] * dul[w+1];
        db[0] = d0;
#pragma unroll
        for (int m = 1; m < 4; ++m) db[m] = (d0 * D.ucon[m] + b0 * du[m] - D.bcon[m] * du[0]) * inv_u0;
        lower4(G.gcov, db, dbl);
        const double dbs = S.bsq_clamped ? 0. : 2. * dot4(D.bcov, db);
        double dT[4];
#pragma unroll
        for (int mu = 0; mu < 4; ++mu)
            dT[mu] = dbs * u0 * D.ucov[mu] + S.eta * (du[0] * D.ucov[mu] + u0 * dul[mu])
                   + 0.5 * dbs * (double)(mu == 0) - (db[0] * D.bcov[mu] + b0 * dbl[mu]);
        if (emt) {
            const double dqb = -S.q * 0.5 * dbs * inv_bmag * inv_bsq;
            const double yb = b0 * dbs * inv_bsq * inv_bsq;
#pragma unroll
            for (int mu = 0; mu < 4; ++mu) {
                const double dX = du[0] * D.bcov[mu] + u0 * dbl[mu] + db[0] * D.ucov[mu] + b0 * dul[mu];
                const double dY = (db[0] * D.bcov[mu] + b0 * dbl[mu]) * inv_bsq - yb * D.bcov[mu]
                                - (du[0] * D.ucov[mu] + u0 * dul[mu]) * (1. / 3.);
                dT[mu] += dqb * X[mu] + qb * dX - S.dP * dY;
            }
        }
        double dtu[4], ddiv = 0.;
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) { dtu[mu] = dul[mu] * inv_dt; ddiv += G.gcon0[mu] * dtu[mu]; }
        column(2 + v, dT, 0., du[0], 0., 0., 0., ddiv, dtu);
    }
    // q~ and dP~
    if (HQ) {
        double dT[4];
        const double a = fq * inv_bmag;
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) dT[mu] = emt ? a * X[mu] : 0.;
        column(I::IQ, dT, 0., 0., 1., 0., 0., 0., nullptr);
    }
    if (HD) {
        double dT[4];
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) dT[mu] = emt ? -fd * Y[mu] : 0.;
        column(I::ID, dT, 0., 0., 0., 1., 0., 0., nullptr);
    }
}

// ------------------------------------------------------------------------------ dense solves
// Householder QR with column pivoting, Q^T b, back substitution and the inverse permutation, in the
// operation order of KokkosBatched SerialQR / SerialApplyQ (left, transpose) / SerialTrsv (upper,
// non-unit) / SerialApplyPivot (left, backward) as called at implicit.cpp:374-383.  Every index is
// a compile-time constant so A stays in registers.
template <int N>
__device__ __forceinline__ void qr_solve(double (&A)[N][N], double (&b)[N])
{
    double tau[N], norm[N];
    int piv[N];
#pragma unroll
    for (int c = 0; c < N; ++c) {
        double s = 0.;
#pragma unroll
        for (int r = 0; r < N; ++r) s += A[r][c] * A[r][c];
        norm[c] = s;
    }
#pragma unroll
    for (int k = 0; k < N; ++k) {
        int p = 0;
        double mx = norm[k];
#pragma unroll
        for (int c = k + 1; c < N; ++c) if (norm[c] > mx) { mx = norm[c]; p = c - k; }
        piv[k] = p;
#pragma unroll
        for (int c = k + 1; c < N; ++c) {
            if (c == k + p) {
                const double t = norm[k]; norm[k] = norm[c]; norm[c] = t;
#pragma unroll
                for (int r = 0; r < N; ++r) { const double a = A[r][k]; A[r][k] = A[r][c]; A[r][c] = a; }
            }
        }
        double nx2 = 0.;
#pragma unroll
        for (int r = k + 1; r < N; ++r) nx2 += A[r][k] * A[r][k];
        if (nx2 == 0.) {
            A[k][k] = -A[k][k];
            tau[k] = 0.5;
        } else {
            const double chi1 = A[k][k];
            const double nchi1 = fabs(chi1);
            const double nx = sqrt(nx2 + nchi1 * nchi1);
            const double alph = (chi1 < 0 ? 1. : -1.) * nx;
            const double cma = chi1 - alph;
            const double inv = 1. / cma;
#pragma unroll
            for (int r = k + 1; r < N; ++r) A[r][k] *= inv;
            const double cma2 = cma * cma;
            tau[k] = 0.5 + 0.5 * (nx2 / cma2);
            A[k][k] = alph;
        }
        const double inv_tau = 1. / tau[k];
        double w[N];
#pragma unroll
        for (int c = k + 1; c < N; ++c) {
            double t = A[k][c];
#pragma unroll
            for (int r = k + 1; r < N; ++r) t += A[r][k] * A[r][c];
            w[c] = t * inv_tau;
        }
#pragma unroll
        for (int c = k + 1; c < N; ++c) A[k][c] -= w[c];
#pragma unroll
        for (int c = k + 1; c < N; ++c)
#pragma unroll
            for (int r = k + 1; r < N; ++r) A[r][c] -= A[r][k] * w[c];
#pragma unroll
        for (int c = k + 1; c < N; ++c) norm[c] -= A[k][c] * A[k][c];
    }
#pragma unroll
    for (int k = 0; k < N; ++k) {
        const double inv_tau = 1. / tau[k];
        double t = b[k];
#pragma unroll
        for (int r = k + 1; r < N; ++r) t += A[r][k] * b[r];
        const double wk = t * inv_tau;
        b[k] -= wk;
#pragma unroll
        for (int r = k + 1; r < N; ++r) b[r] -= A[r][k] * wk;
    }
#pragma unroll
    for (int p = N - 1; p >= 0; --p) {
        b[p] = b[p] / A[p][p];
#pragma unroll
        for (int r = 0; r < p; ++r) b[r] -= A[r][p] * b[p];
    }
#pragma unroll
    for (int k = N - 1; k >= 0; --k) {
#pragma unroll
        for (int c = k + 1; c < N; ++c) {
            if (c == k + piv[k]) { const double t = b[k]; b[k] = b[c]; b[c] = t; }
        }
    }
}

// The use_qr = false path: KokkosBatched SerialLU (no pivoting, diagonal nudged by SMALL) and the
// upper-triangular solve alone, as implicit.cpp:387-401 calls them.
template <int N>
__device__ __forceinline__ void lu_solve(double (&A)[N][N], double (&b)[N])
{
#pragma unroll
    for (int p = 0; p < N; ++p) {
        const double a_real = A[p][p];
        A[p][p] += -SMALL * (double)(a_real < 0);
        A[p][p] += SMALL * (double)(a_real >= 0);
        const double a11 = A[p][p];
#pragma unroll
        for (int r = p + 1; r < N; ++r) {
            A[r][p] /= a11;
#pragma unroll
            for (int c = p + 1; c < N; ++c) A[r][c] -= A[r][p] * A[p][c];
        }
    }
#pragma unroll
    for (int p = N - 1; p >= 0; --p) {
        b[p] = b[p] / A[p][p];
#pragma unroll
        for (int r = 0; r < p; ++r) b[r] -= A[r][p] * b[p];
    }
}

// ------------------------------------------------------------------------------ kernels
__device__ __forceinline__ bool interior_zone(const Dims& d, long long t, int& k, int& j, int& i, long long& c)
{
    const long long nz = (long long)d.nx1 * d.nx2 * d.nx3;
    if (t >= nz) return false;
    i = d.is + (int)(t % d.nx1);
    j = d.js + (int)((t / d.nx1) % d.nx2);
    k = d.ks + (int)(t / ((long long)d.nx1 * d.nx2));
    c = ((long long)k * d.n2 + j) * d.n1 + i;
    return true;
}

__device__ __forceinline__ void load10(const khb_fields& F, long long c, double* out)
{
#pragma unroll
    for (int p = 0; p < 10; ++p) out[p] = F.v[p] ? F.v[p][c] : 0.;
}

// Flux::MeshPtoU for the 10-slot state over the entire block
__global__ void __launch_bounds__(128) k_emhd_ptou(Dims d, DevGeom g, double gam, EmhdArgs E, khb_fields P, khb_fields U)
{
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= d.N) return;
    int k, j, i;
    zone_kji(d, c, k, j, i);
    CenterGeom G;
    load_center(g, j, i, G);
    double Pz[10], Uz[10];
    load10(P, c, Pz);
    emhd_p_to_u(E, gam, G, Pz, Uz);
#pragma unroll
    for (int p = 0; p < 8; ++p) U.v[p][c] = Uz[p];
    if (E.conduction) U.v[8][c] = Uz[8];
    if (E.viscosity) U.v[9][c] = Uz[9];
}

// ------------------------------------------------------------------------------ explicit EMHD step
// Flux::GetFlux with the EMHD variables (get_flux.hpp:60-373): one thread per face, every active
// slot reconstructed, U and F with the EMHD tensor, EMHD signal speeds, LLF/HLLE.  F is [10][N].
template <int DIR, int RECON, bool HQ, bool HD>
__global__ void __launch_bounds__(128) k_flux_emhd(Dims d, DevGeom g, Phys ph, EmhdArgs E, khb_fields P,
                                                   double* __restrict__ F, double* __restrict__ ctop, Box bx)
{
    int i, j, k;
    if (!box_cell(bx, blockIdx.x, i, j, k)) return;
    const long long c = ((long long)k*d.n2 + j)*d.n1 + i;
    const long long st = (DIR == 1) ? 1 : ((DIR == 2) ? d.sj : d.sk);
    const int loc = DIR - 1;
    const double gam = ph.gam;
    const long long gi = (long long)j*g.G1 + i;
    double gcov[4][4], gcon0[4];
#pragma unroll
    for (int m = 0; m < 16; ++m) gcov[m/4][m%4] = __ldg(g.gcov[loc] + m*g.gs + gi);
#pragma unroll
    for (int m = 0; m < 4; ++m) gcon0[m] = __ldg(g.gcon[loc] + m*g.gs + gi);
    const double gcondd = __ldg(g.gcon[loc] + (DIR*4 + DIR)*g.gs + gi);
    const double gdet = __ldg(g.gdet[loc] + gi);
    double Pl[10], Pr[10];
#pragma unroll
    for (int p = 0; p < 10; ++p) {
        const bool on = p < 8 || (p == 8 && HQ) || (p == 9 && HD);
        if (!on) { Pl[p] = Pr[p] = 0.; continue; }
        const double* q = P.v[p];
        const double x0 = __ldg(q + c - 3*st), x1 = __ldg(q + c - 2*st), x2 = __ldg(q + c - st);
        const double x3 = __ldg(q + c), x4 = __ldg(q + c + st), x5 = __ldg(q + c + 2*st);
        Pl[p] = recon_right<RECON, double>(x0, x1, x2, x3, x4);
        Pr[p] = recon_left<RECON, double>(x1, x2, x3, x4, x5);
    }
    FourVec<double> D;
    double Ul[10], Fl[10], Ur[10], Fr[10], cmaxL, cminL, cmaxR, cminR;
    calc_4vecs<double, true>(gcov, gcon0[0], gcon0, Pl, D);
    emhd_prim_to_flux(E, gam, gdet, Pl, D, 0, Ul);
    emhd_prim_to_flux(E, gam, gdet, Pl, D, DIR, Fl);
    emhd_vchar(E, gam, Pl, D, gcon0[0], gcon0[DIR], gcondd, DIR, cmaxL, cminL);
    calc_4vecs<double, true>(gcov, gcon0[0], gcon0, Pr, D);
    emhd_prim_to_flux(E, gam, gdet, Pr, D, 0, Ur);
    emhd_prim_to_flux(E, gam, gdet, Pr, D, DIR, Fr);
    emhd_vchar(E, gam, Pr, D, gcon0[0], gcon0[DIR], gcondd, DIR, cmaxR, cminR);
    const double cmax = kmax(kmax(0., cmaxL), cmaxR);
    const double cmin = -kmin(kmin(0., cminL), cminR);
#pragma unroll
    for (int p = 0; p < 10; ++p) {
        const bool on = p < 8 || (p == 8 && HQ) || (p == 9 && HD);
        double f = 0.;
        if (on) {
            if (ph.riemann == 0) f = 0.5 * (Fl[p] + Fr[p] - kmax(cmax, cmin) * (Ur[p] - Ul[p]));
            else f = (cmax*Fl[p] + cmin*Fr[p] - cmax*cmin*(Ur[p] - Ul[p])) / (cmax + cmin);
        }
        F[p*d.N + c] = f;
    }
    ctop[c] = kmax(cmax, cmin);
}

// dU/dt over the interior: -div F of every active slot (flux-CT for B), plus Flux::AddGeoSource with
// the EMHD stress tensor (flux.cpp:395-444); the EMHD explicit sources are added by k_emhd_sources.
// With dtm the stage's zone timestep minimum is accumulated as in k_zone.
template <bool HQ, bool HD>
__global__ void __launch_bounds__(128) k_emhd_dudt(Dims d, DevGeom g, Phys ph, EmhdArgs E, const double* F1,
                                                   const double* F2, const double* F3, const double* c1,
                                                   const double* c2, const double* c3, khb_fields Ps,
                                                   khb_fields dUdt, int dtm, unsigned long long* word, Box bx)
{
    int i, j, k;
    double ndt_zone = 1.7976931348623157e308;
    if (box_cell(bx, blockIdx.x, i, j, k)) {
        const long long c = ((long long)k*d.n2 + j)*d.n1 + i;
        const long long N = d.N, sj = d.sj, sk = d.sk;
        const double a1 = ph.dx2*ph.dx3, a2 = ph.dx1*ph.dx3, a3 = ph.dx1*ph.dx2;
        const double vol = ph.dx1*ph.dx2*ph.dx3;
        double du_[10];
#pragma unroll
        for (int p = 0; p < 10; ++p) {
            const bool on = p < 5 || (p == 8 && HQ) || (p == 9 && HD);
            if (!on) { du_[p] = 0.; continue; }
            double du = (a1 * __ldg(F1 + p*N + c + 1) - a1 * __ldg(F1 + p*N + c));
            if (d.ndim >= 2) du += a2 * __ldg(F2 + p*N + c + sj) - a2 * __ldg(F2 + p*N + c);
            if (d.ndim == 3) du += a3 * __ldg(F3 + p*N + c + sk) - a3 * __ldg(F3 + p*N + c);
            du_[p] = -du / vol;
        }
        double db[3];
        ct_divergence<double>(d, ph, F1, F2, F3, c, j, db);
#pragma unroll
        for (int v = 0; v < 3; ++v) du_[5 + v] = db[v];
        if (!ph.cart_minkowski) {
            CenterGeom G;
            load_center(g, j, i, G);
            double Pz[10];
            load10(Ps, c, Pz);
            FourVec<double> D;
            calc_4vecs<double, true>(G.gcov, G.gcon0[0], G.gcon0, Pz, D);
            double new_du[4] = {0., 0., 0., 0.};
            const long long cg = (long long)j*g.n1 + i, cs = (long long)(d.n2)*g.n1;
            const double gam = ph.gam;
#pragma unroll
            for (int mu = 0; mu < 4; ++mu) {
                double Tmu[4];
                if ((E.conduction || E.viscosity) && E.feedback) {
                    const double qt = E.conduction ? Pz[8] : 0., dPt = E.viscosity ? Pz[9] : 0.;
                    const double Theta = (gam - 1) * Pz[1] / Pz[0];
                    const double cs2 = gam * (gam - 1) * Pz[1] / (Pz[0] + gam * Pz[1]);
                    double q, dP;
                    convert_q_dP(E, qt, dPt, Pz[0], Theta, cs2, q, dP);
                    emhd_tensor(Pz[0], Pz[1], (gam - 1) * Pz[1], q, dP, D, mu, Tmu);
                } else {
                    calc_tensor<double, true>(Pz[0], Pz[1], (gam - 1) * Pz[1], D, mu, Tmu);
                }
#pragma unroll
                for (int nu = 0; nu < 4; ++nu)
#pragma unroll
                    for (int lam = 0; lam < 4; ++lam)
                        new_du[lam] += Tmu[nu] * __ldg(g.gdet_conn + ((nu*4 + lam)*4 + mu)*cs + cg);
            }
            du_[1] += new_du[0];
            du_[2] += new_du[1];
            du_[3] += new_du[2];
            du_[4] += new_du[3];
        }
#pragma unroll
        for (int p = 0; p < 10; ++p) if (dUdt.v[p]) dUdt.v[p][c] = du_[p];
        if (dtm) {
            const double z = 1.0 / (1 / (ph.dx1 / kmax(c1[c], 0.0)) + 1 / (ph.dx2 / kmax(c2[c], 0.0)) +
                                    1 / (ph.dx3 * 1 / kmax(c3[c], 0.0)));
            if (!isnan(z)) ndt_zone = z;
        }
    }
    if (dtm) block_min_ndt(ndt_zone, word);
}

// The explicit half of AddStateUpdate for an ImEx stage (imex_step.cpp:200-215 with the Explicit
// flag on B only) and the solver's starting state: P_out/U_out = the sub-step state over the whole
// block (the implicit guess copy, imex_step.cpp:228-238), B_U updated over the interior with the
// stage weights, then B_P = B_U/gdet everywhere (B_FluxCT::BlockUtoP).
__global__ void __launch_bounds__(128) k_imex_explicit(Dims d, DevGeom g, khb_fields Psub, khb_fields Usub,
                                                       khb_fields Ufull, khb_fields dUdt, khb_fields Pout,
                                                       khb_fields Uout, double g0, double g1, double bdt)
{
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= d.N) return;
    int k, j, i;
    zone_kji(d, c, k, j, i);
    const bool interior = i >= d.is && i <= d.ie && j >= d.js && j <= d.je && k >= d.ks && k <= d.ke;
    const double gdet = __ldg(g.gdet[3] + (long long)j*g.G1 + i);
#pragma unroll
    for (int p = 0; p < 10; ++p) {
        if (!Pout.v[p]) continue;
        if (p >= 5 && p < 8) {
            double u = Usub.v[p][c];
            if (interior) {
                u = g0 * u + g1 * Ufull.v[p][c];
                u = 1.0 * u + bdt * dUdt.v[p][c];
            }
            Uout.v[p][c] = u;
            Pout.v[p][c] = u / gdet;
        } else {
            Pout.v[p][c] = Psub.v[p][c];
            Uout.v[p][c] = Usub.v[p][c];
        }
    }
}

// EMHD::AddSource temporaries (emhd.cpp:329-343): u_mu (4) and Theta over the interior plus one halo zone
__global__ void __launch_bounds__(128) k_emhd_temps(Dims d, DevGeom g, double gam, khb_fields P, double* tmp,
                                                    int il, int jl, int kl, int ci, int cj, int ck)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)ci * cj * ck) return;
    const int i = il + (int)(t % ci);
    const int j = jl + (int)((t / ci) % cj);
    const int k = kl + (int)(t / ((long long)ci * cj));
    const long long c = ((long long)k * d.n2 + j) * d.n1 + i;
    CenterGeom G;
    load_center(g, j, i, G);
    const double rho = P.v[0][c], u = P.v[1][c], u1 = P.v[2][c], u2 = P.v[3][c], u3 = P.v[4][c];
    const double gamma = lorentz(G.gcov, u1, u2, u3);
    const double alpha = 1. / sqrt(-G.gcon0[0]);
    double ucon[4], ucov[4];
    ucon[0] = gamma / alpha;
    ucon[1] = u1 - gamma * alpha * G.gcon0[1];
    ucon[2] = u2 - gamma * alpha * G.gcon0[2];
    ucon[3] = u3 - gamma * alpha * G.gcon0[3];
    lower4(G.gcov, ucon, ucov);
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) tmp[mu * d.N + c] = ucov[mu];
    tmp[4 * d.N + c] = kmax((gam - 1) * u / rho, SMALL);
}

// KReconstruction::slope_limit<linear_mc> (reconstruction.hpp:781-798)
__device__ __forceinline__ double slope_mc(double x1, double x2, double x3, double dx)
{
    const double Dqm = 2 * (x2 - x1) / dx;
    const double Dqp = 2 * (x3 - x2) / dx;
    const double Dqc = 0.5 * (x3 - x1) / dx;
    if (Dqm * Dqp <= 0) return 0;
    if ((fabs(Dqm) < fabs(Dqp)) && (fabs(Dqm) < fabs(Dqc))) return Dqm;
    else if (fabs(Dqp) < fabs(Dqc)) return Dqp;
    return Dqc;
}

// EMHD::AddSource explicit sources (emhd.cpp:346-394, gradient_calc emhd_utils.hpp:55-79), added to dUdt
__global__ void __launch_bounds__(128) k_emhd_sources(Dims d, DevGeom g, const double* conn, double gam, EmhdArgs E,
                                                      Phys ph, khb_fields P, const double* tmp, khb_fields dUdt)
{
    int k, j, i;
    long long c;
    if (!interior_zone(d, (long long)blockIdx.x * blockDim.x + threadIdx.x, k, j, i, c)) return;
    CenterGeom G;
    load_center(g, j, i, G);
    double Pz[10];
    load10(P, c, Pz);
    FourVec<double> D;
    calc_4vecs<double, true>(G.gcov, G.gcon0[0], G.gcon0, Pz, D);
    const double bsq = kmax(dot4(D.bcon, D.bcov), SMALL);
    double tau, chi_e, nu_e;
    set_parameters(E, gam, Pz[0], Pz[1], E.conduction ? Pz[8] : 0., E.viscosity ? Pz[9] : 0., bsq,
                   g.rcen[(long long)j * d.n1 + i], tau, chi_e, nu_e);
    const long long N = d.N, sj = d.sj, sk = d.sk;
    const bool do_2d = d.ndim > 1, do_3d = d.ndim > 2;
    double grad_ucov[4][4], grad_Theta[4];
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
        const double* T = tmp + mu * N;
        grad_ucov[0][mu] = 0;
        grad_ucov[1][mu] = slope_mc(T[c - 1], T[c], T[c + 1], ph.dx1);
        grad_ucov[2][mu] = do_2d ? slope_mc(T[c - sj], T[c], T[c + sj], ph.dx2) : 0.;
        grad_ucov[3][mu] = do_3d ? slope_mc(T[c - sk], T[c], T[c + sk], ph.dx3) : 0.;
    }
    const long long gj = (long long)j * d.n1 + i, gs = (long long)d.n1 * d.n2;
    double ucov_c[4];
#pragma unroll
    for (int lam = 0; lam < 4; ++lam) ucov_c[lam] = tmp[lam * N + c];
#pragma unroll
    for (int mu = 0; mu < 4; ++mu)
#pragma unroll
        for (int nu = 0; nu < 4; ++nu)
#pragma unroll
            for (int lam = 0; lam < 4; ++lam)
                grad_ucov[mu][nu] -= __ldg(conn + (lam*16 + mu*4 + nu) * gs + gj) * ucov_c[lam];
    {
        const double* T = tmp + 4 * N;
        grad_Theta[0] = 0;
        grad_Theta[1] = slope_mc(T[c - 1], T[c], T[c + 1], ph.dx1);
        grad_Theta[2] = do_2d ? slope_mc(T[c - sj], T[c], T[c + sj], ph.dx2) : 0.;
        grad_Theta[3] = do_3d ? slope_mc(T[c - sk], T[c], T[c + sk], ph.dx3) : 0.;
    }
    const long long gi = (long long)j * g.G1 + i;
    double div_ucon = 0;
#pragma unroll
    for (int mu = 0; mu < 4; ++mu)
#pragma unroll
        for (int nu = 0; nu < 4; ++nu)
            div_ucon += __ldg(g.gcon[3] + (mu*4 + nu) * g.gs + gi) * grad_ucov[mu][nu];
    const double rho = Pz[0];
    const double Theta = tmp[4 * N + c];
    const double gdet = G.gdet;
    if (E.conduction) {
        const double qtilde = Pz[8];
        const double inv_mag_b = 1. / sqrt(bsq);
        double q0 = 0;
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) q0 -= rho * chi_e * (D.bcon[mu] * inv_mag_b) * grad_Theta[mu];
#pragma unroll
        for (int mu = 0; mu < 4; ++mu)
#pragma unroll
            for (int nu = 0; nu < 4; ++nu)
                q0 -= rho * chi_e * (D.bcon[mu] * inv_mag_b) * Theta * D.ucon[nu] * grad_ucov[nu][mu];
        double q0_tilde = q0;
        if (E.higher_order_terms) q0_tilde *= (chi_e != 0) ? sqrt(tau / (chi_e * rho * Theta * Theta)) : 0.0;
        double s = dUdt.v[8][c];
        s += gdet * q0_tilde / tau;
        if (E.higher_order_terms) s += gdet * (qtilde / 2.) * div_ucon;
        dUdt.v[8][c] = s;
    }
    if (E.viscosity) {
        const double dPtilde = Pz[9];
        double dP0 = -rho * nu_e * div_ucon;
#pragma unroll
        for (int mu = 0; mu < 4; ++mu)
#pragma unroll
            for (int nu = 0; nu < 4; ++nu)
                dP0 += 3. * rho * nu_e * (D.bcon[mu] * D.bcon[nu] / bsq) * grad_ucov[mu][nu];
        double dP0_tilde = dP0;
        if (E.higher_order_terms) dP0_tilde *= (nu_e != 0) ? sqrt(tau / (nu_e * rho * Theta)) : 0.0;
        double s = dUdt.v[9][c];
        s += gdet * dP0_tilde / tau;
        if (E.higher_order_terms) s += gdet * (dPtilde / 2.) * div_ucon;
        dUdt.v[9][c] = s;
    }
}

// Block maximum of non-negative doubles (NaN ignored, as Kokkos::Max's `>` join ignores it) and one
// atomicMax on the bit pattern, whose integer order matches the order of non-negative doubles.
__device__ __forceinline__ void block_max_norm(double v, unsigned long long* word)
{
    unsigned long long b = (v == v && v > 0.) ? (unsigned long long)__double_as_longlong(v) : 0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long x = __shfl_xor_sync(0xffffffffu, b, o);
        b = x > b ? x : b;
    }
    __shared__ unsigned long long wmax[32];
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = b;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long m = wmax[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = wmax[w] > m ? wmax[w] : m;
        atomicMax(word, m);
    }
}

// One Newton iteration of Implicit::Step for every interior zone (implicit.cpp:286-522).
// words[it-1]: maximum solve_norm of iteration it (bits); words[IMP_ITER_WORD]: iterations taken.
template <bool HQ, bool HD, int JAC>
__global__ void __launch_bounds__(128) k_implicit_iter(Dims d, DevGeom g, double gam, EmhdArgs E, ImplicitArgs ip,
                                                       ImpFields f, double dt, unsigned long long* words, int iter)
{
    using I = Imp<HQ, HD>;
    constexpr int NF = I::NF;
    if (iter > 1) {
        const double prev = __longlong_as_double((long long)words[iter - 2]);
        if ((iter - 1) >= ip.min_nonlinear_iter && prev < ip.rootfind_tol) return;   // the loop has ended
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicMax(words + IMP_ITER_WORD, (unsigned long long)iter);
    int k, j, i;
    long long c;
    double norm_out = 0.;
    if (interior_zone(d, (long long)blockIdx.x * blockDim.x + threadIdx.x, k, j, i, c)) {
        double sf = f.solve_fail[c];
        double sn = f.solve_norm[c];
        if (sf != SOLVE_FAIL) {
            sf = SOLVE_CONVERGED;
            ResidZone<NF> Z;
            load_center(g, j, i, Z.G);
            double Pf[10], Uf[10], Ps[10], Sz[10], Psol[10];
            load10(f.Pf, c, Pf); load10(f.Uf, c, Uf); load10(f.Ps, c, Ps); load10(f.S, c, Sz); load10(f.Psol, c, Psol);
            setup_zone<HQ, HD>(E, gam, g.rcen[(long long)j * d.n1 + i], Pf, Uf, Ps, Sz, Psol, Z);
            double x[NF], xs[NF];
#pragma unroll
            for (int p = 0; p < 5; ++p) { x[p] = Psol[p]; xs[p] = Ps[p]; }
            if (HQ) { x[I::IQ] = Psol[8]; xs[I::IQ] = Ps[8]; }
            if (HD) { x[I::ID] = Psol[9]; xs[I::ID] = Ps[9]; }
            double J[NF][NF], res[NF], delta[NF];
            if (JAC == 1) jacobian_exact<HQ, HD>(E, gam, dt, Z, x, res, J);
            else jacobian_fd<HQ, HD>(E, gam, dt, ip.jacobian_delta, Z, x, res, J);
#pragma unroll
            for (int p = 0; p < NF; ++p) delta[p] = -res[p];
            if (ip.use_qr) qr_solve<NF>(J, delta);
            else lu_solve<NF>(J, delta);
            // implicit_set_step (implicit.cpp:426-521)
            bool failed_now = false;
            double lambda = ip.linesearch_lambda;
            if ((x[0] + lambda*delta[0] < 0.) || (x[1] + lambda*delta[1] < 0.)) {
                sf = SOLVE_BACKTRACK;
                lambda = 0.1;
            }
            if ((x[0] + lambda*delta[0] < 0.) || (x[1] + lambda*delta[1] < 0.)) {
                sf = SOLVE_FAIL;
#pragma unroll
                for (int p = 0; p < NF; ++p) x[p] = xs[p];
                failed_now = true;
            }
            if (!failed_now) {
                if (ip.linesearch) {
                    double nrm = 0.;
#pragma unroll
                    for (int p = 0; p < NF; ++p) nrm += res[p]*res[p];
                    sn = sqrt(nrm);
                    const double f0 = 0.5 * sn;
                    const double fprime0 = -2. * f0;
                    for (int it = 0; it < ip.max_linesearch_iter; it++) {
                        double xl[NF];
#pragma unroll
                        for (int p = 0; p < NF; ++p) xl[p] = x[p] + (lambda * delta[p]);
                        residual<HQ, HD>(E, gam, dt, Z, xl, res);
                        nrm = 0.;
#pragma unroll
                        for (int p = 0; p < NF; ++p) nrm += res[p]*res[p];
                        sn = sqrt(nrm);
                        const double f1 = 0.5 * sn;
                        const int condition = f1 > (f0 * (1. - ip.linesearch_eps * lambda) + SMALL);
                        const double denom = (f1 - f0 - (fprime0 * lambda)) * condition + (1 - condition);
                        const double lambda_new = -fprime0 * lambda * lambda / denom * 0.5;
                        lambda = lambda * (1 - condition) + (condition * lambda_new);
                        if (condition == 0) break;
                    }
                }
#pragma unroll
                for (int p = 0; p < NF; ++p) x[p] += lambda * delta[p];
                residual<HQ, HD>(E, gam, dt, Z, x, res);
                double nrm = 0;
#pragma unroll
                for (int p = 0; p < NF; ++p) nrm += res[p]*res[p];
                sn = sqrt(nrm);
                if (isnan(sn)) {
                    sf = SOLVE_FAIL;
#pragma unroll
                    for (int p = 0; p < NF; ++p) x[p] = xs[p];
                } else if (sn > ip.rootfind_tol) {
                    sf = SOLVE_BEYOND_TOL;
                }
            }
#pragma unroll
            for (int p = 0; p < 5; ++p) f.Psol.v[p][c] = x[p];
            if (HQ) f.Psol.v[8][c] = x[I::IQ];
            if (HD) f.Psol.v[9][c] = x[I::ID];
            f.solve_fail[c] = sf;
            f.solve_norm[c] = sn;
        }
        norm_out = sn;
    }
    block_max_norm(norm_out, words + (iter - 1));
}

// Residual and Jacobian at the solver state (the split "implicit_jacobian" kernel, implicit.cpp:286-320)
template <bool HQ, bool HD, int JAC>
__global__ void __launch_bounds__(128) k_implicit_jacobian(Dims d, DevGeom g, double gam, EmhdArgs E, ImplicitArgs ip,
                                                           ImpFields f, double dt, double* jac, double* resid)
{
    using I = Imp<HQ, HD>;
    constexpr int NF = I::NF;
    int k, j, i;
    long long c;
    if (!interior_zone(d, (long long)blockIdx.x * blockDim.x + threadIdx.x, k, j, i, c)) return;
    ResidZone<NF> Z;
    load_center(g, j, i, Z.G);
    double Pf[10], Uf[10], Ps[10], Sz[10], Psol[10];
    load10(f.Pf, c, Pf); load10(f.Uf, c, Uf); load10(f.Ps, c, Ps); load10(f.S, c, Sz); load10(f.Psol, c, Psol);
    setup_zone<HQ, HD>(E, gam, g.rcen[(long long)j * d.n1 + i], Pf, Uf, Ps, Sz, Psol, Z);
    double x[NF];
#pragma unroll
    for (int p = 0; p < 5; ++p) x[p] = Psol[p];
    if (HQ) x[I::IQ] = Psol[8];
    if (HD) x[I::ID] = Psol[9];
    double J[NF][NF], res[NF];
    if (JAC == 1) jacobian_exact<HQ, HD>(E, gam, dt, Z, x, res, J);
    else jacobian_fd<HQ, HD>(E, gam, dt, ip.jacobian_delta, Z, x, res, J);
#pragma unroll
    for (int r = 0; r < NF; ++r) {
        resid[r * d.N + c] = res[r];
#pragma unroll
        for (int q = 0; q < NF; ++q) jac[(r * NF + q) * d.N + c] = J[r][q];
    }
}

// Implicit::FixSolve (fix_solve.cpp:44-130), pass 1: replacement values of failed zones from their
// neighbours' state before the pass, into out[nf][N]
template <bool HQ, bool HD>
__global__ void __launch_bounds__(128) k_fix_solve_avg(Dims d, khb_fields P, const double* solve_fail, double* out)
{
    using I = Imp<HQ, HD>;
    constexpr int NF = I::NF;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= d.N) return;
    if ((int)solve_fail[c] != SOLVE_FAIL) return;
    int k, j, i;
    zone_kji(d, c, k, j, i);
    int slot[NF];
#pragma unroll
    for (int p = 0; p < 5; ++p) slot[p] = p;
    if (HQ) slot[I::IQ] = 8;
    if (HD) slot[I::ID] = 9;
    double wsum = 0., wsum_x = 0., sum[NF], sum_x[NF];
#pragma unroll
    for (int p = 0; p < NF; ++p) { sum[p] = 0.; sum_x[p] = 0.; }
    for (int n = -1; n <= 1; n++) for (int m = -1; m <= 1; m++) for (int l = -1; l <= 1; l++) {
        const int ii = i + l, jj = j + m, kk = k + n;
        if (ii < 0 || ii >= d.n1 || jj < 0 || jj >= d.n2 || kk < 0 || kk >= d.n3) continue;
        const double w = 1./(abs(l) + abs(m) + abs(n) + 1);
        const long long cn = ((long long)kk * d.n2 + jj) * d.n1 + ii;
        const bool good = (int)solve_fail[cn] != SOLVE_FAIL;
        if (good) wsum += w;
        wsum_x += w;
#pragma unroll
        for (int p = 0; p < NF; ++p) {
            const double v = P.v[slot[p]][cn];
            if (good) sum[p] += w * v;
            sum_x[p] += w * v;
        }
    }
#pragma unroll
    for (int p = 0; p < NF; ++p) out[p * d.N + c] = (wsum < 1.e-10) ? sum_x[p]/wsum_x : sum[p]/wsum;
}

// Pass 2: write the replacements and recompute the conserved variables of the failed zones
template <bool HQ, bool HD>
__global__ void __launch_bounds__(128) k_fix_solve_apply(Dims d, DevGeom g, double gam, EmhdArgs E, khb_fields P,
                                                         khb_fields U, const double* solve_fail, const double* in)
{
    using I = Imp<HQ, HD>;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= d.N) return;
    if ((int)solve_fail[c] != SOLVE_FAIL) return;
    int k, j, i;
    zone_kji(d, c, k, j, i);
#pragma unroll
    for (int p = 0; p < 5; ++p) P.v[p][c] = in[p * d.N + c];
    if (HQ) P.v[8][c] = in[I::IQ * d.N + c];
    if (HD) P.v[9][c] = in[I::ID * d.N + c];
    CenterGeom G;
    load_center(g, j, i, G);
    double Pz[10], Uz[10];
    load10(P, c, Pz);
    emhd_p_to_u(E, gam, G, Pz, Uz);
#pragma unroll
    for (int p = 0; p < 8; ++p) U.v[p][c] = Uz[p];
    if (HQ) U.v[8][c] = Uz[8];
    if (HD) U.v[9][c] = Uz[9];
}

// ------------------------------------------------------------------------------ launchers
template <bool HQ, bool HD>
static void iter_hd(const Dims& d, const DevGeom& g, double gam, const EmhdArgs& E, const ImplicitArgs& ip,
                    const ImpFields& f, double dt, unsigned long long* words, int iter, cudaStream_t st)
{
    const long long nz = (long long)d.nx1 * d.nx2 * d.nx3;
    if (ip.jacobian == 1)
        k_implicit_iter<HQ, HD, 1><<<blocks_for(nz, 128), 128, 0, st>>>(d, g, gam, E, ip, f, dt, words, iter);
    else
        k_implicit_iter<HQ, HD, 0><<<blocks_for(nz, 128), 128, 0, st>>>(d, g, gam, E, ip, f, dt, words, iter);
}
template <bool HQ, bool HD>
static void jac_hd(const Dims& d, const DevGeom& g, double gam, const EmhdArgs& E, const ImplicitArgs& ip,
                   const ImpFields& f, double dt, double* jac, double* res, cudaStream_t st)
{
    const long long nz = (long long)d.nx1 * d.nx2 * d.nx3;
    if (ip.jacobian == 1)
        k_implicit_jacobian<HQ, HD, 1><<<blocks_for(nz, 128), 128, 0, st>>>(d, g, gam, E, ip, f, dt, jac, res);
    else
        k_implicit_jacobian<HQ, HD, 0><<<blocks_for(nz, 128), 128, 0, st>>>(d, g, gam, E, ip, f, dt, jac, res);
}
template <bool HQ, bool HD>
static void fix_hd(const Dims& d, const DevGeom& g, double gam, const EmhdArgs& E, const khb_fields& P,
                   const khb_fields& U, const double* sf, double* scratch, cudaStream_t st)
{
    k_fix_solve_avg<HQ, HD><<<blocks_for(d.N, 128), 128, 0, st>>>(d, P, sf, scratch);
    k_fix_solve_apply<HQ, HD><<<blocks_for(d.N, 128), 128, 0, st>>>(d, g, gam, E, P, U, sf, scratch);
}

#define KHB_DISPATCH_HD(E, FN, ...)                                  \
    do {                                                             \
        if ((E).conduction && (E).viscosity) FN<true, true>(__VA_ARGS__);   \
        else if ((E).conduction) FN<true, false>(__VA_ARGS__);       \
        else if ((E).viscosity) FN<false, true>(__VA_ARGS__);        \
        else FN<false, false>(__VA_ARGS__);                          \
    } while (0)

template <int DIR, bool HQ, bool HD>
static void flux_emhd_dir(int recon, const Dims& d, const DevGeom& g, const Phys& ph, const EmhdArgs& E,
                          const khb_fields& P, double* F, double* ctop, const Box& bx, cudaStream_t st)
{
    const unsigned nb = box_blocks(bx);
    switch (recon) {
    case RECON_DONOR: k_flux_emhd<DIR, RECON_DONOR, HQ, HD><<<nb, 128, 0, st>>>(d, g, ph, E, P, F, ctop, bx); break;
    case RECON_MC:    k_flux_emhd<DIR, RECON_MC, HQ, HD><<<nb, 128, 0, st>>>(d, g, ph, E, P, F, ctop, bx); break;
    case RECON_WENO5: k_flux_emhd<DIR, RECON_WENO5, HQ, HD><<<nb, 128, 0, st>>>(d, g, ph, E, P, F, ctop, bx); break;
    default:          k_flux_emhd<DIR, RECON_PPM, HQ, HD><<<nb, 128, 0, st>>>(d, g, ph, E, P, F, ctop, bx); break;
    }
}
template <bool HQ, bool HD>
static void flux_emhd_hd(int recon, int dir, const Dims& d, const DevGeom& g, const Phys& ph, const EmhdArgs& E,
                         const khb_fields& P, double* F, double* ctop, const Box& bx, cudaStream_t st)
{
    if (dir == 1) flux_emhd_dir<1, HQ, HD>(recon, d, g, ph, E, P, F, ctop, bx, st);
    else if (dir == 2) flux_emhd_dir<2, HQ, HD>(recon, d, g, ph, E, P, F, ctop, bx, st);
    else flux_emhd_dir<3, HQ, HD>(recon, d, g, ph, E, P, F, ctop, bx, st);
}
// Packages::MeshApplyFloors on the EMHD state over the interior (imex_step.cpp:269): the GRMHD floors
// in the fluid or drift frame (floors.cpp:215-229, floors_impl.hpp:77-125), which change the fluid
// primitives only, and the ceilings; the stage's final P -> U over the whole block forms U.  Floor
// bits into fflag.
__global__ void __launch_bounds__(128) k_emhd_floors(Dims d, DevGeom g, Phys ph, khb_fields P, int32_t* fflag)
{
    int k, j, i;
    long long c;
    if (!interior_zone(d, (long long)blockIdx.x * blockDim.x + threadIdx.x, k, j, i, c)) return;
    ZoneGeom G;
    load_zone_geom(g, j, i, G);
    double Pz[8], Uz[8] = {0., 0., 0., 0., 0., 0., 0., 0.};   // the fluid and drift frames leave U alone
#pragma unroll
    for (int p = 0; p < 8; ++p) Pz[p] = P.v[p][c];
    const long long cg = (long long)j*g.n1 + i;
    const Prescription& fl = floors_at(ph, g, j, i);
    double rf, uf;
    FourVec<double> D;
    const int ff = determine_floors<8>(G, fl, __ldg(g.floor_rho + cg), __ldg(g.floor_u + cg), ph.gam, Pz, rf, uf, D);
    if (ff) {
        apply_floors_frame<8>(G, ph.frame, ph.gam, Pz, Uz, rf, uf, 8, &D);
        apply_ceilings(G, fl, ph.gam, Pz);
#pragma unroll
        for (int p = 0; p < 5; ++p) P.v[p][c] = Pz[p];
    }
    fflag[c] = ff;
}

// EMHD::ApplyEMHDLimits / apply_instability_limits (emhd.cpp:399-428, emhd_limits.hpp:55-130) over
// the interior: q~ scaled so that |q| <= 1.07 rho cs^3, dP~ to the mirror and firehose bounds; the
// limit bits (1 q, 2 dP above, 4 dP below) into eflag.  The reference's closing p_to_u is the
// stage's final P -> U.
__global__ void __launch_bounds__(128) k_emhd_limits(Dims d, DevGeom g, double gam, EmhdArgs E, khb_fields P,
                                                    int32_t* eflag)
{
    int k, j, i;
    long long c;
    if (!interior_zone(d, (long long)blockIdx.x * blockDim.x + threadIdx.x, k, j, i, c)) return;
    CenterGeom G;
    load_center(g, j, i, G);
    double Pz[10];
    load10(P, c, Pz);
    const double rho = Pz[0], uu = Pz[1];
    const double qtilde = E.conduction ? Pz[8] : 0., dPtilde = E.viscosity ? Pz[9] : 0.;
    const double pg = (gam - 1.) * uu;
    const double Theta = pg / rho;
    const double cs = sqrt(gam * pg / (rho + (gam * uu)));
    FourVec<double> D;
    calc_4vecs<double, true>(G.gcov, G.gcon0[0], G.gcon0, Pz, D);
    const double bsq = kmax(dot4(D.bcon, D.bcov), SMALL);
    double q, dP;
    convert_q_dP(E, qtilde, dPtilde, rho, Theta, cs*cs, q, dP);
    int ef = 0;
    if (E.conduction) {
        const double qmax = 1.07 * rho * cs*cs*cs;
        const double max_frac = kmax(fabs(q) / qmax, 1.);
        if (fabs(q) / qmax > 1.) ef |= 1;
        P.v[8][c] = Pz[8] / max_frac;
    }
    if (E.viscosity) {
        const double dP_comp_ratio = kmax(pg - 2./3. * dP, SMALL) / kmax(pg + 1./3. * dP, SMALL);
        const double dP_plus = kmin(1.07 * 0.5 * bsq * dP_comp_ratio, 1.49 * pg);
        const double dP_minus = kmax(-1.07 * bsq, -2.99 * pg);
        if (dP > 0. && (dP / dP_plus > 1.)) ef |= 2;
        else if (dP < 0. && (dP / dP_minus > 1.)) ef |= 4;
        if (dP > 0.) P.v[9][c] = Pz[9] * (1. / kmax(dP / dP_plus, 1.));
        else P.v[9][c] = Pz[9] * (1. / kmax(dP / dP_minus, 1.));
    }
    eflag[c] = ef;
}

void LaunchEmhd::flux(int recon, int dir, const Dims& d, const DevGeom& g, const Phys& ph, const EmhdArgs& E,
                      const khb_fields& P, double* F, double* ctop, const int lo[3], const int cnt[3], cudaStream_t st)
{
    const Box bx = make_box(lo[0], lo[1], lo[2], cnt[0], cnt[1], cnt[2]);
    if (E.conduction && E.viscosity) flux_emhd_hd<true, true>(recon, dir, d, g, ph, E, P, F, ctop, bx, st);
    else if (E.conduction) flux_emhd_hd<true, false>(recon, dir, d, g, ph, E, P, F, ctop, bx, st);
    else if (E.viscosity) flux_emhd_hd<false, true>(recon, dir, d, g, ph, E, P, F, ctop, bx, st);
    else flux_emhd_hd<false, false>(recon, dir, d, g, ph, E, P, F, ctop, bx, st);
}
void LaunchEmhd::dudt(const Dims& d, const DevGeom& g, const Phys& ph, const EmhdArgs& E, double* const F[3],
                      double* const ctop[3], const khb_fields& Ps, const khb_fields& dUdt, int dtm,
                      unsigned long long* word, cudaStream_t st)
{
    const Box bx = make_box(d.is, d.js, d.ks, d.ie - d.is + 1, d.je - d.js + 1, d.ke - d.ks + 1);
    const unsigned nb = box_blocks(bx);
    if (E.conduction && E.viscosity)
        k_emhd_dudt<true, true><<<nb, 128, 0, st>>>(d, g, ph, E, F[0], F[1], F[2], ctop[0], ctop[1], ctop[2], Ps, dUdt, dtm, word, bx);
    else if (E.conduction)
        k_emhd_dudt<true, false><<<nb, 128, 0, st>>>(d, g, ph, E, F[0], F[1], F[2], ctop[0], ctop[1], ctop[2], Ps, dUdt, dtm, word, bx);
    else if (E.viscosity)
        k_emhd_dudt<false, true><<<nb, 128, 0, st>>>(d, g, ph, E, F[0], F[1], F[2], ctop[0], ctop[1], ctop[2], Ps, dUdt, dtm, word, bx);
    else
        k_emhd_dudt<false, false><<<nb, 128, 0, st>>>(d, g, ph, E, F[0], F[1], F[2], ctop[0], ctop[1], ctop[2], Ps, dUdt, dtm, word, bx);
}
void LaunchEmhd::imex_explicit(const Dims& d, const DevGeom& g, const khb_fields& Psub, const khb_fields& Usub,
                               const khb_fields& Ufull, const khb_fields& dUdt, const khb_fields& Pout,
                               const khb_fields& Uout, double g0, double g1, double bdt, cudaStream_t st)
{
    k_imex_explicit<<<blocks_for(d.N, 128), 128, 0, st>>>(d, g, Psub, Usub, Ufull, dUdt, Pout, Uout, g0, g1, bdt);
}

void LaunchEmhd::ptou(const Dims& d, const DevGeom& g, double gam, const EmhdArgs& E, const khb_fields& P,
                      const khb_fields& U, cudaStream_t st)
{
    k_emhd_ptou<<<blocks_for(d.N, 128), 128, 0, st>>>(d, g, gam, E, P, U);
}

void LaunchEmhd::add_source(const Dims& d, const DevGeom& g, const double* conn, double gam, const EmhdArgs& E,
                            const Phys& ph, const khb_fields& P, double* tmp, const khb_fields& dUdt, cudaStream_t st)
{
    const int il = d.is - 1, ih = d.ie + 1;
    const int jl = (d.ndim > 1) ? d.js - 1 : d.js, jh = (d.ndim > 1) ? d.je + 1 : d.je;
    const int kl = (d.ndim > 2) ? d.ks - 1 : d.ks, kh = (d.ndim > 2) ? d.ke + 1 : d.ke;
    const int ci = ih - il + 1, cj = jh - jl + 1, ck = kh - kl + 1;
    k_emhd_temps<<<blocks_for((long long)ci * cj * ck, 128), 128, 0, st>>>(d, g, gam, P, tmp, il, jl, kl, ci, cj, ck);
    const long long nz = (long long)d.nx1 * d.nx2 * d.nx3;
    k_emhd_sources<<<blocks_for(nz, 128), 128, 0, st>>>(d, g, conn, gam, E, ph, P, tmp, dUdt);
}

void LaunchEmhd::implicit_iter(const Dims& d, const DevGeom& g, double gam, const EmhdArgs& E, const ImplicitArgs& ip,
                               const ImpFields& f, double dt, unsigned long long* words, int iter, cudaStream_t st)
{
    KHB_DISPATCH_HD(E, iter_hd, d, g, gam, E, ip, f, dt, words, iter, st);
}

void LaunchEmhd::implicit_jacobian(const Dims& d, const DevGeom& g, double gam, const EmhdArgs& E,
                                   const ImplicitArgs& ip, const ImpFields& f, double dt, double* jac, double* res,
                                   cudaStream_t st)
{
    KHB_DISPATCH_HD(E, jac_hd, d, g, gam, E, ip, f, dt, jac, res, st);
}

void LaunchEmhd::floors(const Dims& d, const DevGeom& g, const Phys& ph, const khb_fields& P, int32_t* fflag,
                        cudaStream_t st)
{
    const long long nz = (long long)d.nx1 * d.nx2 * d.nx3;
    k_emhd_floors<<<blocks_for(nz, 128), 128, 0, st>>>(d, g, ph, P, fflag);
}

void LaunchEmhd::limits(const Dims& d, const DevGeom& g, double gam, const EmhdArgs& E, const khb_fields& P,
                        int32_t* eflag, cudaStream_t st)
{
    const long long nz = (long long)d.nx1 * d.nx2 * d.nx3;
    k_emhd_limits<<<blocks_for(nz, 128), 128, 0, st>>>(d, g, gam, E, P, eflag);
}

void LaunchEmhd::fix_solve(const Dims& d, const DevGeom& g, double gam, const EmhdArgs& E, const khb_fields& P,
                           const khb_fields& U, const double* solve_fail, double* scratch, cudaStream_t st)
{
    KHB_DISPATCH_HD(E, fix_hd, d, g, gam, E, P, U, solve_fail, scratch, st);
}

} // namespace khb

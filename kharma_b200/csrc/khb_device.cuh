// khb_device.cuh -- device-side GRMHD functions for the per-step kernels (sm_100a).
//
// These restate KHARMA's device functions for one zone or face at a time.  The flux-side
// functions are templated on the arithmetic type R so that the same code serves the FP64
// path and the FP32-flux form; the zone-side functions (inversion, floors, P->U) are FP64.
// Evaluation order follows the reference expression by expression so the FP64 path agrees
// with a reference build to rounding level.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "khb_types.cuh"

namespace khb {

// Kokkos::max/min semantics, as used through m::max/m::min in the reference
template <typename R> __device__ __forceinline__ R kmax(R a, R b) { return (a < b) ? b : a; }
template <typename R> __device__ __forceinline__ R kmin(R a, R b) { return (b < a) ? b : a; }
template <typename R> __device__ __forceinline__ R kclip(R n, R lo, R hi) { return kmin(kmax(lo, n), hi); }

__device__ __forceinline__ float  dsqrt(float x)  { return sqrtf(x); }
__device__ __forceinline__ double dsqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float  dabs(float x)   { return fabsf(x); }
__device__ __forceinline__ double dabs(double x)  { return fabs(x); }

enum { RECON_DONOR = 0, RECON_MC = 1, RECON_WENO5 = 2, RECON_PPM = 3,
       // the further schemes of flux/reconstruction.hpp, one kernel variant that picks the scheme
       // at run time from Phys::recon_extra
       RECON_EXTRA = 4,
       // WENO5 with its lowered variants or the floor fallback (a separate kernel variant, so that
       // plain WENO5 keeps its code)
       RECON_WENO5X = 5 };
enum { EX_LINEAR_VL = 1, EX_WENO5_LINEAR = 2, EX_PPMX = 3, EX_MP5 = 4 };

// ------------------------------------------------------------------ reconstruction
// flux/reconstruction.hpp:52-56
template <typename R>
__device__ __forceinline__ R mc_lim(R dm, R dp)
{
    const R r = (dabs(dp) > R(0) ? dm/dp : R(2));
    return kmax(R(0), kmin(R(2), kmin(R(2)*r, R(0.5)*(R(1)+r))));
}

// Value at the right face of a zone with stencil x1..x5 (reconstruct_right, :114-204, :351-394)
template <int RECON, typename R>
__device__ __forceinline__ R recon_right(R x1, R x2, R x3, R x4, R x5)
{
    if (RECON == RECON_DONOR) {
        return x3;
    } else if (RECON == RECON_MC) {
        return x3 + R(0.5)*(mc_lim(x3 - x2, x4 - x3)*(x4 - x3));
    } else if (RECON == RECON_WENO5) {
        // WENO5-JS (T07 A18, S11 8-9), reconstruction.hpp:183-204.  Weights are always formed in
        // FP64: with EPS = 1e-26 the squared denominators underflow FP32.
        const double y1 = x1, y2 = x2, y3 = x3, y4 = x4, y5 = x5;
        double c1, c2, b0, b1, b2;
        c1 = y1 - 2.*y2 + y3; c2 = y1 - 4.*y2 + 3.*y3;
        b0 = (13./12.)*c1*c1 + (1./4.)*c2*c2;
        c1 = y2 - 2.*y3 + y4; c2 = y4 - y2;
        b1 = (13./12.)*c1*c1 + (1./4.)*c2*c2;
        c1 = y3 - 2.*y4 + y5; c2 = y5 - 4.*y4 + 3.*y3;
        b2 = (13./12.)*c1*c1 + (1./4.)*c2*c2;
        double d0 = 1.e-26 + b0, d1 = 1.e-26 + b1, d2 = 1.e-26 + b2;
        d0 *= d0; d1 *= d1; d2 *= d2;
        const double w0 = (1./16.)/d0, w1 = (5./8.)/d1, w2 = (5./16.)/d2;
        const double W = w0 + w1 + w2;
        return (R)(((3./8.)*y1 - (5./4.)*y2 + (15./8.)*y3)*(w0 / W) +
                   ((-1./8.)*y2 + (3./4.)*y3 + (3./8.)*y4)*(w1 / W) +
                   ((3./8.)*y3 + (3./4.)*y4 - (1./8.)*y5)*(w2 / W));
    } else {
        // PPM (Colella & Woodward with CS limiters), reconstruction.hpp:351-381: qrv
        R qlv = (R(7)*(x3 + x2) - (x1 + x4))/R(12);
        R qrv = (R(7)*(x3 + x4) - (x2 + x5))/R(12);
        qlv = kmax(qlv, kmin(x3, x2));
        qlv = kmin(qlv, kmax(x3, x2));
        qrv = kmax(qrv, kmin(x3, x4));
        qrv = kmin(qrv, kmax(x3, x4));
        const R qc = qrv - x3, qd = qlv - x3;
        if ((qc*qd) >= R(0)) return x3;
        if (dabs(qc) >= R(2)*dabs(qd)) qrv = x3 - R(2)*qd;
        return qrv;
    }
}
// Value at the left face of a zone (reconstruct_left, :114-204, :351-394)
template <int RECON, typename R>
__device__ __forceinline__ R recon_left(R x1, R x2, R x3, R x4, R x5)
{
    if (RECON == RECON_DONOR) {
        return x3;
    } else if (RECON == RECON_MC) {
        return x3 - R(0.5)*(mc_lim(x3 - x2, x4 - x3)*(x4 - x3));
    } else if (RECON == RECON_WENO5) {
        const double y1 = x1, y2 = x2, y3 = x3, y4 = x4, y5 = x5;
        double c1, c2, b0, b1, b2;
        c1 = y1 - 2.*y2 + y3; c2 = y1 - 4.*y2 + 3.*y3;
        b0 = (13./12.)*c1*c1 + (1./4.)*c2*c2;
        c1 = y2 - 2.*y3 + y4; c2 = y4 - y2;
        b1 = (13./12.)*c1*c1 + (1./4.)*c2*c2;
        c1 = y3 - 2.*y4 + y5; c2 = y5 - 4.*y4 + 3.*y3;
        b2 = (13./12.)*c1*c1 + (1./4.)*c2*c2;
        double d0 = 1.e-26 + b0, d1 = 1.e-26 + b1, d2 = 1.e-26 + b2;
        d0 *= d0; d1 *= d1; d2 *= d2;
        const double w0 = (1./16.)/d2, w1 = (5./8.)/d1, w2 = (5./16.)/d0;
        const double W = w0 + w1 + w2;
        return (R)(((3./8.)*y5 - (5./4.)*y4 + (15./8.)*y3)*(w0 / W) +
                   ((-1./8.)*y4 + (3./4.)*y3 + (3./8.)*y2)*(w1 / W) +
                   ((3./8.)*y3 + (3./4.)*y2 - (1./8.)*y1)*(w2 / W));
    } else {
        R qlv = (R(7)*(x3 + x2) - (x1 + x4))/R(12);
        R qrv = (R(7)*(x3 + x4) - (x2 + x5))/R(12);
        qlv = kmax(qlv, kmin(x3, x2));
        qlv = kmin(qlv, kmax(x3, x2));
        qrv = kmax(qrv, kmin(x3, x4));
        qrv = kmin(qrv, kmax(x3, x4));
        const R qc = qrv - x3, qd = qlv - x3;
        if ((qc*qd) >= R(0)) return x3;
        if (dabs(qd) >= R(2)*dabs(qc)) qlv = x3 - R(2)*qc;
        return qlv;
    }
}

// ------------------------------------------------------------------ further reconstructions
__device__ __forceinline__ double kcopysign(double a, double b) { return ::copysign(a, b); }
__device__ __forceinline__ float kcopysign(float a, float b) { return copysignf(a, b); }
// MC slope with a limiter coefficient (reconstruction.hpp:58-63)
template <typename R>
__device__ __forceinline__ R mc_alpha(R dm, R dp, R alpha)
{
    const R dc = (dm * dp > R(0)) ? R(0.5) * (dm + dp) : R(0);
    return kcopysign(kmin(dabs(dc), alpha * kmin(dabs(dm), dabs(dp))), dc);
}

template <typename R>
__device__ __forceinline__ R minmod_r(R a, R b) { return (a * b > R(0)) ? ((dabs(a) < dabs(b)) ? a : b) : R(0); }

// Linearized WENO5 (reconstruction.hpp:209-268): both faces of the zone x3; formed in FP64 (its
// epsilon, 1e-100, is below FP32's range)
__device__ __forceinline__ void weno5_linear_lr(double x1, double x2, double x3, double x4, double x5,
                                                double& lout, double& rout)
{
    const double a00 = 1.0 / 3.0, a01 = -7.0 / 6.0, a02 = 11.0 / 6.0;
    const double a10 = -1.0 / 6.0, a11 = 5.0 / 6.0, a12 = 1.0 / 3.0;
    const double a20 = 1.0 / 3.0, a21 = 5.0 / 6.0, a22 = -1.0 / 6.0;
    const double g0 = 0.1, g1 = 0.6, g2 = 0.3;
    const double eps = 1e-100, tt = 13.0 / 3.0;
    double a = x1 - 2 * x2 + x3;
    double b = x1 - 4.0 * x2 + 3.0 * x3;
    double beta0 = tt * a * a + b * b + eps;
    a = x2 - 2.0 * x3 + x4;
    b = x4 - x2;
    double beta1 = tt * a * a + b * b + eps;
    a = x3 - 2.0 * x4 + x5;
    b = x5 - 4.0 * x4 + 3.0 * x3;
    double beta2 = tt * a * a + b * b + eps;
    const double tau5 = fabs(beta2 - beta0);
    beta0 = (beta0 + tau5) / beta0;
    beta1 = (beta1 + tau5) / beta1;
    beta2 = (beta2 + tau5) / beta2;
    double w0 = g0 * beta0 + eps, w1 = g1 * beta1 + eps, w2 = g2 * beta2 + eps;
    double wsum = 1.0 / (w0 + w1 + w2);
    rout = w0 * (a00 * x1 + a01 * x2 + a02 * x3);
    rout += w1 * (a10 * x2 + a11 * x3 + a12 * x4);
    rout += w2 * (a20 * x3 + a21 * x4 + a22 * x5);
    rout *= wsum;
    const double alpha_r = 3.0 * wsum * w0 * w1 * w2 / (g2 * w0 * w1 + g1 * w0 * w2 + g0 * w1 * w2) + eps;
    w0 = g0 * beta2 + eps; w1 = g1 * beta1 + eps; w2 = g2 * beta0 + eps;
    wsum = 1.0 / (w0 + w1 + w2);
    lout = w0 * (a00 * x5 + a01 * x4 + a02 * x3);
    lout += w1 * (a10 * x4 + a11 * x3 + a12 * x2);
    lout += w2 * (a20 * x3 + a21 * x2 + a22 * x1);
    lout *= wsum;
    const double alpha_l = 3.0 * wsum * w0 * w1 * w2 / (g2 * w0 * w1 + g1 * w0 * w2 + g0 * w1 * w2) + eps;
    const double dq = mc_alpha<double>(x3 - x2, x4 - x3, 2.0);
    const double alpha_lin = 2.0 * alpha_r * alpha_l / (alpha_r + alpha_l);
    rout = alpha_lin * rout + (1.0 - alpha_lin) * (x3 + 0.5 * dq);
    lout = alpha_lin * lout + (1.0 - alpha_lin) * (x3 - 0.5 * dq);
}

// MP5 (Suresh & Huynh 1997) as reconstruction.hpp:284-325 has it: the value at the face between
// Fj and Fjp1
template <typename R>
__device__ __forceinline__ R mp5_subcalc(R Fjm2, R Fjm1, R Fj, R Fjp1, R Fjp2)
{
    const R alpha = R(4.0), epsm = R(1.e-12);
    R f = R(2.0) * Fjm2 - R(13.0) * Fjm1 + R(47.0) * Fj + R(27.0) * Fjp1 - R(3.0) * Fjp2;
    f /= R(60.0);
    const R fMP = Fj + minmod_r(Fjp1 - Fj, alpha * (Fj - Fjm1));
    if ((f - Fj) * (f - fMP) <= epsm) return f;
    const R d2m = Fjm2 + Fj - R(2.0) * Fjm1;
    const R d2 = Fjm1 + Fjp1 - R(2.0) * Fj;
    const R d2p = Fj + Fjp2 - R(2.0) * Fjp1;
    R scrh1 = minmod_r(R(4.0) * d2 - d2p, R(4.0) * d2p - d2);
    R scrh2 = minmod_r(d2, d2p);
    const R dMMp = minmod_r(scrh1, scrh2);
    scrh1 = minmod_r(R(4.0) * d2m - d2, R(4.0) * d2 - d2m);
    scrh2 = minmod_r(d2, d2m);
    const R dMMm = minmod_r(scrh1, scrh2);
    const R fUL = Fj + alpha * (Fj - Fjm1);
    const R fAV = R(0.5) * (Fj + Fjp1);
    const R fMD = fAV - R(0.5) * dMMp;
    const R fLC = R(0.5) * (R(3.0) * Fj - Fjm1) + R(4.0 / 3.0) * dMMm;
    scrh1 = kmin(kmin(Fj, Fjp1), fMD);
    scrh2 = kmin(kmin(Fj, fUL), fLC);
    const R mn = kmax(scrh1, scrh2);
    scrh1 = kmax(kmax(Fj, Fjp1), fMD);
    scrh2 = kmax(kmax(Fj, fUL), fLC);
    const R mx = kmin(scrh1, scrh2);
    return f + minmod_r(mn - f, mx - f);       // Median(f, mn, mx)
}

// PPMX, extremum-preserving PPM with Colella & Sekora limiters (reconstruction.hpp:403-495)
template <typename R>
__device__ __forceinline__ R sgn_r(R x) { return (x < R(0)) ? R(-1) : R(1); }
template <typename R>
__device__ __forceinline__ void ppmx_lr(R q_im2, R q_im1, R q_i, R q_ip1, R q_ip2, R& qlv, R& qrv)
{
    qlv = (R(7.) * (q_i + q_im1) - (q_im2 + q_ip1)) / R(12.0);
    qrv = (R(7.) * (q_i + q_ip1) - (q_im1 + q_ip2)) / R(12.0);
    R d2qc = R(3.0) * ((q_im1 + q_i) - R(2.0) * qlv);
    R d2ql = (q_im2 + q_i) - R(2.0) * q_im1;
    R d2qr = (q_im1 + q_ip1) - R(2.0) * q_i;
    R d2qlim = R(0.0);
    R lim_slope = kmin(dabs(d2ql), dabs(d2qr));
    if (d2qc > R(0) && d2ql > R(0) && d2qr > R(0)) d2qlim = sgn_r(d2qc) * kmin(R(1.25) * lim_slope, dabs(d2qc));
    if (d2qc < R(0) && d2ql < R(0) && d2qr < R(0)) d2qlim = sgn_r(d2qc) * kmin(R(1.25) * lim_slope, dabs(d2qc));
    if (((q_im1 - qlv) * (q_i - qlv)) > R(0)) qlv = R(0.5) * (q_i + q_im1) - d2qlim / R(6.0);
    d2qc = R(3.0) * ((q_i + q_ip1) - R(2.0) * qrv);
    d2ql = d2qr;
    d2qr = (q_i + q_ip2) - R(2.0) * q_ip1;
    d2qlim = R(0.0);
    lim_slope = kmin(dabs(d2ql), dabs(d2qr));
    if (d2qc > R(0) && d2ql > R(0) && d2qr > R(0)) d2qlim = sgn_r(d2qc) * kmin(R(1.25) * lim_slope, dabs(d2qc));
    if (d2qc < R(0) && d2ql < R(0) && d2qr < R(0)) d2qlim = sgn_r(d2qc) * kmin(R(1.25) * lim_slope, dabs(d2qc));
    if (((q_i - qrv) * (q_ip1 - qrv)) > R(0)) qrv = R(0.5) * (q_i + q_ip1) - d2qlim / R(6.0);
    const R qa = (qrv - q_i) * (q_i - qlv);
    const R qb = (q_im1 - q_i) * (q_i - q_ip1);
    if (qa <= R(0) || qb <= R(0)) {
        const R d2q = R(6.0) * (qlv + qrv - R(2.0) * q_i);
        const R c = (q_im1 + q_ip1) - R(2.0) * q_i;
        const R l = (q_im2 + q_i) - R(2.0) * q_im1;
        const R r = (q_i + q_ip2) - R(2.0) * q_ip1;
        d2qlim = R(0.0);
        lim_slope = kmin(dabs(l), dabs(r));
        lim_slope = kmin(dabs(c), lim_slope);
        if (c > R(0) && l > R(0) && r > R(0) && d2q > R(0)) d2qlim = sgn_r(d2q) * kmin(R(1.25) * lim_slope, dabs(d2q));
        if (c < R(0) && l < R(0) && r < R(0) && d2q < R(0)) d2qlim = sgn_r(d2q) * kmin(R(1.25) * lim_slope, dabs(d2q));
        R rho = R(0.0);
        if (dabs(d2q) > R(1.0e-12) * kmax(dabs(q_im1), kmax(dabs(q_i), dabs(q_ip1)))) rho = d2qlim / d2q;
        qlv = q_i + (qlv - q_i) * rho;
        qrv = q_i + (qrv - q_i) * rho;
    } else {
        const R qc = qrv - q_i, qd = qlv - q_i;
        if (dabs(qc) >= R(2.0) * dabs(qd)) qrv = q_i - R(2.0) * qd;
        if (dabs(qd) >= R(2.0) * dabs(qc)) qlv = q_i - R(2.0) * qc;
    }
}

// Right / left face value of zone x3 by the scheme `ex` (EX_*); linear van Leer is the simplified
// VL limiter of Parthenon's PiecewiseLinear on a uniform grid (2 dql dqr / (dql + dqr) where the
// one-sided differences agree in sign)
template <typename R>
__device__ __forceinline__ R recon_extra(int ex, bool right, R x1, R x2, R x3, R x4, R x5)
{
    if (ex == EX_LINEAR_VL) {
        const R dql = x3 - x2, dqr = x4 - x3;
        const R dq2 = dql * dqr;
        const R dqm = (dq2 > R(0)) ? R(2.0) * dq2 / (dql + dqr) : R(0);
        return right ? x3 + R(0.5) * dqm : x3 - R(0.5) * dqm;
    } else if (ex == EX_WENO5_LINEAR) {
        double l, r;
        weno5_linear_lr(x1, x2, x3, x4, x5, l, r);
        return (R)(right ? r : l);
    } else if (ex == EX_PPMX) {
        R l, r;
        ppmx_lr<R>(x1, x2, x3, x4, x5, l, r);
        return right ? r : l;
    } else {
        return right ? mp5_subcalc<R>(x1, x2, x3, x4, x5) : mp5_subcalc<R>(x5, x4, x3, x2, x1);
    }
}

// ------------------------------------------------------------------ geometry at one point
// Full covariant metric, the inverse-metric entries the flux path uses, and sqrt(-g).
template <typename R>
struct FaceGeom {
    R gcov[4][4];
    R gcon00, gcon0[4];   // gcon[0][mu]
    R gcon_dd;            // gcon[dir][dir]
    R gdet;
};

// 4-vectors (types.hpp:90-95)
template <typename R>
struct FourVec { R ucon[4], ucov[4], bcon[4], bcov[4]; };

template <typename R>
__device__ __forceinline__ R dot4(const R* a, const R* b)
{
    return a[0]*b[0] + a[1]*b[1] + a[2]*b[2] + a[3]*b[3];
}

// gr_coordinates.hpp:227-232 (lower with the full gcov)
template <typename R>
__device__ __forceinline__ void lower4(const R g[4][4], const R* vcon, R* vcov)
{
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
        R s = R(0);
#pragma unroll
        for (int nu = 0; nu < 4; ++nu) s += g[mu][nu] * vcon[nu];
        vcov[mu] = s;
    }
}

// grmhd_functions.hpp:121-133
template <typename R>
__device__ __forceinline__ R lorentz(const R g[4][4], R u1, R u2, R u3)
{
    const R qsq = g[1][1] * u1 * u1 + g[2][2] * u2 * u2 + g[3][3] * u3 * u3 +
                  R(2.) * (g[1][2] * u1 * u2 + g[1][3] * u1 * u3 + g[2][3] * u2 * u3);
    return dsqrt(R(1.) + qsq);
}

// grmhd_functions.hpp:225-246.  P = {rho, u, u1, u2, u3, B1, B2, B3}
template <typename R, bool HAS_B>
__device__ __forceinline__ void calc_4vecs(const R g[4][4], R gcon00, const R* gcon0, const R* P, FourVec<R>& D)
{
    const R gamma = lorentz(g, P[2], P[3], P[4]);
    const R alpha = R(1.) / dsqrt(-gcon00);
    D.ucon[0] = gamma / alpha;
#pragma unroll
    for (int v = 0; v < 3; ++v) D.ucon[v+1] = P[2 + v] - gamma * alpha * gcon0[v+1];
    lower4(g, D.ucon, D.ucov);
    if (HAS_B) {
        R b0 = R(0);
#pragma unroll
        for (int v = 0; v < 3; ++v) b0 += P[5 + v] * D.ucov[v+1];
        D.bcon[0] = b0;
#pragma unroll
        for (int v = 0; v < 3; ++v) D.bcon[v+1] = (P[5 + v] + b0 * D.ucon[v+1]) / D.ucon[0];
        lower4(g, D.bcon, D.bcov);
    } else {
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) D.bcon[mu] = D.bcov[mu] = R(0);
    }
}

// One row T^dir_mu of the MHD (or hydro) stress tensor, grmhd_functions.hpp:51-60, 142-155
template <typename R, bool HAS_B>
__device__ __forceinline__ void calc_tensor(R rho, R u, R pgas, const FourVec<R>& D, int dir, R T[4])
{
    if (HAS_B) {
        const R bsq = dot4(D.bcon, D.bcov);
        const R eta = pgas + rho + u + bsq;
        const R ptot = pgas + R(0.5) * bsq;
#pragma unroll
        for (int mu = 0; mu < 4; ++mu)
            T[mu] = eta * D.ucon[dir] * D.ucov[mu] + ptot * R(dir == mu) - D.bcon[dir] * D.bcov[mu];
    } else {
        const R eta = pgas + rho + u;
#pragma unroll
        for (int mu = 0; mu < 4; ++mu)
            T[mu] = eta * D.ucon[dir] * D.ucov[mu] + pgas * R(dir == mu);
    }
}

// flux_functions.hpp:116-178: conserved variables (dir = 0) or fluxes along dir
template <typename R, int NV>
__device__ __forceinline__ void prim_to_flux(const R* P, const FourVec<R>& D, R gam, R gdet, int dir, R* flux)
{
    constexpr bool HAS_B = NV > 5;
    flux[0] = P[0] * D.ucon[dir] * gdet;
    R T[4];
    calc_tensor<R, HAS_B>(P[0], P[1], (gam - R(1)) * P[1], D, dir, T);
    flux[1] = T[0] * gdet + flux[0];
    flux[2] = T[1] * gdet;
    flux[3] = T[2] * gdet;
    flux[4] = T[3] * gdet;
    if (HAS_B) {
        if (dir == 0) {
#pragma unroll
            for (int v = 0; v < 3; ++v) flux[5 + v] = P[5 + v] * gdet;
        } else {
#pragma unroll
            for (int v = 0; v < 3; ++v) flux[5 + v] = (D.bcon[v+1] * D.ucon[dir] - D.bcon[dir] * D.ucon[v+1]) * gdet;
        }
    }
}

// The fast-magnetosonic signal speeds along dir for a given cms2 (flux_functions.hpp:411-438)
template <typename R>
__device__ __forceinline__ void vchar_speeds(R cms2, const FourVec<R>& D, R gcon00, R gcon0d, R gcondd, int dir,
                                             R& cmax, R& cmin)
{
    const R Asq = gcondd, Bsq = gcon00, AB = gcon0d;
    const R Au = D.ucon[dir], Bu = D.ucon[0];
    const R A  = Bu*Bu - (Bsq + Bu*Bu) * cms2;
    const R Bq = R(2.) * (Au*Bu - (AB + Au*Bu) * cms2);
    const R Cq = Au*Au - (Asq + Au*Au) * cms2;
    const R discr = dsqrt(kmax(Bq * Bq - R(4.) * A * Cq, R(0)));
    const R vp = -(-Bq + discr) / (R(2.) * A);
    const R vm = -(-Bq - discr) / (R(2.) * A);
    cmax = kmax(vp, vm);
    cmin = kmin(vp, vm);
}

// flux_functions.hpp:368-439.  The reference discards its clip() results (:378, :409), so no
// clipping happens here either.  With A_mu = delta^dir_mu and B_mu = delta^0_mu the raised
// vectors and their contractions reduce exactly to single metric entries.
template <typename R, bool HAS_B>
__device__ __forceinline__ void vchar(const R* P, const FourVec<R>& D, R gam, R gcon00, R gcon0d, R gcondd,
                                      int dir, R& cmax, R& cmin)
{
    const R ef  = P[0] + gam * P[1];
    const R cs2 = gam * (gam - R(1)) * P[1] / ef;
    R cms2;
    if (HAS_B) {
        const R bsq = dot4(D.bcon, D.bcov);
        const R va2 = bsq / (bsq + ef);
        cms2 = cs2 + va2 - cs2 * va2;
    } else {
        cms2 = cs2;
    }
    vchar_speeds<R>(cms2, D, gcon00, gcon0d, gcondd, dir, cmax, cmin);
}

// ------------------------------------------------------------------ 1D_W inversion (FP64)
enum Status { ST_SUCCESS = 0, ST_NEG_INPUT, ST_MAX_ITER, ST_BAD_UT, ST_BAD_GAMMA, ST_NEG_RHO, ST_NEG_U, ST_NEG_RHOU };

// onedw.hpp:49-67
__device__ __forceinline__ double lorentz_calc_w(double Bsq, double D, double QdB, double Qtsq, double Wp)
{
    const double QdBsq = QdB * QdB;
    const double W = Wp + D;
    const double W2 = W * W;
    const double WB = W + Bsq;
    const double utsq = -((W + WB) * QdBsq + W2 * Qtsq) / (QdBsq * (W + WB) + W2 * (Qtsq - WB * WB));
    if (utsq < -1.e-15 || utsq > 1.e7) return -1.;
    return sqrt(1. + fabs(utsq));
}
// onedw.hpp:72-84
__device__ __forceinline__ double err_eqn(double gam, double Bsq, double D, double Ep, double QdB, double Qtsq,
                                          double Wp, int& eflag)
{
    const double W = Wp + D;
    const double gamma = lorentz_calc_w(Bsq, D, QdB, Qtsq, Wp);
    if (gamma < 1) eflag = ST_BAD_UT;
    const double w = W / (gamma*gamma);
    const double rho = D / gamma;
    const double p = (w - rho) * (gam - 1) / gam;
    return -Ep + Wp - p + 0.5 * Bsq + 0.5 * (Bsq * Qtsq - QdB * QdB) / ((Bsq + W)*(Bsq + W));
}

// The same residual with one division and one reciprocal square root in place of four divisions
// and a square root: 1/gamma = rsqrt(1 + |utsq|), rho = D/gamma and w = W/gamma^2 by products,
// (gam-1)/gam from the caller (gfac), (Bsq + W)^2 = WB^2.  Equal to err_eqn up to rounding (a few
// ulp); used by the FP32-flux form's inversion, which has no bitwise contract with the reference.
__device__ __forceinline__ double err_eqn_fast(double gfac, double Bsq, double D, double Ep, double QdB, double Qtsq,
                                               double Wp, int& eflag)
{
    const double QdBsq = QdB * QdB;
    const double W = Wp + D;
    const double W2 = W * W;
    const double WB = W + Bsq;
    const double utsq = -((W + WB) * QdBsq + W2 * Qtsq) / (QdBsq * (W + WB) + W2 * (Qtsq - WB * WB));
    double ig;                                   // 1/gamma; gamma = -1 for an unphysical utsq
    if (utsq < -1.e-15 || utsq > 1.e7) { ig = -1.; eflag = ST_BAD_UT; }
    else ig = rsqrt(1. + fabs(utsq));
    const double w = W * (ig * ig);
    const double rho = D * ig;
    const double p = (w - rho) * gfac;
    return -Ep + Wp - p + 0.5 * Bsq + 0.5 * (Bsq * Qtsq - QdBsq) / (WB * WB);
}

// Zone-centre geometry for the inversion, floors and P->U
struct ZoneGeom {
    double gcov[4][4];
    double gcon[4][4];
    double gdet;
};

__device__ __forceinline__ void raise4(const ZoneGeom& G, const double* vcov, double* vcon)
{
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) {
        double s = 0.;
#pragma unroll
        for (int nu = 0; nu < 4; ++nu) s += G.gcon[mu][nu] * vcov[nu];
        vcon[mu] = s;
    }
}

// onedw.hpp:89-233.  U: conserved zone values; P: guess on entry, updated only on success.
// The iteration count is bounded by max_iterations.  FAST (the FP32-flux form): the residual by
// err_eqn_fast and the convergence tests |dW| < tol |Wp|, |err| < tol |Wp| without the divisions;
// FP64 throughout, equal to the plain form up to rounding.
template <int NV, bool FAST = false>
__device__ int u_to_p_onedw(const ZoneGeom& G, double gam, const double* U, double* P, int max_iterations, double tol)
{
    if (U[0] <= 0.) return ST_NEG_INPUT;
    const double alpha = 1./sqrt(-G.gcon[0][0]);
    const double gdet = G.gdet;
    const double a_over_g = alpha / gdet;
    const double D = U[0] * a_over_g;
    double Bcon[4] = {0., 0., 0., 0.};
    if (NV > 5) {
        Bcon[1] = U[5] * a_over_g;
        Bcon[2] = U[6] * a_over_g;
        Bcon[3] = U[7] * a_over_g;
    }
    const double Qcov[4] = {(U[1] - U[0]) * a_over_g, U[2] * a_over_g, U[3] * a_over_g, U[4] * a_over_g};
    const double ncov[4] = {-alpha, 0., 0., 0.};
    double Bcov[4], Qcon[4], ncon[4];
    lower4(G.gcov, Bcon, Bcov);
    raise4(G, Qcov, Qcon);
    raise4(G, ncov, ncon);
    const double Bsq = dot4(Bcon, Bcov);
    const double QdB = dot4(Bcon, Qcov);
    const double Qdotn = dot4(Qcon, ncov);
    double Qtcon[4];
#pragma unroll
    for (int mu = 0; mu < 4; ++mu) Qtcon[mu] = Qcon[mu] + ncon[mu] * Qdotn;
    const double Qtsq = dot4(Qcon, Qcov) + Qdotn*Qdotn;
    const double Ep = -Qdotn - D;
    int eflag = ST_SUCCESS;
    const double gfac = (gam - 1) / gam;
    auto residual = [&](double Wq) {
        return FAST ? err_eqn_fast(gfac, Bsq, D, Ep, QdB, Qtsq, Wq, eflag) : err_eqn(gam, Bsq, D, Ep, QdB, Qtsq, Wq, eflag);
    };
    double Wp, err;
    {
        const double gamma = lorentz(G.gcov, P[2], P[3], P[4]);
        if (gamma < 1) return ST_BAD_UT;
        const double rho = P[0], u = P[1];
        Wp = (rho + u + (gam - 1) * u) * gamma * gamma - rho * gamma;
        err = residual(Wp);
    }
    double dW;
    {
        const double Wpm = (1. - 1.e-5) * Wp;
        const double h = Wp - Wpm;
        const double Wpp = Wp + h;
        const double errm = residual(Wpm);
        const double errp = residual(Wpp);
        if (FAST) {
            const double idedW = (Wpp - Wpm) / (errp - errm);
            const double dedW2 = (errp - 2. * err + errm) / (h*h);
            const double f = kclip(0.5 * err * dedW2 * (idedW*idedW), -0.3, 0.3);
            dW = kclip(-err * idedW / (1. - f), -0.5*Wp, 2.0*Wp);
        } else {
            const double dedW = (errp - errm) / (Wpp - Wpm);
            const double dedW2 = (errp - 2. * err + errm) / (h*h);
            const double f = kclip(0.5 * err * dedW2 / (dedW*dedW), -0.3, 0.3);
            dW = kclip(-err / dedW / (1. - f), -0.5*Wp, 2.0*Wp);
        }
    }
    double Wp1 = Wp;
    double err1 = err;
    Wp += dW;
    err = residual(Wp);
    int iter = 0;
    for (iter = 0; iter < max_iterations; iter++) {
        dW = kclip((Wp1 - Wp) * err / (err - err1), -0.5*Wp, 2.0*Wp);
        Wp1 = Wp;
        err1 = err;
        Wp += dW;
        if (FAST ? fabs(dW) < tol * fabs(Wp) : fabs(dW / Wp) < tol) break;
        err = residual(Wp);
        if (FAST ? fabs(err) < tol * fabs(Wp) : fabs(err / Wp) < tol) break;
    }
    if (iter == max_iterations) return ST_MAX_ITER;
    const double W = Wp + D;
    if (FAST) {
        // gamma = 1/ig with ig = rsqrt(1 + |utsq|), as in err_eqn_fast
        const double QdBsq = QdB * QdB, W2 = W * W, WB = W + Bsq;
        const double utsq = -((W + WB) * QdBsq + W2 * Qtsq) / (QdBsq * (W + WB) + W2 * (Qtsq - WB * WB));
        if (utsq < -1.e-15 || utsq > 1.e7) return ST_BAD_UT;
        const double ig = rsqrt(1. + fabs(utsq));
        const double rho = D * ig;
        const double w = W * (ig * ig);
        const double p = (w - rho) * gfac;
        const double u = w - (rho + p);
        if (rho < 0 && u < 0) return ST_NEG_RHOU;
        else if (rho < 0) return ST_NEG_RHO;
        else if (u < 0) return ST_NEG_U;
        P[0] = rho;
        P[1] = u;
        const double pre = 1. / (ig * WB), qw = QdB / W;
        P[2] = pre * (Qtcon[1] + qw * Bcon[1]);
        P[3] = pre * (Qtcon[2] + qw * Bcon[2]);
        P[4] = pre * (Qtcon[3] + qw * Bcon[3]);
        return ST_SUCCESS;
    }
    const double gamma = lorentz_calc_w(Bsq, D, QdB, Qtsq, Wp);
    if (gamma < 1) return ST_BAD_UT;
    const double rho = D / gamma;
    const double w = W / (gamma*gamma);
    const double p = (w - rho) * (gam - 1) / gam;
    const double u = w - (rho + p);
    if (rho < 0 && u < 0) return ST_NEG_RHOU;
    else if (rho < 0) return ST_NEG_RHO;
    else if (u < 0) return ST_NEG_U;
    P[0] = rho;
    P[1] = u;
    const double pre = (gamma / (W + Bsq));
    P[2] = pre * (Qtcon[1] + QdB * Bcon[1] / W);
    P[3] = pre * (Qtcon[2] + QdB * Bcon[2] / W);
    P[4] = pre * (Qtcon[3] + QdB * Bcon[3] / W);
    return ST_SUCCESS;
}

// ------------------------------------------------------------------ Kastaun inversion (FP64)
// inverter/kastaun.hpp:83-406: master function of mu = 1/(h W), Illinois false position for a
// bracket (eq. 49) and then the root (eq. 44), inverter floors inside the residual.  Returns the
// FFlag bits of the floors hit (FF_INVERTER_*), or ST_MAX_ITER with P untouched.
enum { FF_INVERTER_RHO = 16384, FF_INVERTER_U = 32768, FF_INVERTER_GAMMA = 65536, FF_INVERTER_U_MAX = 131072 };

struct KastaunResidual {
    double D, q, bsq, bsq_rpsq, rsq, rbsq, v0sq, gam, rho_floor, e_floor, e_max;
    bool used_density_floor, used_energy_floor, used_energy_max, used_gamma_max;
    __device__ __forceinline__ double x_mu(double mu) const { return 1.0 / (1.0 + mu * bsq); }
    __device__ __forceinline__ double rbarsq_mu(double mu, double x) const { return x * (x * rsq + mu * (1.0 + x) * rbsq); }
    __device__ __forceinline__ double qbar_mu(double mu, double x) const
    {
        const double mux = mu * x;
        return q - 0.5 * (bsq + mux * mux * bsq_rpsq);
    }
    __device__ __forceinline__ double vhatsq_mu(double mu, double rbarsq)
    {
        const double vsq_trial = mu * mu * rbarsq;
        used_gamma_max = vsq_trial > v0sq;
        return used_gamma_max ? v0sq : vsq_trial;
    }
    __device__ __forceinline__ double rhohat_mu(double iWhat)
    {
        const double rho_trial = D * iWhat;
        used_density_floor = rho_trial <= rho_floor;
        return used_density_floor ? rho_floor : rho_trial;
    }
    __device__ __forceinline__ double ehat_mu(double mu, double qbar, double rbarsq, double vhatsq, double What)
    {
        const double ehat_trial = What * (qbar - mu * rbarsq) + vhatsq * What * What / (1.0 + What);
        used_energy_floor = false;
        used_energy_max = false;
        if (ehat_trial <= e_floor) { used_energy_floor = true; return e_floor; }
        if (ehat_trial > e_max) { used_energy_max = true; return e_max; }
        return ehat_trial;
    }
    __device__ __forceinline__ double master(double mu)      // eq. 44
    {
        const double x = x_mu(mu);
        const double rbarsq = rbarsq_mu(mu, x);
        const double qbar = qbar_mu(mu, x);
        const double vhatsq = vhatsq_mu(mu, rbarsq);
        const double iWhat = sqrt(1.0 - vhatsq);
        const double What = 1.0 / iWhat;
        const double rhohat = rhohat_mu(iWhat);
        const double ehat = ehat_mu(mu, qbar, rbarsq, vhatsq, What);
        const double Phat = ehat * rhohat * (gam - 1.0);
        const double hhat = rhohat * (1.0 + ehat) + Phat;
        const double ahat = Phat / (hhat - Phat);
        const double nua = (1.0 + ahat) * (1.0 + ehat) * iWhat;
        const double nub = (1.0 + ahat) * (1.0 + qbar - mu * rbarsq);
        const double nuhat = kmax(nua, nub);
        const double muhat = 1.0 / (nuhat + mu * rbarsq);
        return mu - muhat;
    }
    __device__ __forceinline__ double aux(double mu) const    // eq. 49
    {
        const double x = 1.0 / (1.0 + mu * bsq);
        const double rbarsq = x * (rsq * x + mu * (1.0 + x) * rbsq);
        return mu * sqrt(1.0 + rbarsq) - 1.0;
    }
    // Illinois false position on [zm, zp] (kastaun.hpp:305-331, 343-368); iter at exit
    template <bool MASTER>
    __device__ __forceinline__ double solve(double zm, double zp, int max_iterations, double tol, int& iter)
    {
        double fm = MASTER ? master(zm) : aux(zm);
        double fp = MASTER ? master(zp) : aux(zp);
        int iterations = max_iterations;
        if ((fabs(zm - zp) < tol) || ((fabs(fm) + fabs(fp)) < 2.0 * tol)) iterations = -1;
        double z = 0.5 * (zm + zp);
        for (iter = 0; iter < iterations; ++iter) {
            z = (zm * fp - zp * fm) / (fp - fm);
            const double fz = MASTER ? master(z) : aux(z);
            if ((fabs(zm - zp) < tol) || (fabs(fz) < tol)) break;
            if (fz * fp < 0.0) { zm = zp; fm = fp; zp = z; fp = fz; }
            else { fm = 0.5 * fm; zp = z; fp = fz; }
        }
        return z;
    }
};

template <int NV>
__device__ int u_to_p_kastaun(const ZoneGeom& G, double gam, const Prescription& fl, const double* U, double* P,
                              int max_iterations, double tol)
{
    const double alpha = 1. / sqrt(-G.gcon[0][0]);
    const double a_over_g = alpha / G.gdet;
    const double D = U[0] * a_over_g;
    const double D_fl = kmax(D, fl.rho_min_const);
    const double Qcov[4] = {(U[1] - U[0]) * a_over_g, U[2] * a_over_g, U[3] * a_over_g, U[4] * a_over_g};
    const double ncov[4] = {-alpha, 0., 0., 0.};
    double ncon[4];
    raise4(G, ncov, ncon);
    const double q = (-dot4(Qcov, ncon) - D) / D;
    const double rcov[3] = {U[2] / U[0], U[3] / U[0], U[4] / U[0]};
    double rcon[3];
#pragma unroll
    for (int a = 0; a < 3; ++a)   // gamma^ij = g^ij - g^0i g^0j / g^00 (kastaun.hpp:250-262)
        rcon[a] = ((G.gcon[a+1][1] - G.gcon[0][a+1]*G.gcon[0][1]/G.gcon[0][0])*rcov[0] +
                   (G.gcon[a+1][2] - G.gcon[0][a+1]*G.gcon[0][2]/G.gcon[0][0])*rcov[1] +
                   (G.gcon[a+1][3] - G.gcon[0][a+1]*G.gcon[0][3]/G.gcon[0][0])*rcov[2]);
    double rsq = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) rsq += rcon[a] * rcov[a];
    double bsq = 0.0, bsq_rpsq = 0.0, rbsq = 0.0, bdotr = 0.0, bu[3] = {0.0, 0.0, 0.0};
    if (NV > 5) {
        const double sD = 1.0 / sqrt(D_fl);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            bu[a] = (U[5 + a] * a_over_g) * sD;
            bdotr += bu[a] * rcov[a];
        }
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) bsq += G.gcov[a + 1][b + 1] * bu[a] * bu[b];
        bsq = kmax(0.0, bsq);
        rbsq = bdotr * bdotr;
        bsq_rpsq = bsq * rsq - rbsq;
    }
    const double zsq = rsq;
    KastaunResidual res;
    res.D = D; res.q = q; res.bsq = bsq; res.bsq_rpsq = bsq_rpsq; res.rsq = rsq; res.rbsq = rbsq;
    res.v0sq = kmin(zsq / (1.0 + zsq), 1.0 - 1.0 / (fl.gamma_max * fl.gamma_max));
    res.gam = gam; res.rho_floor = fl.rho_min_const; res.e_floor = fl.u_min_const / D_fl; res.e_max = fl.u_over_rho_max;
    res.used_density_floor = res.used_energy_floor = res.used_energy_max = res.used_gamma_max = false;
    int iter = 0;
    const double zb = res.solve<false>(0., 1., max_iterations, tol, iter);
    const double mu = res.solve<true>(0., zb, max_iterations, tol, iter);
    if (iter == max_iterations) return ST_MAX_ITER;
    const double x = res.x_mu(mu);
    const double rbarsq = res.rbarsq_mu(mu, x);
    const double vsq = res.vhatsq_mu(mu, rbarsq);
    const double iW = sqrt(1.0 - vsq);
    const double W = 1. / iW;
    P[0] = res.rhohat_mu(iW);
    const double qbar = res.qbar_mu(mu, x);
    P[1] = res.ehat_mu(mu, qbar, rbarsq, vsq, W) * P[0];
#pragma unroll
    for (int a = 0; a < 3; ++a) P[2 + a] = W * mu * x * (rcon[a] + mu * bdotr * bu[a]);
    int fflag = 0;
    if (res.used_density_floor) fflag |= FF_INVERTER_RHO;
    if (res.used_energy_floor) fflag |= FF_INVERTER_U;
    if (res.used_gamma_max) fflag |= FF_INVERTER_GAMMA;
    if (res.used_energy_max) fflag |= FF_INVERTER_U_MAX;
    return fflag;
}

// ------------------------------------------------------------------ floors (FP64)
// FFlag bits, floors.hpp:52-70
enum { FF_GEOM_RHO = 32, FF_GEOM_U = 64, FF_B_RHO = 128, FF_B_U = 256, FF_TEMP = 512, FF_GAMMA = 1024,
       FF_KTOT = 2048, FF_GEOM_RHO_FLUX = 4096, FF_GEOM_U_FLUX = 8192 };

// (gam - 1) u / pow(rho, gam) > ktot_max, decided exactly as that expression evaluates, with pow
// evaluated only when a cheap bound cannot settle the comparison.  The bound takes log2 of each
// factor from its binary exponent plus a single-precision log2 of its mantissa: the estimate of
// log2(ktot / ktot_max) is within 2e-6 of the true value for gam <= 4, and the exact quotient is
// within a few ulp of the true one, so an estimate beyond +-1/64 puts both on the same side.
// Zero, negative, subnormal, huge or non-finite operands and results near the exponent range take
// the exact path.
__device__ __forceinline__ double log2_est(double x)   // x positive and normal
{
    int e;
    const double m = frexp(x, &e);                     // x = m 2^e, m in [0.5, 1)
    return (double)e + (double)__log2f((float)m);
}
__device__ __forceinline__ bool ktot_above(double gam, double rho, double u, double ktot_max)
{
    const double a = (gam - 1.) * u;
    const double dmin = 2.2250738585072014e-308;
    if (rho >= dmin && a >= dmin && ktot_max >= dmin && rho <= 1e300 && a <= 1e300 && ktot_max <= 1e300 &&
        gam > 0. && gam <= 4.) {
        const double lr = gam * log2_est(rho);
        if (lr > -1000. && lr < 1000.) {
            const double est = log2_est(a) - lr - log2_est(ktot_max);
            if (est < -0.015625) return false;
            if (est > 0.015625) return true;
        }
    }
    return a / pow(rho, gam) > ktot_max;
}

// floors_functions.hpp:84-160
// rhoflr_geom, uflr_geom: the geometric floor values of this zone (x3-independent, tabulated per
// (j,i) at set-up with the same formula, floors_functions.hpp:96-104).  D returns the 4-vectors of P.
template <int NV>
__device__ int determine_floors(const ZoneGeom& G, const Prescription& f, double rhoflr_geom, double uflr_geom,
                                double gam, const double* P, double& rhoflr_max, double& uflr_max, FourVec<double>& D)
{
    double gcon0[4] = {G.gcon[0][0], G.gcon[0][1], G.gcon[0][2], G.gcon[0][3]};
    calc_4vecs<double, (NV > 5)>(G.gcov, G.gcon[0][0], gcon0, P, D);
    const double bsq = dot4(D.bcon, D.bcov);
    const double rhoflr_b = bsq / f.bsq_over_rho_max;
    const double uflr_b   = bsq / f.bsq_over_u_max;
    uflr_max = kmax(uflr_geom, uflr_b);
    const double rho = P[0], u = P[1];
    int fflag = 0;
    if (!f.temp_adjust_u) {
        const double rhoflr_temp = kmax(u, uflr_max) / f.u_over_rho_max;
        fflag |= (rhoflr_temp > rho) * FF_TEMP;
        rhoflr_max = kmax(kmax(rhoflr_geom, rhoflr_b), rhoflr_temp);
    } else {
        rhoflr_max = kmax(rhoflr_geom, rhoflr_b);
    }
    if (rhoflr_max > rho || uflr_max > u) {
        fflag |= (rhoflr_geom > rho) * FF_GEOM_RHO;
        fflag |= (uflr_geom > u) * FF_GEOM_U;
        fflag |= (rhoflr_b > rho) * FF_B_RHO;
        fflag |= (uflr_b > u) * FF_B_U;
    }
    if (lorentz(G.gcov, P[2], P[3], P[4]) > f.gamma_max) fflag |= FF_GAMMA;
    if (ktot_above(gam, P[0], P[1], f.ktot_max)) fflag |= FF_KTOT;
    if (f.temp_adjust_u && (P[1] / P[0] > f.u_over_rho_max)) fflag |= FF_TEMP;
    return fflag;
}

// floors_functions.hpp:50-82
__device__ __forceinline__ void apply_ceilings(const ZoneGeom& G, const Prescription& f, double gam, double* P)
{
    const double gamma = lorentz(G.gcov, P[2], P[3], P[4]);
    if (gamma > f.gamma_max) {
        const double fr = sqrt((f.gamma_max*f.gamma_max - 1.) / (gamma*gamma - 1.));
#pragma unroll
        for (int v = 0; v < 3; ++v) P[2 + v] *= fr;
    }
    // ktot is formed from rho and u before either ceiling changes them (the velocity ceiling above
    // leaves both alone)
    if (ktot_above(gam, P[0], P[1], f.ktot_max)) {
        const double ktot = (gam - 1.) * P[1] / pow(P[0], gam);
        P[1] = f.ktot_max / ktot * P[1];
    }
    if (f.temp_adjust_u && P[1] / P[0] > f.u_over_rho_max) P[1] = f.u_over_rho_max * P[0];
}

// floors_functions.hpp:174-179 (fluid), 181-252 (drift), 254-289 (normal observer)
// D_pre: the 4-vectors of P on entry when the caller has them (determine_floors computed them from the
// same P and geometry, so they are the ones the drift frame would compute), else NULL
template <int NV>
__device__ int apply_floors_frame(const ZoneGeom& G, int frame, double gam, double* P, double* U,
                                  double rhoflr_max, double uflr_max, int iter_max_nof,
                                  const FourVec<double>* D_pre = nullptr)
{
    if (frame == 0) {
        P[0] += kmax(0., rhoflr_max - P[0]);
        P[1] += kmax(0., uflr_max - P[1]);
        return 0;
    } else if (frame == 2) {
        const double lapse2 = 1. / (-G.gcon[0][0]);
        double beta[4] = {0., 0., 0., 0.};
        beta[1] = lapse2 * G.gcon[0][1];
        beta[2] = lapse2 * G.gcon[0][2];
        beta[3] = lapse2 * G.gcon[0][3];
        const double rho = P[0];
        const double uu  = P[1];
        const double pg  = (gam - 1.) * uu;
        const double w_old = kmax(rho + uu + pg, 1e-20);
        double Bcon[4] = {0., 0., 0., 0.}, Bcov[4] = {0., 0., 0., 0.};
        if (NV > 5) { Bcon[1] = P[5]; Bcon[2] = P[6]; Bcon[3] = P[7]; }
#pragma unroll
        for (int mu = 0; mu < 4; ++mu)
#pragma unroll
            for (int nu = 0; nu < 4; ++nu) Bcov[mu] += G.gcov[mu][nu] * Bcon[nu];
        const double Bsq   = kmax(dot4(Bcon, Bcov), 1e-20);
        const double B_mag = sqrt(Bsq);
        FourVec<double> D;
        if (D_pre) {
            D = *D_pre;
        } else {
            double gcon0[4] = {G.gcon[0][0], G.gcon[0][1], G.gcon[0][2], G.gcon[0][3]};
            calc_4vecs<double, (NV > 5)>(G.gcov, G.gcon[0][0], gcon0, P, D);
        }
        double Qcov[4];
        Qcov[0] = w_old * D.ucon[0] * D.ucov[0] + pg;
        Qcov[1] = w_old * D.ucon[0] * D.ucov[1];
        Qcov[2] = w_old * D.ucon[0] * D.ucov[2];
        Qcov[3] = w_old * D.ucon[0] * D.ucov[3];
        const double QdotB = dot4(Bcon, Qcov);
        double vpar = QdotB / (B_mag * w_old * D.ucon[0]*D.ucon[0]);
        double ucon_dr[4] = {0., 0., 0., 0.};
        ucon_dr[0] = 1. / sqrt(1. / (D.ucon[0]*D.ucon[0]) + vpar*vpar);
#pragma unroll
        for (int mu = 0; mu < 4; ++mu)
            ucon_dr[mu] = D.ucon[mu] * (ucon_dr[0] / D.ucon[0]) - (vpar * Bcon[mu] * ucon_dr[0] / B_mag);
        P[0] = kmax(rho, rhoflr_max);
        P[1] = kmax(uu, uflr_max);
        const double pg_new = (gam - 1.) * P[1];
        const double w_new  = P[0] + P[1] + pg_new;
        const double x = (2. * QdotB) / (B_mag * w_new * ucon_dr[0]);
        vpar = x / (1 + sqrt(1 + x*x)) * (1. / ucon_dr[0]);
        double uc[4];
        uc[0] = 1. / sqrt(1/(ucon_dr[0]*ucon_dr[0]) - vpar*vpar);
#pragma unroll
        for (int mu = 0; mu < 4; ++mu) uc[mu] = ucon_dr[mu] * (uc[0] / ucon_dr[0]) + (vpar * Bcon[mu] * uc[0] / B_mag);
        P[2] = uc[1] + (beta[1] * uc[0]);
        P[3] = uc[2] + (beta[2] * uc[0]);
        P[4] = uc[3] + (beta[3] * uc[0]);
        return 0;
    } else {
        const double rho_add = kmax(0., rhoflr_max - P[0]);
        const double u_add   = kmax(0., uflr_max - P[1]);
        double Pa[8] = {rho_add, u_add, 0., 0., 0., 0., 0., 0.};
        FourVec<double> D;
        double gcon0[4] = {G.gcon[0][0], G.gcon[0][1], G.gcon[0][2], G.gcon[0][3]};
        calc_4vecs<double, true>(G.gcov, G.gcon[0][0], gcon0, Pa, D);
        const double rho_ut = rho_add * D.ucon[0] * G.gdet;
        double mhd[4];
        calc_tensor<double, true>(rho_add, u_add, (gam - 1) * u_add, D, 0, mhd);
        P[0] += rho_add;
        P[1] += u_add;
        U[0] += rho_ut;
        U[1] += mhd[0] * G.gdet + rho_ut;
        U[2] += mhd[1] * G.gdet;
        U[3] += mhd[2] * G.gdet;
        U[4] += mhd[3] * G.gdet;
        return u_to_p_onedw<NV>(G, gam, U, P, iter_max_nof, 1e-8);
    }
}

} // namespace khb

// khb_geometry.cpp -- host construction of the per-block geometry tables (GRCoordinates caches).
//
// The metric is independent of x3 for every supported system, so the tables are 2D in (j, i).
// Restates coordinates/coordinate_systems.hpp, coordinate_embedding.hpp, matrix.hpp and
// gr_coordinates.cpp:96-205 with connection_average_points = 1.  Runs once per block at setup;
// the kernels only read the tables khb_set_geometry uploads.
#include "../../include/khb.h"

#include <cmath>
#include <cstring>

namespace {

const double kSmall = 1e-20;   // decs.hpp:82

inline double excise(double n, double c, double r)   // kharma_utils.hpp:118-122
{
    return (std::fabs(n - c) > r) ? n : ((n > c) ? c + r : c - r);
}

struct System {
    khb_coords s;
    double poly_norm;

    explicit System(const khb_coords& cs) : s(cs)
    {
        poly_norm = 0.5 * M_PI * 1./(1. + 1./(s.poly_alpha + 1.) * 1./std::pow(s.poly_xt, s.poly_alpha));
    }
    bool spherical() const { return s.base != KHB_BASE_CART_MINKOWSKI; }

    // Native -> embedding coordinates
    void to_embed(const double X[4], double Xe[4]) const
    {
        Xe[0] = X[0];
        Xe[3] = X[3];
        if (s.transform == KHB_TRANSFORM_NULL) { Xe[1] = X[1]; Xe[2] = X[2]; return; }
        Xe[1] = std::exp(X[1]);
        double th;
        if (s.transform == KHB_TRANSFORM_EKS) {
            th = X[2];
        } else if (s.transform == KHB_TRANSFORM_MKS) {
            th = M_PI*X[2] + ((1. - s.hslope)/2.)*std::sin(2.*M_PI*X[2]);
        } else {
            const double thG = M_PI*X[2] + ((1. - s.hslope)/2.)*std::sin(2.*M_PI*X[2]);
            const double y = 2*X[2] - 1.;
            const double thJ = poly_norm * y * (1. + std::pow(y/s.poly_xt, s.poly_alpha) / (s.poly_alpha + 1.)) + 0.5 * M_PI;
            th = thG + std::exp(s.mks_smooth * (s.startx1 - X[1])) * (thJ - thG);
        }
        Xe[2] = excise(excise(th, 0.0, kSmall), M_PI, kSmall);
    }

    // Jacobian d(embedding)/d(native)
    void jac(const double X[4], double J[4][4]) const
    {
        for (int a = 0; a < 4; ++a) for (int b = 0; b < 4; ++b) J[a][b] = (a == b);
        if (s.transform == KHB_TRANSFORM_NULL) return;
        for (int a = 0; a < 4; ++a) for (int b = 0; b < 4; ++b) J[a][b] = 0.;
        J[0][0] = 1.; J[3][3] = 1.;
        J[1][1] = std::exp(X[1]);
        if (s.transform == KHB_TRANSFORM_EKS) {
            J[2][2] = 1.;
        } else if (s.transform == KHB_TRANSFORM_MKS) {
            J[2][2] = M_PI - (s.hslope - 1.)*M_PI*std::cos(2.*M_PI*X[2]);
        } else {
            const double h = s.hslope, ms = s.mks_smooth, x0 = s.startx1, xt = s.poly_xt, pa = s.poly_alpha;
            J[2][1] = -std::exp(ms * (x0 - X[1])) * ms
                * (M_PI / 2. - M_PI * X[2]
                   + poly_norm * (2. * X[2] - 1.) * (1 + (std::pow((-1. + 2 * X[2]) / xt, pa)) / (1 + pa))
                   - 1. / 2. * (1. - h) * std::sin(2. * M_PI * X[2]));
            J[2][2] = M_PI + (1. - h) * M_PI * std::cos(2. * M_PI * X[2])
                + std::exp(ms * (x0 - X[1]))
                    * (-M_PI
                       + 2. * poly_norm * (1. + std::pow((2. * X[2] - 1.) / xt, pa) / (pa + 1.))
                       + (2. * pa * poly_norm * (2. * X[2] - 1.) * std::pow((2. * X[2] - 1.) / xt, pa - 1.))
                           / ((1. + pa) * xt)
                       - (1. - h) * M_PI * std::cos(2. * M_PI * X[2]));
        }
    }

    // Metric of the base system at embedding coordinates
    void base_gcov(const double Xe[4], double g[4][4]) const
    {
        const double a = s.a;
        for (int m = 0; m < 4; ++m) for (int n = 0; n < 4; ++n) g[m][n] = 0.;
        if (s.base == KHB_BASE_CART_MINKOWSKI) {
            for (int m = 0; m < 4; ++m) for (int n = 0; n < 4; ++n) g[m][n] = (m == n) - 2*(m == 0 && n == 0);
            return;
        }
        const double th = excise(excise(Xe[2], 0.0, kSmall), M_PI, kSmall);
        if (s.base == KHB_BASE_SPH_MINKOWSKI) {
            const double r = (Xe[1] < kSmall) ? kSmall : Xe[1];
            const double sth = std::sin(th);
            g[0][0] = 1.; g[1][1] = 1.; g[2][2] = r*r; g[3][3] = sth*sth*r*r;
        } else if (s.base == KHB_BASE_SPH_KS) {
            const double r = Xe[1];
            const double cth = std::cos(th), sth = std::sin(th);
            const double sin2 = sth*sth;
            const double rho2 = r*r + a*a*cth*cth;
            g[0][0] = -1. + 2.*r/rho2;
            g[0][1] = 2.*r/rho2;
            g[0][3] = -2.*a*r*sin2/rho2;
            g[1][0] = 2.*r/rho2;
            g[1][1] = 1. + 2.*r/rho2;
            g[1][3] = -a*sin2*(1. + 2.*r/rho2);
            g[2][2] = rho2;
            g[3][0] = -2.*a*r*sin2/rho2;
            g[3][1] = -a*sin2*(1. + 2.*r/rho2);
            g[3][3] = sin2*(rho2 + a*a*sin2*(1. + 2.*r/rho2));
        } else {
            const double r = Xe[1];
            const double cth = std::cos(th), sth = std::sin(th);
            const double sin2 = sth*sth, a2 = a*a, r2 = r*r;
            const double mmu = 1. + a2*cth*cth/r2;
            g[0][0] = -(1. - 2./(r*mmu));
            g[0][3] = -2.*a*sin2/(r*mmu);
            g[1][1] = mmu/(1. - 2./r + a2/r2);
            g[2][2] = r2*mmu;
            g[3][0] = -2.*a*sin2/(r*mmu);
            g[3][3] = sin2*(r2 + a2 + 2.*a2*sin2/(r*mmu));
        }
    }

    // Covariant metric in native coordinates: g_mn = J^l_m J^k_n g_lk
    void gcov(const double X[4], double g[4][4]) const
    {
        double Xe[4], gb[4][4], J[4][4];
        to_embed(X, Xe);
        base_gcov(Xe, gb);
        jac(X, J);
        for (int m = 0; m < 4; ++m) for (int n = 0; n < 4; ++n) {
            double acc = 0;
            for (int l = 0; l < 4; ++l) for (int k = 0; k < 4; ++k) acc += gb[l][k]*J[l][m]*J[k][n];
            g[m][n] = acc;
        }
    }

    double radius(const double X[4]) const
    {
        double Xe[4];
        to_embed(X, Xe);
        return spherical() ? Xe[1] : std::sqrt(Xe[1]*Xe[1] + Xe[2]*Xe[2] + Xe[3]*Xe[3]);
    }
};

// 4x4 inverse by cofactors (matrix.hpp:56-115); returns the determinant
inline double minor3(const double* m, int r0, int r1, int r2, int c0, int c1, int c2)
{
    return m[4*r0+c0]*(m[4*r1+c1]*m[4*r2+c2] - m[4*r2+c1]*m[4*r1+c2]) -
           m[4*r0+c1]*(m[4*r1+c0]*m[4*r2+c2] - m[4*r2+c0]*m[4*r1+c2]) +
           m[4*r0+c2]*(m[4*r1+c0]*m[4*r2+c1] - m[4*r2+c0]*m[4*r1+c1]);
}
double inverse4(const double* m, double* o)
{
    static const int R[4][3] = {{1,2,3},{0,2,3},{0,1,3},{0,1,2}};
    for (int row = 0; row < 4; ++row)
        for (int col = 0; col < 4; ++col) {
            // adjugate: o[row][col] = (-1)^(row+col) * minor(col removed row, row removed col)
            const int* rr = R[col];
            const int* cc = R[row];
            const double mm = minor3(m, rr[0], rr[1], rr[2], cc[0], cc[1], cc[2]);
            o[4*row + col] = ((row + col) % 2) ? -mm : mm;
        }
    const double det = m[0]*minor3(m,1,2,3,1,2,3) - m[1]*minor3(m,1,2,3,0,2,3) +
                       m[2]*minor3(m,1,2,3,0,1,3) - m[3]*minor3(m,1,2,3,0,1,2);
    const double inv = 1. / det;
    for (int x = 0; x < 16; ++x) o[x] *= inv;
    return det;
}

// Connection Gamma^l_{n m} by centred differences of gcov (coordinate_embedding.hpp:526-572)
void connection(const System& S, const double X[4], double delta, double conn[4][4][4])
{
    double dg[4][4][4];   // dg[l][k][n] = d_n g_lk
    for (int n = 0; n < 4; ++n) {
        double Xh[4], Xl[4], gh[4][4], gl[4][4];
        for (int m = 0; m < 4; ++m) { Xl[m] = X[m] - delta*(m == n); Xh[m] = X[m] + delta*(m == n); }
        S.gcov(Xh, gh);
        S.gcov(Xl, gl);
        for (int l = 0; l < 4; ++l) for (int k = 0; k < 4; ++k) dg[l][k][n] = (gh[l][k] - gl[l][k]) / (Xh[n] - Xl[n]);
    }
    double low[4][4][4];
    for (int l = 0; l < 4; ++l) for (int n = 0; n < 4; ++n) for (int m = 0; m < 4; ++m)
        low[l][n][m] = 0.5 * (dg[n][l][m] + dg[m][l][n] - dg[m][n][l]);
    double g[4][4], gi[4][4];
    S.gcov(X, g);
    inverse4(&g[0][0], &gi[0][0]);
    for (int l = 0; l < 4; ++l) for (int n = 0; n < 4; ++n) for (int m = 0; m < 4; ++m) {
        double acc = 0.;
        for (int k = 0; k < 4; ++k) acc += gi[l][k] * low[k][n][m];
        conn[l][n][m] = acc;
    }
}

} // namespace

extern "C" int khb_build_geometry(const khb_coords* coords, const khb_config* cfg,
                                  double x1min, double x2min, double x3min,
                                  double* gcov, double* gcon, double* gdet, double* gdet_conn, double* r_center)
{
    if (!coords || !cfg || !gcov || !gcon || !gdet || !gdet_conn || !r_center) return KHB_ERR_ARG;
    const System S(*coords);
    const int ng = cfg->ng;
    const int n1 = cfg->nx1 + 2*ng;
    const int n2 = (cfg->nx2 > 1) ? cfg->nx2 + 2*ng : 1;
    const int g2 = (cfg->nx2 > 1) ? ng : 0, g3 = (cfg->nx3 > 1) ? ng : 0;
    const int G1 = n1 + 1, G2 = n2 + 1;
    // Parthenon UniformCartesian positions: faces at xmin + (idx - nghost) dx, centres half a zone on
    const double o1 = x1min - ng*cfg->dx1, o2 = x2min - g2*cfg->dx2, o3 = x3min - g3*cfg->dx3;
    auto Xf = [&](int d, int idx) { return (d == 1 ? o1 : (d == 2 ? o2 : o3)) + idx*(d == 1 ? cfg->dx1 : (d == 2 ? cfg->dx2 : cfg->dx3)); };
    auto Xc = [&](int d, int idx) { return (d == 1 ? o1 : (d == 2 ? o2 : o3)) + (idx + 0.5)*(d == 1 ? cfg->dx1 : (d == 2 ? cfg->dx2 : cfg->dx3)); };
    std::memset(gcov, 0, sizeof(double)*7*G2*G1*16);
    std::memset(gcon, 0, sizeof(double)*7*G2*G1*16);
    std::memset(gdet, 0, sizeof(double)*7*G2*G1);
    for (int j = 0; j < G2; ++j) for (int i = 0; i < G1; ++i) {
        for (int loc = 0; loc < 7; ++loc) {
            // centre and face3 tables stop at the last zone (gr_coordinates.cpp:130-132)
            if ((loc == 2 || loc == 3) && (i >= n1 || j >= n2)) continue;
            double X[4] = {0., Xc(1, i), Xc(2, j), Xc(3, 0)};
            if (loc == 0) X[1] = Xf(1, i);
            if (loc == 1) X[2] = Xf(2, j);
            if (loc == 2) X[3] = Xf(3, 0);
            if (loc == 4) { X[1] = Xf(1, i); X[2] = Xf(2, j); X[3] = Xf(3, 0); }
            if (loc == 5) X[2] = (Xc(2, j) + Xf(2, j+1)) / 2;
            if (loc == 6) X[2] = (Xc(2, j) + Xf(2, j)) / 2;
            double g[4][4], gi[4][4];
            S.gcov(X, g);
            const double det = inverse4(&g[0][0], &gi[0][0]);
            const long long o = ((long long)loc*G2 + j)*G1 + i;
            gdet[o] = std::sqrt(std::fabs(det));
            for (int m = 0; m < 4; ++m) for (int n = 0; n < 4; ++n) {
                gcov[o*16 + m*4 + n] = g[m][n];
                gcon[o*16 + m*4 + n] = gi[m][n];
            }
            if (loc == 3) {
                double cn[4][4][4];
                connection(S, X, 1.e-8, cn);
                const long long q = ((long long)j*n1 + i)*64;
                for (int a = 0; a < 4; ++a) for (int b = 0; b < 4; ++b) for (int c = 0; c < 4; ++c)
                    gdet_conn[q + a*16 + b*4 + c] = gdet[o]*cn[a][b][c];
                r_center[(long long)j*n1 + i] = S.radius(X);
            }
        }
    }
    return KHB_OK;
}

// The connection itself at zone centres (conn_direct, gr_coordinates.cpp:156-161): 0 + conn/1 with
// connection_average_points = 1, i.e. the centred-difference value unchanged.
extern "C" int khb_build_connection(const khb_coords* coords, const khb_config* cfg,
                                    double x1min, double x2min, double x3min, double* conn)
{
    if (!coords || !cfg || !conn) return KHB_ERR_ARG;
    const System S(*coords);
    const int ng = cfg->ng;
    const int n1 = cfg->nx1 + 2*ng;
    const int n2 = (cfg->nx2 > 1) ? cfg->nx2 + 2*ng : 1;
    const int g2 = (cfg->nx2 > 1) ? ng : 0, g3 = (cfg->nx3 > 1) ? ng : 0;
    const double o1 = x1min - ng*cfg->dx1, o2 = x2min - g2*cfg->dx2, o3 = x3min - g3*cfg->dx3;
    for (int j = 0; j < n2; ++j) for (int i = 0; i < n1; ++i) {
        double X[4] = {0., o1 + (i + 0.5)*cfg->dx1, o2 + (j + 0.5)*cfg->dx2, o3 + (0 + 0.5)*cfg->dx3};
        double cn[4][4][4];
        connection(S, X, 1.e-8, cn);
        const long long q = ((long long)j*n1 + i)*64;
        for (int a = 0; a < 4; ++a) for (int b = 0; b < 4; ++b) for (int c = 0; c < 4; ++c)
            conn[q + a*16 + b*4 + c] = cn[a][b][c];
    }
    return KHB_OK;
}

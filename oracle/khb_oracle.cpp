/*
 * khb_oracle.cpp -- CPU ORACLE for the KHARMA per-step GRMHD hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path in
 * kharma_b200/ is compared against.  Only tests/, __graft_entry__.smoke() and
 * the CPU-baseline leg of bench.py may load it.  The product never links it.
 *
 * It is a plain, scalar, line-by-line restatement of the reference's device
 * functions and step sequencing (AFD-Illinois/kharma), compiled with
 * g++ -O2 -ffp-contract=off so every add/mul/div/sqrt is a single IEEE
 * operation in the reference's evaluation order.  Each function cites the
 * reference file:line it follows.
 *
 * Parity pinning: the reference cannot be built here (Parthenon, Kokkos and
 * mpark::variant are empty submodules), so the oracle is pinned by the
 * reference's own known-answer tests: the MHD linear-mode eigenvectors of
 * kharma/prob/mhdmodes.hpp and the second-order convergence slopes that
 * tests/mhdmodes/check.py asserts.  The pieces that live in the un-vendored
 * Parthenon (RK2 coefficients, FluxDivHelper, WeightedSumData, outflow and
 * reflecting boundary functions, UniformCartesian cell positions) are restated
 * from their published algorithms and marked "Parthenon (unvendored)".
 *
 * Layout: every cell field is [var][k][j][i], i fastest, over the entire block
 * including ghosts (n1 = nx1 + 2 ng; n2, n3 likewise when the direction is
 * active, else 1).  Fluxes use the same shape; face index i is the left face
 * of cell i.  Geometry caches follow GRCoordinates:
 *   gcov/gcon [7][n2+1][n1+1][4][4], gdet [7][n2+1][n1+1],
 *   conn/gdet_conn [n2][n1][4][4][4]           (gr_coordinates.cpp:105-109)
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <limits>
#include <omp.h>

namespace orc {

// ---------------------------------------------------------------- basics
static const double SMALL = 1e-20;                  // decs.hpp:82
enum Loci { face1 = 0, face2, face3, center, corner, outer_half, inner_half };  // decs.hpp:104
static const int NLOC = 7;

// Kokkos::max/min semantics ((a<b)?b:a), used by the reference as m::max/m::min
static inline double kmax(double a, double b) { return (a < b) ? b : a; }
static inline double kmin(double a, double b) { return (b < a) ? b : a; }
// kharma_utils.hpp:100-110
static inline double clip(double n, double lower, double upper) { return kmin(kmax(lower, n), upper); }
// kharma_utils.hpp:118-122
static inline double excise(double n, double center, double range)
{
    return (std::fabs(n - center) > range) ? n : ((n > center) ? center + range : center - range);
}
// matrix.hpp:51-54
static inline double dot4(const double* a, const double* b)
{
    return a[0]*b[0] + a[1]*b[1] + a[2]*b[2] + a[3]*b[3];
}

// ---------------------------------------------------------------- config
struct Prescription {          // floors.hpp:100-117
    double rho_min_const, u_min_const;
    double rho_min_geom, u_min_geom, r_char;
    double bsq_over_rho_max, bsq_over_u_max, u_over_rho_max;
    double ktot_max, gamma_max;
    int32_t use_r_char, temp_adjust_u, adjust_k, radius_dependent_floors;
    double floors_switch_r;
};

struct CoordSpec {
    int32_t base;       // 0 cartesian minkowski, 1 spherical minkowski, 2 spherical KS, 3 spherical BL
    int32_t transform;  // 0 null, 1 exponential (eks), 2 modified (mks), 3 funky (fmks)
    double a, hslope, mks_smooth, poly_xt, poly_alpha, startx1;
};

enum Recon { RECON_DONOR = 0, RECON_MC = 1, RECON_WENO5 = 2, RECON_PPM = 3, RECON_LINEAR_VL = 4,
             RECON_WENO5_LINEAR = 5, RECON_PPMX = 6, RECON_MP5 = 7 };
enum BC { BC_PERIODIC = 0, BC_OUTFLOW = 1, BC_REFLECT = 2, BC_EXCHANGE = 3, BC_TRANSMIT = 4 };
// Exchange faces are internal block boundaries whose ghost zones the caller fills (Parthenon's
// boundary communication); only outflow and reflecting faces are global "user" boundaries.
static inline bool phys_face(int bc) { return bc == BC_OUTFLOW || bc == BC_REFLECT || bc == BC_TRANSMIT; }
enum Frame { FRAME_FLUID = 0, FRAME_NORMAL = 1, FRAME_DRIFT = 2, FRAME_MIXED_FLUID_NORMAL = 3, FRAME_MIXED_NORMAL_DRIFT = 4 };

struct Config {
    int32_t nx1, nx2, nx3, ng;
    double x1min, x2min, x3min, dx1, dx2, dx3;     // interior block start and widths (native coords)
    double gam;
    int32_t recon, riemann;                         // riemann: 0 llf, 1 hlle
    int32_t nvar;                                   // 5 (GRHD) or 8 (GRMHD with flux-CT B)
    int32_t driver;                                 // 0 simple, 1 kharma
    int32_t bc[6];                                  // inner_x1, outer_x1, inner_x2, outer_x2, inner_x3, outer_x3
    int32_t check_inflow_inner_x1, check_inflow_outer_x1;
    int32_t zero_polar_flux, fix_polar_flux, fix_corner_inner;
    int32_t floors_on, floor_frame, recon_floors;
    int32_t iter_max; double err_tol;
    int32_t fix_average_neighbors, fix_atmosphere;
    double cfl, dt_min, max_dt_increase;
    Prescription floors;
    int32_t inverter;                               // 0 onedw, 1 kastaun (inverter/type)
    int32_t fofc, fofc_polar_cells;                 // fofc/on, fofc/polar_cells
    double fofc_eh_buffer, r_horizon;               // fofc/eh_buffer, coords.get_horizon()
    int32_t ct_scheme;                              // 0 B_FluxCT; B_CT: 1 bs99, 2 gs05_0, 3 gs05_c (b_ct.cpp:65)
    int32_t recon_lower;                            // weno5 lowered to MC: 1 low_order_edges, 2 low_order_poles
    int32_t recon_fallback;                         // flux/reconstruction_fallback
    Prescription floors_inner;                      // floors_inner (floors.hpp:155-167)
    double frame_switch_r, frame_switch_beta;       // floors/frame_switch_r, floors/frame_switch_beta
    int32_t fofc_use_glf, fofc_use_source_term;     // fofc/use_glf, fofc/use_source_term
};

// ---------------------------------------------------------------- coordinates
// coordinate_systems.hpp / coordinate_embedding.hpp restated
struct Coords {
    CoordSpec s;
    double poly_norm;
    bool spherical() const { return s.base != 0; }
    bool cart_minkowski() const { return s.base == 0 && s.transform == 0; }   // coordinate_embedding.hpp:269-272

    void init()
    {
        // coordinate_systems.hpp:599-601 (FunkyTransform constructor)
        poly_norm = 0.5 * M_PI * 1./(1. + 1./(s.poly_alpha + 1.) * 1./std::pow(s.poly_xt, s.poly_alpha));
    }
    // coord_to_embed for each transform: coordinate_systems.hpp:358-367, 414-425, 538-549, 603-618
    void coord_to_embed(const double X[4], double Xe[4]) const
    {
        switch (s.transform) {
        case 0:
            for (int mu = 0; mu < 4; ++mu) Xe[mu] = X[mu];
            break;
        case 1:
            Xe[0] = X[0];
            Xe[1] = std::exp(X[1]);
            Xe[2] = excise(excise(X[2], 0.0, SMALL), M_PI, SMALL);
            Xe[3] = X[3];
            break;
        case 2: {
            Xe[0] = X[0];
            Xe[1] = std::exp(X[1]);
            const double th = M_PI*X[2] + ((1. - s.hslope)/2.)*std::sin(2.*M_PI*X[2]);
            Xe[2] = excise(excise(th, 0.0, SMALL), M_PI, SMALL);
            Xe[3] = X[3];
            break;
        }
        default: {
            Xe[0] = X[0];
            Xe[1] = std::exp(X[1]);
            const double thG = M_PI*X[2] + ((1. - s.hslope)/2.)*std::sin(2.*M_PI*X[2]);
            const double y = 2*X[2] - 1.;
            const double thJ = poly_norm * y * (1. + std::pow(y/s.poly_xt, s.poly_alpha) / (s.poly_alpha + 1.)) + 0.5 * M_PI;
            const double th = thG + std::exp(s.mks_smooth * (s.startx1 - X[1])) * (thJ - thG);
            Xe[2] = excise(excise(th, 0.0, SMALL), M_PI, SMALL);
            Xe[3] = X[3];
            break;
        }
        }
    }
    // dxdX: coordinate_systems.hpp:367-375, 435-443, 561-569, 630-656
    void dxdX(const double X[4], double J[4][4]) const
    {
        for (int mu = 0; mu < 4; ++mu) for (int nu = 0; nu < 4; ++nu) J[mu][nu] = (mu == nu);
        switch (s.transform) {
        case 0: break;
        case 1:
            for (int mu = 0; mu < 4; ++mu) for (int nu = 0; nu < 4; ++nu) J[mu][nu] = 0.;
            J[0][0] = 1.; J[1][1] = std::exp(X[1]); J[2][2] = 1.; J[3][3] = 1.;
            break;
        case 2:
            for (int mu = 0; mu < 4; ++mu) for (int nu = 0; nu < 4; ++nu) J[mu][nu] = 0.;
            J[0][0] = 1.;
            J[1][1] = std::exp(X[1]);
            J[2][2] = M_PI - (s.hslope - 1.)*M_PI*std::cos(2.*M_PI*X[2]);
            J[3][3] = 1.;
            break;
        default: {
            for (int mu = 0; mu < 4; ++mu) for (int nu = 0; nu < 4; ++nu) J[mu][nu] = 0.;
            const double hslope = s.hslope, mks_smooth = s.mks_smooth, startx1 = s.startx1;
            const double poly_xt = s.poly_xt, poly_alpha = s.poly_alpha;
            J[0][0] = 1.;
            J[1][1] = std::exp(X[1]);
            J[2][1] = -std::exp(mks_smooth * (startx1 - X[1])) * mks_smooth
                * (
                M_PI / 2. -
                M_PI * X[2]
                    + poly_norm * (2. * X[2] - 1.)
                        * (1
                            + (std::pow((-1. + 2 * X[2]) / poly_xt, poly_alpha))
                                / (1 + poly_alpha))
                    - 1. / 2. * (1. - hslope) * std::sin(2. * M_PI * X[2]));
            J[2][2] = M_PI + (1. - hslope) * M_PI * std::cos(2. * M_PI * X[2])
                + std::exp(mks_smooth * (startx1 - X[1]))
                    * (-M_PI
                        + 2. * poly_norm
                            * (1.
                                + std::pow((2. * X[2] - 1.) / poly_xt, poly_alpha)
                                    / (poly_alpha + 1.))
                        + (2. * poly_alpha * poly_norm * (2. * X[2] - 1.)
                            * std::pow((2. * X[2] - 1.) / poly_xt, poly_alpha - 1.))
                            / ((1. + poly_alpha) * poly_xt)
                        - (1. - hslope) * M_PI * std::cos(2. * M_PI * X[2]));
            J[3][3] = 1.;
            break;
        }
        }
    }
    // gcov_embed for each base system: coordinate_systems.hpp:80-84, 94-105, 120-150, 271-289
    void gcov_embed(const double Xe[4], double g[4][4]) const
    {
        const double a = s.a;
        switch (s.base) {
        case 0:
            for (int mu = 0; mu < 4; ++mu) for (int nu = 0; nu < 4; ++nu)
                g[mu][nu] = (mu == nu) - 2*(mu == 0 && nu == 0);
            break;
        case 1: {
            const double r = kmax(Xe[1], SMALL);
            const double th = excise(excise(Xe[2], 0.0, SMALL), M_PI, SMALL);
            const double sth = std::sin(th);
            for (int mu = 0; mu < 4; ++mu) for (int nu = 0; nu < 4; ++nu) g[mu][nu] = 0.;
            g[0][0] = 1.;  // sic: coordinate_systems.hpp:101
            g[1][1] = 1.;
            g[2][2] = r*r;
            g[3][3] = sth*sth*r*r;
            break;
        }
        case 2: {
            const double r = Xe[1];
            const double th = excise(excise(Xe[2], 0.0, SMALL), M_PI, SMALL);
            const double cth = std::cos(th);
            const double sth = std::sin(th);
            const double sin2 = sth*sth;
            const double rho2 = r*r + a*a*cth*cth;
            g[0][0] = -1. + 2.*r/rho2;
            g[0][1] = 2.*r/rho2;
            g[0][2] = 0.;
            g[0][3] = -2.*a*r*sin2/rho2;
            g[1][0] = 2.*r/rho2;
            g[1][1] = 1. + 2.*r/rho2;
            g[1][2] = 0.;
            g[1][3] = -a*sin2*(1. + 2.*r/rho2);
            g[2][0] = 0.;
            g[2][1] = 0.;
            g[2][2] = rho2;
            g[2][3] = 0.;
            g[3][0] = -2.*a*r*sin2/rho2;
            g[3][1] = -a*sin2*(1. + 2.*r/rho2);
            g[3][2] = 0.;
            g[3][3] = sin2*(rho2 + a*a*sin2*(1. + 2.*r/rho2));
            break;
        }
        default: {
            const double r = Xe[1];
            const double th = excise(excise(Xe[2], 0.0, SMALL), M_PI, SMALL);
            const double cth = std::cos(th), sth = std::sin(th);
            const double sin2 = sth*sth;
            const double a2 = a*a;
            const double r2 = r*r;
            const double mmu = 1. + a2*cth*cth/r2;
            for (int mu = 0; mu < 4; ++mu) for (int nu = 0; nu < 4; ++nu) g[mu][nu] = 0.;
            g[0][0] = -(1. - 2./(r*mmu));
            g[0][3] = -2.*a*sin2/(r*mmu);
            g[1][1] = mmu/(1. - 2./r + a2/r2);
            g[2][2] = r2*mmu;
            g[3][0] = -2.*a*sin2/(r*mmu);
            g[3][3] = sin2*(r2 + a2 + 2.*a2*sin2/(r*mmu));
            break;
        }
        }
    }
    // coordinate_embedding.hpp:488-500 (cov_tensor_to_native) and 503-514 (gcov_native)
    void gcov_native(const double X[4], double g[4][4]) const
    {
        double gem[4][4], Xe[4], J[4][4];
        coord_to_embed(X, Xe);
        gcov_embed(Xe, gem);
        dxdX(X, J);
        for (int mu = 0; mu < 4; ++mu) for (int nu = 0; nu < 4; ++nu) {
            g[mu][nu] = 0;
            for (int lam = 0; lam < 4; lam++)
                for (int kap = 0; kap < 4; kap++)
                    g[mu][nu] += gem[lam][kap]*J[lam][mu]*J[kap][nu];
        }
    }
    double r_of(const double X[4]) const   // coordinate_embedding.hpp:362-373
    {
        double Xe[4];
        coord_to_embed(X, Xe);
        if (spherical()) return Xe[1];
        return std::sqrt(Xe[1]*Xe[1] + Xe[2]*Xe[2] + Xe[3]*Xe[3]);
    }
};

// matrix.hpp:56-115
static inline double MINOR(const double m[16], int r0, int r1, int r2, int c0, int c1, int c2)
{
    return m[4*r0+c0]*(m[4*r1+c1]*m[4*r2+c2] - m[4*r2+c1]*m[4*r1+c2]) -
           m[4*r0+c1]*(m[4*r1+c0]*m[4*r2+c2] - m[4*r2+c0]*m[4*r1+c2]) +
           m[4*r0+c2]*(m[4*r1+c0]*m[4*r2+c1] - m[4*r2+c0]*m[4*r1+c1]);
}
static double invert(const double* m, double* o)
{
    o[ 0] =  MINOR(m,1,2,3,1,2,3); o[ 1] = -MINOR(m,0,2,3,1,2,3);
    o[ 2] =  MINOR(m,0,1,3,1,2,3); o[ 3] = -MINOR(m,0,1,2,1,2,3);
    o[ 4] = -MINOR(m,1,2,3,0,2,3); o[ 5] =  MINOR(m,0,2,3,0,2,3);
    o[ 6] = -MINOR(m,0,1,3,0,2,3); o[ 7] =  MINOR(m,0,1,2,0,2,3);
    o[ 8] =  MINOR(m,1,2,3,0,1,3); o[ 9] = -MINOR(m,0,2,3,0,1,3);
    o[10] =  MINOR(m,0,1,3,0,1,3); o[11] = -MINOR(m,0,1,2,0,1,3);
    o[12] = -MINOR(m,1,2,3,0,1,2); o[13] =  MINOR(m,0,2,3,0,1,2);
    o[14] = -MINOR(m,0,1,3,0,1,2); o[15] =  MINOR(m,0,1,2,0,1,2);
    const double det = m[0]*MINOR(m,1,2,3,1,2,3) - m[1]*MINOR(m,1,2,3,0,2,3) +
                       m[2]*MINOR(m,1,2,3,0,1,3) - m[3]*MINOR(m,1,2,3,0,1,2);
    const double inv_det = 1. / det;
    for (int i = 0; i < 16; ++i) o[i] *= inv_det;
    return det;
}
// coordinate_embedding.hpp:297-301
static double gcon_from_gcov(const double g[4][4], double gc[4][4])
{
    const double gdet = invert(&g[0][0], &gc[0][0]);
    return std::sqrt(std::fabs(gdet));
}
// coordinate_embedding.hpp:526-572
static void conn_native(const Coords& C, const double X[4], double delta, double conn[4][4][4])
{
    double tmp[4][4][4], gcon[4][4], gcov[4][4], Xh[4], Xl[4], gh[4][4], gl[4][4];
    for (int nu = 0; nu < 4; nu++) {
        for (int mu = 0; mu < 4; ++mu) Xl[mu] = X[mu] - delta*(mu == nu);
        for (int mu = 0; mu < 4; ++mu) Xh[mu] = X[mu] + delta*(mu == nu);
        C.gcov_native(Xh, gh);
        C.gcov_native(Xl, gl);
        for (int lam = 0; lam < 4; lam++)
            for (int kap = 0; kap < 4; kap++)
                conn[lam][kap][nu] = (gh[lam][kap] - gl[lam][kap]) / (Xh[nu] - Xl[nu]);
    }
    for (int lam = 0; lam < 4; lam++)
        for (int nu = 0; nu < 4; nu++)
            for (int mu = 0; mu < 4; mu++)
                tmp[lam][nu][mu] = 0.5 * (conn[nu][lam][mu] + conn[mu][lam][nu] - conn[mu][nu][lam]);
    C.gcov_native(X, gcov);
    gcon_from_gcov(gcov, gcon);
    for (int lam = 0; lam < 4; lam++)
        for (int nu = 0; nu < 4; nu++)
            for (int mu = 0; mu < 4; mu++) {
                conn[lam][nu][mu] = 0.;
                for (int kap = 0; kap < 4; kap++)
                    conn[lam][nu][mu] += gcon[lam][kap] * tmp[kap][nu][mu];
            }
}

// ---------------------------------------------------------------- block
struct Block {
    Config c;
    Coords C;
    int ndim, n1, n2, n3;
    int is, ie, js, je, ks, ke;
    size_t N;
    int nv;
    // geometry caches (GRCoordinates layout)
    std::vector<double> gcov, gcon, gdet, conn, gdet_conn;
    std::vector<double> rcen;   // r at cell centres (j,i): floors use G.r(k,j,i)

    void init(const Config& cfg, const CoordSpec& cs)
    {
        c = cfg; C.s = cs; C.init();
        ndim = 1 + (c.nx2 > 1) + (c.nx3 > 1);
        n1 = c.nx1 + 2*c.ng;
        n2 = (c.nx2 > 1) ? c.nx2 + 2*c.ng : 1;
        n3 = (c.nx3 > 1) ? c.nx3 + 2*c.ng : 1;
        is = c.ng; ie = c.ng + c.nx1 - 1;
        js = (c.nx2 > 1) ? c.ng : 0; je = js + c.nx2 - 1;
        ks = (c.nx3 > 1) ? c.ng : 0; ke = ks + c.nx3 - 1;
        N = (size_t)n1*n2*n3;
        nv = c.nvar;
    }
    inline size_t id(int k, int j, int i) const { return ((size_t)k*n2 + j)*n1 + i; }

    // Parthenon UniformCartesian (unvendored): Xf = xmin_entire + i dx, Xc = xmin_entire + (i+1/2) dx,
    // xmin_entire = block xmin - nghost dx in active directions.
    double Xf(int d, int idx) const
    {
        if (d == 1) return (c.x1min - c.ng*c.dx1) + idx*c.dx1;
        if (d == 2) return (c.x2min - ((c.nx2 > 1) ? c.ng : 0)*c.dx2) + idx*c.dx2;
        return (c.x3min - ((c.nx3 > 1) ? c.ng : 0)*c.dx3) + idx*c.dx3;
    }
    double Xc(int d, int idx) const
    {
        if (d == 1) return (c.x1min - c.ng*c.dx1) + (idx + 0.5)*c.dx1;
        if (d == 2) return (c.x2min - ((c.nx2 > 1) ? c.ng : 0)*c.dx2) + (idx + 0.5)*c.dx2;
        return (c.x3min - ((c.nx3 > 1) ? c.ng : 0)*c.dx3) + (idx + 0.5)*c.dx3;
    }
    double Dx(int d) const { return d == 1 ? c.dx1 : (d == 2 ? c.dx2 : c.dx3); }
    // gr_coordinates.hpp:184-225
    void coord(int k, int j, int i, int loc, double X[4]) const
    {
        X[0] = 0;
        switch (loc) {
        case face1:  X[1] = Xf(1, i); X[2] = Xc(2, j); X[3] = Xc(3, k); break;
        case face2:  X[1] = Xc(1, i); X[2] = Xf(2, j); X[3] = Xc(3, k); break;
        case face3:  X[1] = Xc(1, i); X[2] = Xc(2, j); X[3] = Xf(3, k); break;
        case center: X[1] = Xc(1, i); X[2] = Xc(2, j); X[3] = Xc(3, k); break;
        case corner: X[1] = Xf(1, i); X[2] = Xf(2, j); X[3] = Xf(3, k); break;
        case outer_half: X[1] = Xc(1, i); X[2] = (Xc(2, j) + Xf(2, j+1)) / 2; X[3] = Xc(3, k); break;
        default:     X[1] = Xc(1, i); X[2] = (Xc(2, j) + Xf(2, j)) / 2; X[3] = Xc(3, k); break;
        }
    }

    // gr_coordinates.cpp:96-205 with connection_average_points = 1 (the default)
    void build_geometry()
    {
        const int G1 = n1 + 1, G2 = n2 + 1;
        gcov.assign((size_t)NLOC*G2*G1*16, 0.);
        gcon.assign((size_t)NLOC*G2*G1*16, 0.);
        gdet.assign((size_t)NLOC*G2*G1, 0.);
        conn.assign((size_t)n2*n1*64, 0.);
        gdet_conn.assign((size_t)n2*n1*64, 0.);
        rcen.assign((size_t)n2*n1, 0.);
        for (int j = 0; j < G2; ++j) for (int i = 0; i < G1; ++i) {
            for (int loc = 0; loc < NLOC; ++loc) {
                if ((loc == center || loc == face3) && (i >= n1 || j >= n2)) continue;
                double X[4];
                coord(0, j, i, loc, X);
                double gl[4][4], gc[4][4];
                C.gcov_native(X, gl);
                const double gd = gcon_from_gcov(gl, gc);
                const size_t g = ((size_t)loc*G2 + j)*G1 + i;
                // averaging over one point: 0 + x/1 is exact
                gdet[g] = gd;
                for (int mu = 0; mu < 4; ++mu) for (int nu = 0; nu < 4; ++nu) {
                    gcov[g*16 + mu*4 + nu] = gl[mu][nu];
                    gcon[g*16 + mu*4 + nu] = gc[mu][nu];
                }
                if (loc == center) {
                    double cn[4][4][4];
                    conn_native(C, X, 1.e-8, cn);      // gr_coordinates.cpp:49,158
                    const size_t cg = ((size_t)j*n1 + i)*64;
                    for (int mu = 0; mu < 4; ++mu) for (int nu = 0; nu < 4; ++nu) for (int lam = 0; lam < 4; ++lam) {
                        conn[cg + mu*16 + nu*4 + lam] = cn[mu][nu][lam];
                        gdet_conn[cg + mu*16 + nu*4 + lam] = gd*cn[mu][nu][lam] / 1;
                    }
                    rcen[(size_t)j*n1 + i] = C.r_of(X);
                }
            }
        }
    }
    inline size_t gi(int loc, int j, int i) const { return ((size_t)loc*(n2+1) + j)*(n1+1) + i; }
    inline double Gcov(int loc, int j, int i, int mu, int nu) const { return gcov[gi(loc,j,i)*16 + mu*4 + nu]; }
    inline double Gcon(int loc, int j, int i, int mu, int nu) const { return gcon[gi(loc,j,i)*16 + mu*4 + nu]; }
    inline double Gdet(int loc, int j, int i) const { return gdet[gi(loc,j,i)]; }
    inline double GdetConn(int j, int i, int mu, int nu, int lam) const
    { return gdet_conn[((size_t)j*n1 + i)*64 + mu*16 + nu*4 + lam]; }
    // gr_coordinates.hpp:227-238
    void lower(const double* vcon, double* vcov, int j, int i, int loc) const
    {
        for (int mu = 0; mu < 4; ++mu) vcov[mu] = 0;
        for (int mu = 0; mu < 4; ++mu) for (int nu = 0; nu < 4; ++nu) vcov[mu] += Gcov(loc, j, i, mu, nu) * vcon[nu];
    }
    void raise(const double* vcov, double* vcon, int j, int i, int loc) const
    {
        for (int mu = 0; mu < 4; ++mu) vcon[mu] = 0;
        for (int mu = 0; mu < 4; ++mu) for (int nu = 0; nu < 4; ++nu) vcon[mu] += Gcon(loc, j, i, mu, nu) * vcov[nu];
    }
};

// ---------------------------------------------------------------- reconstruction
// reconstruction.hpp:46-56 and 106-204, 351-381
static const double WENO_EPS = 1.e-26;
static inline double mc(double dm, double dp)
{
    const double r = (std::fabs(dp) > 0. ? dm/dp : 2.0);
    return kmax(0.0, kmin(2.0, kmin(2*r, 0.5*(1+r))));
}
// Single-zone reconstruction: lout = value at the left face of the zone, rout = at the right face
// reconstruction.hpp:58-63 (mc with a limiter coefficient) and 66-71 (MINMOD, Median)
static inline double mc_alpha(double dm, double dp, double alpha)
{
    const double dc = (dm * dp > 0.0) * 0.5 * (dm + dp);
    return std::copysign(std::min(std::fabs(dc), alpha * std::min(std::fabs(dm), std::fabs(dp))), dc);
}
static inline double minmod(double a, double b) { return a * b > 0.0 ? (std::fabs(a) < std::fabs(b) ? a : b) : 0.0; }
static inline double median(double a, double b, double c) { return a + minmod(b - a, c - a); }

// reconstruction.hpp:284-325
static double mp5_subcalc(double Fjm2, double Fjm1, double Fj, double Fjp1, double Fjp2)
{
    const double alpha = 4.0, epsm = 1.e-12;
    double f = 2.0 * Fjm2 - 13.0 * Fjm1 + 47.0 * Fj + 27.0 * Fjp1 - 3.0 * Fjp2;
    f /= 60.0;
    const double fMP = Fj + minmod(Fjp1 - Fj, alpha * (Fj - Fjm1));
    if ((f - Fj) * (f - fMP) <= epsm) return f;
    const double d2m = Fjm2 + Fj - 2.0 * Fjm1;
    const double d2 = Fjm1 + Fjp1 - 2.0 * Fj;
    const double d2p = Fj + Fjp2 - 2.0 * Fjp1;
    double scrh1 = minmod(4.0 * d2 - d2p, 4.0 * d2p - d2);
    double scrh2 = minmod(d2, d2p);
    const double dMMp = minmod(scrh1, scrh2);
    scrh1 = minmod(4.0 * d2m - d2, 4.0 * d2 - d2m);
    scrh2 = minmod(d2, d2m);
    const double dMMm = minmod(scrh1, scrh2);
    const double fUL = Fj + alpha * (Fj - Fjm1);
    const double fAV = 0.5 * (Fj + Fjp1);
    const double fMD = fAV - 0.5 * dMMp;
    const double fLC = 0.5 * (3.0 * Fj - Fjm1) + 4.0 / 3.0 * dMMm;
    scrh1 = kmin(kmin(Fj, Fjp1), fMD);
    scrh2 = kmin(kmin(Fj, fUL), fLC);
    const double mn = kmax(scrh1, scrh2);
    scrh1 = kmax(kmax(Fj, Fjp1), fMD);
    scrh2 = kmax(kmax(Fj, fUL), fLC);
    const double mx = kmin(scrh1, scrh2);
    return median(f, mn, mx);
}

static inline double sgn(double x) { return (x < 0.0) ? -1.0 : 1.0; }

static void recon_zone(int recon, double x1, double x2, double x3, double x4, double x5, double& lout, double& rout)
{
    switch (recon) {
    case RECON_LINEAR_VL: {
        // Parthenon PiecewiseLinear, simplified van Leer limiter on a uniform grid
        const double dql = x3 - x2, dqr = x4 - x3;
        const double dq2 = dql * dqr;
        double dqm = 0.0;
        if (dq2 > 0.0) dqm = 2.0 * dq2 / (dql + dqr);
        rout = x3 + 0.5 * dqm;
        lout = x3 - 0.5 * dqm;
        break;
    }
    case RECON_WENO5_LINEAR: {      // reconstruction.hpp:209-268
        const double w5alpha[3][3] = {{1.0 / 3.0, -7.0 / 6.0, 11.0 / 6.0},
                                      {-1.0 / 6.0, 5.0 / 6.0, 1.0 / 3.0},
                                      {1.0 / 3.0, 5.0 / 6.0, -1.0 / 6.0}};
        const double w5gamma[3] = {0.1, 0.6, 0.3};
        const double eps = 1e-100, thirteen_thirds = 13.0 / 3.0;
        double a = x1 - 2 * x2 + x3;
        double b = x1 - 4.0 * x2 + 3.0 * x3;
        double beta0 = thirteen_thirds * a * a + b * b + eps;
        a = x2 - 2.0 * x3 + x4;
        b = x4 - x2;
        double beta1 = thirteen_thirds * a * a + b * b + eps;
        a = x3 - 2.0 * x4 + x5;
        b = x5 - 4.0 * x4 + 3.0 * x3;
        double beta2 = thirteen_thirds * a * a + b * b + eps;
        const double tau5 = std::fabs(beta2 - beta0);
        beta0 = (beta0 + tau5) / beta0;
        beta1 = (beta1 + tau5) / beta1;
        beta2 = (beta2 + tau5) / beta2;
        double w0 = w5gamma[0] * beta0 + eps, w1 = w5gamma[1] * beta1 + eps, w2 = w5gamma[2] * beta2 + eps;
        double wsum = 1.0 / (w0 + w1 + w2);
        rout = w0 * (w5alpha[0][0] * x1 + w5alpha[0][1] * x2 + w5alpha[0][2] * x3);
        rout += w1 * (w5alpha[1][0] * x2 + w5alpha[1][1] * x3 + w5alpha[1][2] * x4);
        rout += w2 * (w5alpha[2][0] * x3 + w5alpha[2][1] * x4 + w5alpha[2][2] * x5);
        rout *= wsum;
        const double alpha_r = 3.0 * wsum * w0 * w1 * w2 /
                               (w5gamma[2] * w0 * w1 + w5gamma[1] * w0 * w2 + w5gamma[0] * w1 * w2) + eps;
        w0 = w5gamma[0] * beta2 + eps; w1 = w5gamma[1] * beta1 + eps; w2 = w5gamma[2] * beta0 + eps;
        wsum = 1.0 / (w0 + w1 + w2);
        lout = w0 * (w5alpha[0][0] * x5 + w5alpha[0][1] * x4 + w5alpha[0][2] * x3);
        lout += w1 * (w5alpha[1][0] * x4 + w5alpha[1][1] * x3 + w5alpha[1][2] * x2);
        lout += w2 * (w5alpha[2][0] * x3 + w5alpha[2][1] * x2 + w5alpha[2][2] * x1);
        lout *= wsum;
        const double alpha_l = 3.0 * wsum * w0 * w1 * w2 /
                               (w5gamma[2] * w0 * w1 + w5gamma[1] * w0 * w2 + w5gamma[0] * w1 * w2) + eps;
        double dq = x4 - x3;
        dq = mc_alpha(x3 - x2, dq, 2.0);
        const double alpha_lin = 2.0 * alpha_r * alpha_l / (alpha_r + alpha_l);
        rout = alpha_lin * rout + (1.0 - alpha_lin) * (x3 + 0.5 * dq);
        lout = alpha_lin * lout + (1.0 - alpha_lin) * (x3 - 0.5 * dq);
        break;
    }
    case RECON_MP5:
        lout = mp5_subcalc(x5, x4, x3, x2, x1);
        rout = mp5_subcalc(x1, x2, x3, x4, x5);
        break;
    case RECON_PPMX: {              // reconstruction.hpp:403-495
        const double q_im2 = x1, q_im1 = x2, q_i = x3, q_ip1 = x4, q_ip2 = x5;
        double qlv = (7.*(q_i + q_im1) - (q_im2 + q_ip1))/12.0;
        double qrv = (7.*(q_i + q_ip1) - (q_im1 + q_ip2))/12.0;
        double d2qc = 3.0*((q_im1 + q_i) - 2.0*qlv);
        double d2ql = (q_im2 + q_i  ) - 2.0*q_im1;
        double d2qr = (q_im1 + q_ip1) - 2.0*q_i;
        double d2qlim = 0.0;
        double lim_slope = std::min(std::fabs(d2ql), std::fabs(d2qr));
        if (d2qc > 0.0 && d2ql > 0.0 && d2qr > 0.0) d2qlim = sgn(d2qc)*std::min(1.25*lim_slope, std::fabs(d2qc));
        if (d2qc < 0.0 && d2ql < 0.0 && d2qr < 0.0) d2qlim = sgn(d2qc)*std::min(1.25*lim_slope, std::fabs(d2qc));
        if (((q_im1 - qlv)*(q_i - qlv)) > 0.0) qlv = 0.5*(q_i + q_im1) - d2qlim/6.0;
        d2qc = 3.0*((q_i + q_ip1) - 2.0*qrv);
        d2ql = d2qr;
        d2qr = (q_i + q_ip2) - 2.0*q_ip1;
        d2qlim = 0.0;
        lim_slope = std::min(std::fabs(d2ql), std::fabs(d2qr));
        if (d2qc > 0.0 && d2ql > 0.0 && d2qr > 0.0) d2qlim = sgn(d2qc)*std::min(1.25*lim_slope, std::fabs(d2qc));
        if (d2qc < 0.0 && d2ql < 0.0 && d2qr < 0.0) d2qlim = sgn(d2qc)*std::min(1.25*lim_slope, std::fabs(d2qc));
        if (((q_i - qrv)*(q_ip1 - qrv)) > 0.0) qrv = 0.5*(q_i + q_ip1) - d2qlim/6.0;
        const double qa = (qrv - q_i)*(q_i - qlv);
        const double qb = (q_im1 - q_i)*(q_i - q_ip1);
        if (qa <= 0.0 || qb <= 0.0) {
            const double d2q = 6.0*(qlv + qrv - 2.0*q_i);
            const double c2 = (q_im1 + q_ip1) - 2.0*q_i;
            const double l2 = (q_im2 + q_i  ) - 2.0*q_im1;
            const double r2 = (q_i   + q_ip2) - 2.0*q_ip1;
            d2qlim = 0.0;
            lim_slope = std::min(std::fabs(l2), std::fabs(r2));
            lim_slope = std::min(std::fabs(c2), lim_slope);
            if (c2 > 0.0 && l2 > 0.0 && r2 > 0.0 && d2q > 0.0) d2qlim = sgn(d2q)*std::min(1.25*lim_slope, std::fabs(d2q));
            if (c2 < 0.0 && l2 < 0.0 && r2 < 0.0 && d2q < 0.0) d2qlim = sgn(d2q)*std::min(1.25*lim_slope, std::fabs(d2q));
            double rho = 0.0;
            if (std::fabs(d2q) > (1.0e-12)*std::max(std::fabs(q_im1), std::max(std::fabs(q_i), std::fabs(q_ip1))))
                rho = d2qlim/d2q;
            qlv = q_i + (qlv - q_i)*rho;
            qrv = q_i + (qrv - q_i)*rho;
        } else {
            const double qc = qrv - q_i;
            const double qd = qlv - q_i;
            if (std::fabs(qc) >= 2.0*std::fabs(qd)) qrv = q_i - 2.0*qd;
            if (std::fabs(qd) >= 2.0*std::fabs(qc)) qlv = q_i - 2.0*qc;
        }
        lout = qlv; rout = qrv;
        break;
    }
    case RECON_DONOR:
        rout = x3; lout = x3;
        break;
    case RECON_MC: {
        const double dq = mc(x3 - x2, x4 - x3)*(x4 - x3);
        rout = x3 + 0.5*dq;
        lout = x3 - 0.5*dq;
        break;
    }
    case RECON_WENO5: {
        double beta[3], c1, c2;
        c1 = x1 - 2.*x2 + x3; c2 = x1 - 4.*x2 + 3.*x3;
        beta[0] = (13./12.)*c1*c1 + (1./4.)*c2*c2;
        c1 = x2 - 2.*x3 + x4; c2 = x4 - x2;
        beta[1] = (13./12.)*c1*c1 + (1./4.)*c2*c2;
        c1 = x3 - 2.*x4 + x5; c2 = x5 - 4.*x4 + 3.*x3;
        beta[2] = (13./12.)*c1*c1 + (1./4.)*c2*c2;
        double den[3] = {WENO_EPS + beta[0], WENO_EPS + beta[1], WENO_EPS + beta[2]};
        den[0] *= den[0]; den[1] *= den[1]; den[2] *= den[2];
        double wtr[3] = {(1./16.)/den[0], (5./8. )/den[1], (5./16.)/den[2]};
        double Wr = wtr[0] + wtr[1] + wtr[2];
        double wtl[3] = {(1./16.)/den[2], (5./8. )/den[1], (5./16.)/den[0]};
        double Wl = wtl[0] + wtl[1] + wtl[2];
        lout = ((3./8.)*x5 - (5./4.)*x4 + (15./8.)*x3)*(wtl[0] / Wl) +
                ((-1./8.)*x4 + (3./4.)*x3 + (3./8.)*x2)*(wtl[1] / Wl) +
                ((3./8.)*x3 + (3./4.)*x2 - (1./8.)*x1)*(wtl[2] / Wl);
        rout = ((3./8.)*x1 - (5./4.)*x2 + (15./8.)*x3)*(wtr[0] / Wr) +
                ((-1./8.)*x2 + (3./4.)*x3 + (3./8.)*x4)*(wtr[1] / Wr) +
                ((3./8.)*x3 + (3./4.)*x4 - (1./8.)*x5)*(wtr[2] / Wr);
        break;
    }
    default: {  // PPM
        const double q_im2 = x1, q_im1 = x2, q_i = x3, q_ip1 = x4, q_ip2 = x5;
        double qlv = (7.*(q_i + q_im1) - (q_im2 + q_ip1))/12.0;
        double qrv = (7.*(q_i + q_ip1) - (q_im1 + q_ip2))/12.0;
        qlv = kmax(qlv, kmin(q_i, q_im1));
        qlv = kmin(qlv, kmax(q_i, q_im1));
        qrv = kmax(qrv, kmin(q_i, q_ip1));
        qrv = kmin(qrv, kmax(q_i, q_ip1));
        double qc = qrv - q_i;
        double qd = qlv - q_i;
        if ((qc*qd) >= 0.0) {
            qlv = q_i;
            qrv = q_i;
        } else {
            if (std::fabs(qc) >= 2.0*std::fabs(qd)) qrv = q_i - 2.0*qd;
            if (std::fabs(qd) >= 2.0*std::fabs(qc)) qlv = q_i - 2.0*qc;
        }
        lout = qlv; rout = qrv;
        break;
    }
    }
}

// ---------------------------------------------------------------- GRMHD device functions
struct FourVectors { double ucon[4], ucov[4], bcon[4], bcov[4]; };   // types.hpp:90-95

// grmhd_functions.hpp:121-133 (local primitives)
static double lorentz_calc(const Block& B, const double* P, int j, int i, int loc)
{
    const double qsq = B.Gcov(loc, j, i, 1, 1) * P[2] * P[2] +
                       B.Gcov(loc, j, i, 2, 2) * P[3] * P[3] +
                       B.Gcov(loc, j, i, 3, 3) * P[4] * P[4] +
                       2. * (B.Gcov(loc, j, i, 1, 2) * P[2] * P[3] +
                             B.Gcov(loc, j, i, 1, 3) * P[2] * P[4] +
                             B.Gcov(loc, j, i, 2, 3) * P[3] * P[4]);
    return std::sqrt(1. + qsq);
}
// grmhd_functions.hpp:225-246
static void calc_4vecs(const Block& B, const double* P, bool has_b, int j, int i, int loc, FourVectors& D)
{
    const double gamma = lorentz_calc(B, P, j, i, loc);
    const double alpha = 1. / std::sqrt(-B.Gcon(loc, j, i, 0, 0));
    D.ucon[0] = gamma / alpha;
    for (int v = 0; v < 3; ++v) D.ucon[v+1] = P[2 + v] - gamma * alpha * B.Gcon(loc, j, i, 0, v+1);
    B.lower(D.ucon, D.ucov, j, i, loc);
    if (has_b) {
        D.bcon[0] = 0;
        for (int v = 0; v < 3; ++v) D.bcon[0] += P[5 + v] * D.ucov[v+1];
        for (int v = 0; v < 3; ++v) D.bcon[v+1] = (P[5 + v] + D.bcon[0] * D.ucon[v+1]) / D.ucon[0];
        B.lower(D.bcon, D.bcov, j, i, loc);
    } else {
        for (int mu = 0; mu < 4; ++mu) D.bcon[mu] = D.bcov[mu] = 0.;
    }
}
// grmhd_functions.hpp:51-60 (GRHD) and 142-155 (GRMHD)
static void calc_tensor(double rho, double u, double pgas, const FourVectors& D, int dir, bool has_b, double T[4])
{
    if (has_b) {
        const double bsq = dot4(D.bcon, D.bcov);
        const double eta = pgas + rho + u + bsq;
        const double ptot = pgas + 0.5 * bsq;
        for (int mu = 0; mu < 4; ++mu)
            T[mu] = eta * D.ucon[dir] * D.ucov[mu] + ptot * (dir == mu) - D.bcon[dir] * D.bcov[mu];
    } else {
        const double eta = pgas + rho + u;
        for (int mu = 0; mu < 4; ++mu)
            T[mu] = eta * D.ucon[dir] * D.ucov[mu] + pgas * (dir == mu);
    }
}
// flux_functions.hpp:116-178 (local form, GRMHD variables)
static void prim_to_flux(const Block& B, const double* P, const FourVectors& D, int j, int i, int dir,
                         double* flux, int loc)
{
    const double gam = B.c.gam;
    const bool has_b = B.nv > 5;
    const double gdet = B.Gdet(loc, j, i);
    flux[0] = P[0] * D.ucon[dir] * gdet;
    double T[4];
    calc_tensor(P[0], P[1], (gam - 1) * P[1], D, dir, has_b, T);
    flux[1] = T[0] * gdet + flux[0];
    flux[2] = T[1] * gdet;
    flux[3] = T[2] * gdet;
    flux[4] = T[3] * gdet;
    if (has_b) {
        if (dir == 0) {
            for (int v = 0; v < 3; ++v) flux[5 + v] = P[5 + v] * gdet;
        } else {
            for (int v = 0; v < 3; ++v) flux[5 + v] = (D.bcon[v+1] * D.ucon[dir] - D.bcon[dir] * D.ucon[v+1]) * gdet;
        }
    }
}
// flux_functions.hpp:368-439.  Note clip() results are discarded in the reference (:378, :409).
static void vchar(const Block& B, const double* P, const FourVectors& D, int j, int i, int loc, int dir,
                  double& cmax, double& cmin)
{
    const double gam = B.c.gam;
    const double ef  = P[0] + gam * P[1];
    const double cs2 = gam * (gam - 1) * P[1] / ef;
    double cms2;
    if (B.nv > 5) {
        const double bsq = dot4(D.bcon, D.bcov);
        const double va2 = bsq / (bsq + ef);
        cms2 = cs2 + va2 - cs2 * va2;
    } else {
        cms2 = cs2;
    }
    double Bcov[4] = {1., 0., 0., 0.};
    double Acov[4] = {0., 0., 0., 0.}; Acov[dir] = 1.;
    double Acon[4], Bcon[4];
    B.raise(Acov, Acon, j, i, loc);
    B.raise(Bcov, Bcon, j, i, loc);
    const double Asq = dot4(Acon, Acov);
    const double Bsq = dot4(Bcon, Bcov);
    const double Au  = dot4(Acov, D.ucon);
    const double Bu  = dot4(Bcov, D.ucon);
    const double AB  = dot4(Acon, Bcov);
    const double A  = Bu*Bu - (Bsq + Bu*Bu) * cms2;
    const double Bq = 2. * (Au*Bu - (AB + Au*Bu) * cms2);
    const double Cq = Au*Au - (Asq + Au*Au) * cms2;
    const double discr = std::sqrt(kmax(Bq * Bq - 4. * A * Cq, 0.));
    const double vp = -(-Bq + discr) / (2. * A);
    const double vm = -(-Bq - discr) / (2. * A);
    cmax = kmax(vp, vm);
    cmin = kmin(vp, vm);
}
// flux.hpp:110-121
static inline double llf(double fL, double fR, double cmax, double cmin, double Ul, double Ur)
{
    const double ctop = kmax(cmax, cmin);
    return 0.5 * (fL + fR - ctop * (Ur - Ul));
}
static inline double hlle(double fL, double fR, double cmax, double cmin, double Ul, double Ur)
{
    return (cmax*fL + cmin*fR - cmax*cmin*(Ur - Ul)) / (cmax + cmin);
}

// floors_functions.hpp:320-354 (local form; loc ignored for r as in the reference, which uses G.r(0,j,i))
static int apply_geo_floors_local(const Block& B, double* P, int j, int i)
{
    // the inner prescription inside floors_switch_r (floors_functions.hpp:307-308)
    const Prescription& f = (B.c.floors.radius_dependent_floors && B.rcen[(size_t)j*B.n1 + i] < B.c.floors.floors_switch_r)
                                ? B.c.floors_inner : B.c.floors;
    double rhoflr_geom, uflr_geom;
    if (B.C.spherical()) {
        const double r = B.rcen[(size_t)j*B.n1 + i];
        const double rhoscal = (f.use_r_char) ? 1. / ((r*r) * (1 + r / f.r_char)) : 1. / std::sqrt(r*r*r);
        rhoflr_geom = kmax(f.rho_min_geom * rhoscal, f.rho_min_const);
        uflr_geom   = kmax(f.u_min_geom * std::pow(rhoscal, B.c.gam), f.u_min_const);
    } else {
        rhoflr_geom = f.rho_min_const;
        uflr_geom   = f.u_min_const;
    }
    int fflag = 0;
    fflag |= (rhoflr_geom > P[0]) * 4096;
    fflag |= (uflr_geom > P[1]) * 8192;
    P[0] += kmax(0., rhoflr_geom - P[0]);
    P[1] += kmax(0., uflr_geom - P[1]);
    return fflag;
}

// ---------------------------------------------------------------- GetFlux
// get_flux.hpp:60-373.  Faces are computed on the range every consumer needs:
// face direction [s, e+1], transverse directions [s-1, e+1] (the reference's range is a superset).
static void get_flux(const Block& B, int dir, const double* P, double* F, double* cmaxo, double* cmino)
{
    const int nv = B.nv, loc = dir - 1;   // loc_of(dir): face1/2/3 = 0/1/2
    const int d1 = (dir == 1), d2 = (dir == 2), d3 = (dir == 3);
    const int i0 = B.is - (B.ndim >= 1 && !d1 ? 1 : 0), i1 = B.ie + 1;
    const int j0 = (B.ndim >= 2) ? B.js - (d2 ? 0 : 1) : B.js, j1 = (B.ndim >= 2) ? B.je + 1 : B.je;
    const int k0 = (B.ndim >= 3) ? B.ks - (d3 ? 0 : 1) : B.ks, k1 = (B.ndim >= 3) ? B.ke + 1 : B.ke;
    const int si = d1, sj = d2 ? B.n1 : 0, sk = d3 ? B.n1*B.n2 : 0;
    const ptrdiff_t st = si + sj + (ptrdiff_t)sk;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = k0; k <= k1; ++k) for (int j = j0; j <= j1; ++j) for (int i = i0; i <= i1; ++i) {
        const size_t c = B.id(k, j, i);
        double Pl[8], Pr[8];
        // weno5 lowered to MC (reconstruction.hpp:694-771): X1 faces near the block's X1 edges (zones
        // [is-1, is+3] and [ie-2, ie+2] of ReconstructX1's range), or every face in rows j <= 6 and
        // j >= n2 - 6
        int rl = B.c.recon, rr = B.c.recon;
        if (B.c.recon == RECON_WENO5 && B.c.recon_lower == 1 && d1) {
            if (i - 1 <= B.is + 3 || i - 1 >= B.ie - 2) rl = RECON_MC;
            if (i <= B.is + 3 || i >= B.ie - 2) rr = RECON_MC;
        }
        if (B.c.recon == RECON_WENO5 && B.c.recon_lower == 2 && !(j > 6 && j < B.n2 - 6)) rl = rr = RECON_MC;
        for (int p = 0; p < nv; ++p) {
            const double* q = P + (size_t)p*B.N;
            double l, r;
            // Left state: right face of zone c-1 (ReconstructX1 ql(i+1) / ReconstructX{2,3}l reconstruct_right)
            recon_zone(rl, q[c - 3*st], q[c - 2*st], q[c - st], q[c], q[c + st], l, r);
            Pl[p] = r;
            // Right state: left face of zone c (qr(i) / reconstruct_left)
            recon_zone(rr, q[c - 2*st], q[c - st], q[c], q[c + st], q[c + 2*st], l, r);
            Pr[p] = l;
        }
        if (B.c.recon_floors || B.c.recon_fallback) {    // get_flux.hpp:174-199
            int hit = apply_geo_floors_local(B, Pl, j, i);
            hit |= apply_geo_floors_local(B, Pr, j, i);
            if (B.c.recon_fallback && hit) {
                for (int p = 0; p < nv; ++p) {
                    const double* q = P + (size_t)p*B.N;
                    double l, r;
                    recon_zone(RECON_PPM, q[c - 3*st], q[c - 2*st], q[c - st], q[c], q[c + st], l, r);
                    Pl[p] = r;
                    recon_zone(RECON_PPM, q[c - 2*st], q[c - st], q[c], q[c + st], q[c + 2*st], l, r);
                    Pr[p] = l;
                }
            }
        }
        FourVectors Dl, Dr;
        double Ul[8], Fl[8], Ur[8], Fr[8], cmaxL, cminL, cmaxR, cminR;
        calc_4vecs(B, Pl, nv > 5, j, i, loc, Dl);
        prim_to_flux(B, Pl, Dl, j, i, 0, Ul, loc);
        prim_to_flux(B, Pl, Dl, j, i, dir, Fl, loc);
        vchar(B, Pl, Dl, j, i, loc, dir, cmaxL, cminL);
        double cmax = kmax(0., cmaxL);
        double cmin = kmin(0., cminL);
        calc_4vecs(B, Pr, nv > 5, j, i, loc, Dr);
        prim_to_flux(B, Pr, Dr, j, i, 0, Ur, loc);
        prim_to_flux(B, Pr, Dr, j, i, dir, Fr, loc);
        vchar(B, Pr, Dr, j, i, loc, dir, cmaxR, cminR);
        cmax = kmax(cmax, cmaxR);
        cmin = -kmin(cmin, cminR);
        cmaxo[c] = cmax; cmino[c] = cmin;
        for (int p = 0; p < nv; ++p)
            F[(size_t)p*B.N + c] = B.c.riemann ? hlle(Fl[p], Fr[p], cmax, cmin, Ul[p], Ur[p])
                                               : llf(Fl[p], Fr[p], cmax, cmin, Ul[p], Ur[p]);
    }
}

// ---------------------------------------------------------------- FixFlux
// b_flux_ct.cpp:372-418 (ZeroBoundaryFlux, X2 faces only: fix_polar_flux)
static void zero_boundary_flux_x2(const Block& B, double* F1, double* F2, double* F3, bool inner)
{
    if (B.ndim < 2) return;
    const size_t N = B.N;
    const int ibs_s = B.is - 1, ibs_e = B.ie + 1;
    const int kbs_s = B.ks - (B.ndim > 2), kbs_e = B.ke + (B.ndim > 2);
    const int j = inner ? B.js : B.je + 1;
    for (int k = kbs_s; k <= kbs_e; ++k) for (int i = ibs_s; i <= ibs_e; ++i) {
        F2[5*N + B.id(k, j, i)] = 0.;
        F2[7*N + B.id(k, j, i)] = 0.;
        if (inner) {
            F1[6*N + B.id(k, j-1, i)] = -F1[6*N + B.id(k, j, i)];
            if (B.ndim > 2) F3[6*N + B.id(k, j-1, i)] = -F3[6*N + B.id(k, j, i)];
        } else {
            F1[6*N + B.id(k, j, i)] = -F1[6*N + B.id(k, j-1, i)];
            if (B.ndim > 2) F3[6*N + B.id(k, j, i)] = -F3[6*N + B.id(k, j-1, i)];
        }
    }
}
// b_flux_ct.cpp:307-370
static void flux_ct(const Block& B, double* F1, double* F2, double* F3)
{
    if (B.ndim < 2) return;
    const size_t N = B.N;
    const int ndim = B.ndim;
    const int il_s = B.is, il_e = B.ie + 1, jl_s = B.js, jl_e = B.je + 1;
    const int kl_s = B.ks, kl_e = (ndim > 2) ? B.ke + 1 : B.ke;
    std::vector<double> emf(3*N, 0.);
    double* e1 = emf.data(); double* e2 = e1 + N; double* e3 = e2 + N;
    const size_t sj = B.n1, sk = (size_t)B.n1*B.n2;
    for (int k = kl_s; k <= kl_e; ++k) for (int j = jl_s; j <= jl_e; ++j) for (int i = il_s; i <= il_e; ++i) {
        const size_t c = B.id(k, j, i);
        if (ndim > 2) {
            e1[c] = 0.25 * (F2[7*N + c] + F2[7*N + c - sk] - F3[6*N + c] - F3[6*N + c - sj]);
            e2[c] = 0.25 * (F3[5*N + c] + F3[5*N + c - 1] - F1[7*N + c] - F1[7*N + c - sk]);
        }
        e3[c] = 0.25 * (F1[6*N + c] + F1[6*N + c - sj] - F2[5*N + c] - F2[5*N + c - 1]);
    }
    for (int k = B.ks; k <= B.ke; ++k) for (int j = B.js; j <= B.je; ++j) for (int i = il_s; i <= il_e; ++i) {
        const size_t c = B.id(k, j, i);
        F1[5*N + c] = 0.0;
        F1[6*N + c] = 0.5 * (e3[c] + e3[c + sj]);
        if (ndim > 2) F1[7*N + c] = -0.5 * (e2[c] + e2[c + sk]);
    }
    for (int k = B.ks; k <= B.ke; ++k) for (int j = jl_s; j <= jl_e; ++j) for (int i = B.is; i <= B.ie; ++i) {
        const size_t c = B.id(k, j, i);
        F2[5*N + c] = -0.5 * (e3[c] + e3[c + 1]);
        F2[6*N + c] = 0.0;
        if (ndim > 2) F2[7*N + c] = 0.5 * (e1[c] + e1[c + sk]);
    }
    if (ndim > 2) {
        for (int k = kl_s; k <= kl_e; ++k) for (int j = B.js; j <= B.je; ++j) for (int i = B.is; i <= B.ie; ++i) {
            const size_t c = B.id(k, j, i);
            F3[5*N + c] = 0.5 * (e2[c] + e2[c + 1]);
            F3[6*N + c] = -0.5 * (e1[c] + e1[c + sj]);
            F3[7*N + c] = 0.0;
        }
    }
}
// boundaries.cpp:611-690 (check_inflow flux limiting on X1, zero_flux on X2 poles)
// nvars: the variables whose fluxes the polar faces zero (8, or 10 with the EMHD slots)
static void boundaries_fix_flux(const Block& B, double* F[3], int nvars = 0)
{
    if (nvars <= 0) nvars = B.nv;
    const size_t N = B.N;
    for (int face = 0; face < 4; ++face) {
        const int bdir = face / 2 + 1;
        const bool binner = (face % 2) == 0;
        if (bdir > B.ndim) continue;
        if (!phys_face(B.c.bc[face])) continue;       // only global "user" boundaries
        // one-zone halo range, collapsed to the boundary face
        int is_ = B.is - 1, ie_ = B.ie + 1, js_ = B.js - (B.ndim > 1), je_ = B.je + (B.ndim > 1);
        int ks_ = B.ks - (B.ndim > 2), ke_ = B.ke + (B.ndim > 2);
        if (bdir == 1) is_ = ie_ = binner ? B.is : B.ie + 1;
        else if (bdir == 2) js_ = je_ = binner ? B.js : B.je + 1;
        const bool check_inflow = (face == 0 && B.c.check_inflow_inner_x1) || (face == 1 && B.c.check_inflow_outer_x1);
        const bool zero_flux = B.c.zero_polar_flux && bdir == 2;
        for (int k = ks_; k <= ke_; ++k) for (int j = js_; j <= je_; ++j) for (int i = is_; i <= ie_; ++i) {
            const size_t c = B.id(k, j, i);
            if (check_inflow) {
                double& f = F[bdir-1][c];
                f = binner ? kmin(f, 0.) : kmax(f, 0.);
            }
            if (zero_flux)
                for (int p = 0; p < nvars; ++p) F[bdir-1][(size_t)p*N + c] = 0.;
        }
    }
}

// ---------------------------------------------------------------- divergence and sources
// Parthenon FluxDivHelper (unvendored), called from kharma_driver.hpp:208-231
static void flux_divergence(const Block& B, double* F[3], double* dudt)
{
    const size_t N = B.N;
    const double a1 = B.c.dx2*B.c.dx3, a2 = B.c.dx1*B.c.dx3, a3 = B.c.dx1*B.c.dx2;
    const double vol = B.c.dx1*B.c.dx2*B.c.dx3;
    const size_t sj = B.n1, sk = (size_t)B.n1*B.n2;
#pragma omp parallel for collapse(2) schedule(static)
    for (int p = 0; p < B.nv; ++p)
    for (int k = B.ks; k <= B.ke; ++k) for (int j = B.js; j <= B.je; ++j) for (int i = B.is; i <= B.ie; ++i) {
        const size_t c = B.id(k, j, i), pc = (size_t)p*N + c;
        double du = (a1 * F[0][pc + 1] - a1 * F[0][pc]);
        if (B.ndim >= 2) du += a2 * F[1][pc + sj] - a2 * F[1][pc];
        if (B.ndim == 3) du += a3 * F[2][pc + sk] - a3 * F[2][pc];
        dudt[pc] = -du / vol;
    }
}
// flux.cpp:395-444
// The geometric source T^mu_lam gdet Gamma^lam_nu mu of one zone (flux.cpp:413-441) into new_du[4]
// (the UU and U1-U3 components)
static void geo_source_cell(const Block& B, const double* Pc, int j, int i, double new_du[4])
{
    FourVectors D;
    calc_4vecs(B, Pc, B.nv > 5, j, i, center, D);
    double Tmu[4] = {0};
    for (int x = 0; x < 4; ++x) new_du[x] = 0.;
    for (int mu = 0; mu < 4; ++mu) {
        calc_tensor(Pc[0], Pc[1], (B.c.gam - 1) * Pc[1], D, mu, B.nv > 5, Tmu);
        for (int nu = 0; nu < 4; ++nu)
            for (int lam = 0; lam < 4; ++lam)
                new_du[lam] += Tmu[nu] * B.GdetConn(j, i, nu, lam, mu);
    }
}

static void add_geo_source(const Block& B, const double* P, double* dudt)
{
    if (B.C.cart_minkowski()) return;
    const size_t N = B.N;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = B.ks; k <= B.ke; ++k) for (int j = B.js; j <= B.je; ++j) for (int i = B.is; i <= B.ie; ++i) {
        const size_t c = B.id(k, j, i);
        double Pc[8];
        for (int p = 0; p < B.nv; ++p) Pc[p] = P[(size_t)p*N + c];
        double new_du[4];
        geo_source_cell(B, Pc, j, i, new_du);
        dudt[1*N + c] += new_du[0];
        for (int v = 0; v < 3; ++v) dudt[(size_t)(2 + v)*N + c] += new_du[1 + v];
    }
}

// ---------------------------------------------------------------- P <-> U
// flux_functions.hpp:343-352 (Flux::p_to_u, global): 4-vectors at the centre, gdet at loc=center
static void p_to_u_cell(const Block& B, const double* P, double* U, size_t c, int j, int i)
{
    double Pc[8], Uc[8];
    for (int p = 0; p < B.nv; ++p) Pc[p] = P[(size_t)p*B.N + c];
    FourVectors D;
    calc_4vecs(B, Pc, B.nv > 5, j, i, center, D);
    prim_to_flux(B, Pc, D, j, i, 0, Uc, center);
    for (int p = 0; p < B.nv; ++p) U[(size_t)p*B.N + c] = Uc[p];
}
// flux_functions.hpp:354-363 / 312-328 (p_to_u_mhd: only rho, u, uvec conserved)
static void p_to_u_mhd_cell(const Block& B, const double* P, double* U, size_t c, int j, int i)
{
    double Pc[8], Uc[8];
    for (int p = 0; p < B.nv; ++p) Pc[p] = P[(size_t)p*B.N + c];
    FourVectors D;
    calc_4vecs(B, Pc, B.nv > 5, j, i, center, D);
    prim_to_flux(B, Pc, D, j, i, 0, Uc, center);
    for (int p = 0; p < 5; ++p) U[(size_t)p*B.N + c] = Uc[p];
}

// ---------------------------------------------------------------- 1D_W inversion
enum Status { success = 0, neg_input, max_iter, bad_ut, bad_gamma, neg_rho, neg_u, neg_rhou };  // invert_template.hpp:53
// onedw.hpp:49-67
static inline double lorentz_calc_w(double Bsq, double D, double QdB, double Qtsq, double Wp)
{
    const double QdBsq = QdB * QdB;
    const double W = Wp + D;
    const double W2 = W * W;
    const double WB = W + Bsq;
    const double utsq = -((W + WB) * QdBsq + W2 * Qtsq) / (QdBsq * (W + WB) + W2 * (Qtsq - WB * WB));
    if (utsq < -1.e-15 || utsq > 1.e7) return -1.;
    return std::sqrt(1. + std::fabs(utsq));
}
// onedw.hpp:72-84
static inline double err_eqn(double gam, double Bsq, double D, double Ep, double QdB, double Qtsq, double Wp, int& eflag)
{
    const double W = Wp + D;
    const double gamma = lorentz_calc_w(Bsq, D, QdB, Qtsq, Wp);
    if (gamma < 1) eflag = bad_ut;
    const double w = W / (gamma*gamma);
    const double rho = D / gamma;
    const double p = (w - rho) * (gam - 1) / gam;
    return -Ep + Wp - p + 0.5 * Bsq + 0.5 * (Bsq * Qtsq - QdB * QdB) / ((Bsq + W)*(Bsq + W));
}
// onedw.hpp:89-233.  U and P are the cell's conserved/primitive values; P is updated only on success.
static int u_to_p_onedw(const Block& B, const double* U, double* P, int j, int i, int loc, int max_iterations, double tol)
{
    const double gam = B.c.gam;
    if (U[0] <= 0.) return neg_input;
    const double alpha = 1./std::sqrt(-B.Gcon(loc, j, i, 0, 0));
    const double gdet = B.Gdet(loc, j, i);
    const double a_over_g = alpha / gdet;
    const double D = U[0] * a_over_g;
    double Bcon[4] = {0};
    if (B.nv > 5) {
        Bcon[1] = U[5] * a_over_g;
        Bcon[2] = U[6] * a_over_g;
        Bcon[3] = U[7] * a_over_g;
    }
    const double Qcov[4] = {(U[1] - U[0]) * a_over_g, U[2] * a_over_g, U[3] * a_over_g, U[4] * a_over_g};
    const double ncov[4] = {-alpha, 0., 0., 0.};
    double Bcov[4], Qcon[4], ncon[4];
    B.lower(Bcon, Bcov, j, i, loc);
    B.raise(Qcov, Qcon, j, i, loc);
    B.raise(ncov, ncon, j, i, loc);
    const double Bsq = dot4(Bcon, Bcov);
    const double QdB = dot4(Bcon, Qcov);
    const double Qdotn = dot4(Qcon, ncov);
    double Qtcon[4];
    for (int mu = 0; mu < 4; ++mu) Qtcon[mu] = Qcon[mu] + ncon[mu] * Qdotn;
    const double Qtsq = dot4(Qcon, Qcov) + Qdotn*Qdotn;
    const double Ep = -Qdotn - D;
    int eflag = success;
    double Wp, err;
    {
        const double gamma = lorentz_calc(B, P, j, i, loc);
        if (gamma < 1) return bad_ut;
        const double rho = P[0], u = P[1];
        Wp = (rho + u + (gam - 1) * u) * gamma * gamma - rho * gamma;
        err = err_eqn(gam, Bsq, D, Ep, QdB, Qtsq, Wp, eflag);
    }
    double dW;
    {
        const double Wpm = (1. - 1.e-5) * Wp;
        const double h = Wp - Wpm;
        const double Wpp = Wp + h;
        const double errm = err_eqn(gam, Bsq, D, Ep, QdB, Qtsq, Wpm, eflag);
        const double errp = err_eqn(gam, Bsq, D, Ep, QdB, Qtsq, Wpp, eflag);
        const double dedW = (errp - errm) / (Wpp - Wpm);
        const double dedW2 = (errp - 2. * err + errm) / (h*h);
        const double f = clip(0.5 * err * dedW2 / (dedW*dedW), -0.3, 0.3);
        dW = clip(-err / dedW / (1. - f), -0.5*Wp, 2.0*Wp);
    }
    double Wp1 = Wp;
    double err1 = err;
    Wp += dW;
    err = err_eqn(gam, Bsq, D, Ep, QdB, Qtsq, Wp, eflag);
    int iter = 0;
    for (iter = 0; iter < max_iterations; iter++) {
        dW = clip((Wp1 - Wp) * err / (err - err1), -0.5*Wp, 2.0*Wp);
        Wp1 = Wp;
        err1 = err;
        Wp += dW;
        if (std::fabs(dW / Wp) < tol) break;
        err = err_eqn(gam, Bsq, D, Ep, QdB, Qtsq, Wp, eflag);
        if (std::fabs(err / Wp) < tol) break;
    }
    if (iter == max_iterations) return max_iter;
    const double gamma = lorentz_calc_w(Bsq, D, QdB, Qtsq, Wp);
    if (gamma < 1) return bad_ut;
    const double rho = D / gamma;
    const double W = Wp + D;
    const double w = W / (gamma*gamma);
    const double p = (w - rho) * (gam - 1) / gam;
    const double u = w - (rho + p);
    if (rho < 0 && u < 0) return neg_rhou;
    else if (rho < 0) return neg_rho;
    else if (u < 0) return neg_u;
    P[0] = rho;
    P[1] = u;
    const double pre = (gamma / (W + Bsq));
    P[2] = pre * (Qtcon[1] + QdB * Bcon[1] / W);
    P[3] = pre * (Qtcon[2] + QdB * Bcon[2] / W);
    P[4] = pre * (Qtcon[3] + QdB * Bcon[3] / W);
    return success;
}

// ---------------------------------------------------------------- floors
// The prescription of zone (j, i): the inner one inside floors_switch_r with radius-dependent floors
// (floors_functions.hpp:56-57, 89-90; inverter.cpp:165-168)
static const Prescription& myfloors(const Block& B, int j, int i)
{
    return (B.c.floors.radius_dependent_floors && B.rcen[(size_t)j*B.n1 + i] < B.c.floors.floors_switch_r)
               ? B.c.floors_inner : B.c.floors;
}
// floors_functions.hpp:84-160
static int determine_floors(const Block& B, const double* P, int j, int i, double& rhoflr_max, double& uflr_max)
{
    const Prescription& f = myfloors(B, j, i);
    const double gam = B.c.gam;
    double rhoflr_geom, uflr_geom;
    if (B.C.spherical()) {
        const double r = B.rcen[(size_t)j*B.n1 + i];
        const double rhoscal = (f.use_r_char) ? 1. / ((r*r) * (1 + r / f.r_char)) : 1. / std::sqrt(r*r*r);
        rhoflr_geom = kmax(f.rho_min_geom * rhoscal, f.rho_min_const);
        uflr_geom   = kmax(f.u_min_geom * std::pow(rhoscal, gam), f.u_min_const);
    } else {
        rhoflr_geom = f.rho_min_const;
        uflr_geom   = f.u_min_const;
    }
    FourVectors D;
    calc_4vecs(B, P, B.nv > 5, j, i, center, D);
    const double bsq = dot4(D.bcon, D.bcov);
    const double rhoflr_b = bsq / f.bsq_over_rho_max;
    const double uflr_b   = bsq / f.bsq_over_u_max;
    uflr_max = kmax(uflr_geom, uflr_b);
    const double rho = P[0], u = P[1];
    int fflag = 0;
    if (!f.temp_adjust_u) {
        const double rhoflr_temp = kmax(u, uflr_max) / f.u_over_rho_max;
        fflag |= (rhoflr_temp > rho) * 512;
        rhoflr_max = kmax(kmax(rhoflr_geom, rhoflr_b), rhoflr_temp);
    } else {
        rhoflr_max = kmax(rhoflr_geom, rhoflr_b);
    }
    if (rhoflr_max > rho || uflr_max > u) {
        fflag |= (rhoflr_geom > rho) * 32;
        fflag |= (uflr_geom > u) * 64;
        fflag |= (rhoflr_b > rho) * 128;
        fflag |= (uflr_b > u) * 256;
    }
    if (lorentz_calc(B, P, j, i, center) > f.gamma_max) fflag |= 1024;
    if ((gam - 1.) * P[1] / std::pow(P[0], gam) > f.ktot_max) fflag |= 2048;
    if (f.temp_adjust_u && (P[1] / P[0] > f.u_over_rho_max)) fflag |= 512;
    return fflag;
}
// floors_functions.hpp:50-82
static void apply_ceilings(const Block& B, double* P, int j, int i)
{
    const Prescription& f = myfloors(B, j, i);
    const double gam = B.c.gam;
    const double gamma = lorentz_calc(B, P, j, i, center);
    const double ktot = (gam - 1.) * P[1] / std::pow(P[0], gam);
    if (gamma > f.gamma_max) {
        const double fr = std::sqrt((f.gamma_max*f.gamma_max - 1.) / (gamma*gamma - 1.));
        for (int v = 0; v < 3; ++v) P[2 + v] *= fr;
    }
    if (ktot > f.ktot_max) P[1] = f.ktot_max / ktot * P[1];
    if (f.temp_adjust_u && P[1] / P[0] > f.u_over_rho_max) P[1] = f.u_over_rho_max * P[0];
}
// floors_functions.hpp:174-179 (fluid) and 181-252 (drift)
static int apply_floors_frame(const Block& B, double* P, double* U, int j, int i, double rhoflr_max, double uflr_max)
{
    const double gam = B.c.gam;
    // mixed frames (floors_impl.hpp:84-106): by radius, or by min(rho, u)/b^2 before the floors
    int frame = B.c.floor_frame;
    if (frame == FRAME_MIXED_FLUID_NORMAL) {
        frame = (B.rcen[(size_t)j*B.n1 + i] > B.c.frame_switch_r) ? FRAME_FLUID : FRAME_NORMAL;
    } else if (frame == FRAME_MIXED_NORMAL_DRIFT) {
        FourVectors Dt;
        calc_4vecs(B, P, B.nv > 5, j, i, center, Dt);
        const double mag_switch = std::min(P[0], P[1]) / dot4(Dt.bcon, Dt.bcov);
        frame = (mag_switch < B.c.frame_switch_beta) ? FRAME_DRIFT : FRAME_NORMAL;
    }
    if (frame == FRAME_FLUID) {
        P[0] += kmax(0., rhoflr_max - P[0]);
        P[1] += kmax(0., uflr_max - P[1]);
        return 0;
    } else if (frame == FRAME_DRIFT) {
        const double lapse2 = 1. / (-B.Gcon(center, j, i, 0, 0));
        double beta[4] = {0};
        beta[1] = lapse2 * B.Gcon(center, j, i, 0, 1);
        beta[2] = lapse2 * B.Gcon(center, j, i, 0, 2);
        beta[3] = lapse2 * B.Gcon(center, j, i, 0, 3);
        const double rho = P[0];
        const double uu = P[1];
        const double pg = (gam - 1.) * uu;
        const double w_old = kmax(rho + uu + pg, SMALL);
        double Bcon[4] = {0}, Bcov[4] = {0};
        if (B.nv > 5) { Bcon[0] = 0; Bcon[1] = P[5]; Bcon[2] = P[6]; Bcon[3] = P[7]; }
        for (int mu = 0; mu < 4; ++mu) for (int nu = 0; nu < 4; ++nu) Bcov[mu] += B.Gcov(center, j, i, mu, nu) * Bcon[nu];
        const double Bsq = kmax(dot4(Bcon, Bcov), SMALL);
        const double B_mag = std::sqrt(Bsq);
        FourVectors D;
        calc_4vecs(B, P, B.nv > 5, j, i, center, D);
        double Qcov[4] = {0};
        Qcov[0] = w_old * D.ucon[0] * D.ucov[0] + pg;
        Qcov[1] = w_old * D.ucon[0] * D.ucov[1];
        Qcov[2] = w_old * D.ucon[0] * D.ucov[2];
        Qcov[3] = w_old * D.ucon[0] * D.ucov[3];
        const double QdotB = dot4(Bcon, Qcov);
        double vpar = QdotB / (B_mag * w_old * D.ucon[0]*D.ucon[0]);
        double ucon_dr[4] = {0};
        ucon_dr[0] = 1. / std::sqrt(1. / (D.ucon[0]*D.ucon[0]) + vpar*vpar);
        for (int mu = 0; mu < 4; ++mu) ucon_dr[mu] = D.ucon[mu] * (ucon_dr[0] / D.ucon[0]) - (vpar * Bcon[mu] * ucon_dr[0] / B_mag);
        P[0] = kmax(rho, rhoflr_max);
        P[1] = kmax(uu, uflr_max);
        const double pg_new = (gam - 1.) * P[1];
        const double w_new  = P[0] + P[1] + pg_new;
        const double x = (2. * QdotB) / (B_mag * w_new * ucon_dr[0]);
        vpar = x / (1 + std::sqrt(1 + x*x)) * (1. / ucon_dr[0]);
        D.ucon[0] = 1. / std::sqrt(1/(ucon_dr[0]*ucon_dr[0]) - vpar*vpar);
        for (int mu = 0; mu < 4; ++mu) D.ucon[mu] = ucon_dr[mu] * (D.ucon[0] / ucon_dr[0]) + (vpar * Bcon[mu] * D.ucon[0] / B_mag);
        B.lower(D.ucon, D.ucov, j, i, center);
        P[2] = D.ucon[1] + (beta[1] * D.ucon[0]);
        P[3] = D.ucon[2] + (beta[2] * D.ucon[0]);
        P[4] = D.ucon[3] + (beta[3] * D.ucon[0]);
        return 0;
    } else {
        // normal observer frame: floors_functions.hpp:254-289
        const double rho_add = kmax(0., rhoflr_max - P[0]);
        const double u_add   = kmax(0., uflr_max - P[1]);
        double Pa[8] = {rho_add, u_add, 0., 0., 0., 0., 0., 0.};
        FourVectors D;
        calc_4vecs(B, Pa, true, j, i, center, D);
        const double gdet = B.Gdet(center, j, i);
        const double rho_ut = rho_add * D.ucon[0] * gdet;
        double mhd[4];
        calc_tensor(rho_add, u_add, (gam - 1) * u_add, D, 0, true, mhd);
        double T[4];
        T[0] = mhd[0] * gdet + rho_ut;
        for (int v = 0; v < 3; ++v) T[1 + v] = mhd[1 + v] * gdet;
        P[0] += rho_add;
        P[1] += u_add;
        U[0] += rho_ut;
        U[1] += T[0];
        U[2] += T[1];
        U[3] += T[2];
        U[4] += T[3];
        return u_to_p_onedw(B, U, P, j, i, center, 8, 1e-8);
    }
}

// ---------------------------------------------------------------- Kastaun inversion
// inverter/kastaun.hpp:83-406 (Kastaun et al. 2021, as adapted from Phoebus and AthenaK): a master
// function of mu = 1/(h W) solved by the Illinois false-position method, first for a bracket (the
// auxiliary function, eq. 49) and then for the root (eq. 44), with the inverter floors applied
// inside the residual.  Returns the Inverter FFlag bits of the floors hit, or max_iter.
enum { FF_INVERTER_RHO = 16384, FF_INVERTER_U = 32768, FF_INVERTER_GAMMA = 65536, FF_INVERTER_U_MAX = 131072 };

struct KastaunResidual {            // kastaun.hpp:83-218
    double D, q, bsq, bsq_rpsq, rsq, rbsq, v0sq, gam, rho_floor, e_floor, gamma_max, e_max;
    bool used_density_floor = false, used_energy_floor = false, used_energy_max = false, used_gamma_max = false;
    double x_mu(double mu) const { return 1.0 / (1.0 + mu * bsq); }
    double rbarsq_mu(double mu, double x) const { return x * (x * rsq + mu * (1.0 + x) * rbsq); }
    double qbar_mu(double mu, double x) const
    {
        const double mux = mu * x;
        return q - 0.5 * (bsq + mux * mux * bsq_rpsq);
    }
    double vhatsq_mu(double mu, double rbarsq)
    {
        const double vsq_trial = mu * mu * rbarsq;
        if (vsq_trial > v0sq) { used_gamma_max = true; return v0sq; }
        used_gamma_max = false;
        return vsq_trial;
    }
    double iWhat_mu(double vhatsq) const { return std::sqrt(1.0 - vhatsq); }
    double rhohat_mu(double iWhat)
    {
        const double rho_trial = D * iWhat;
        if (rho_trial <= rho_floor) { used_density_floor = true; return rho_floor; }
        used_density_floor = false;
        return rho_trial;
    }
    double ehat_mu(double mu, double qbar, double rbarsq, double vhatsq, double What)
    {
        const double ehat_trial = What * (qbar - mu * rbarsq) + vhatsq * What * What / (1.0 + What);
        used_energy_floor = false;
        used_energy_max = false;
        if (ehat_trial <= e_floor) { used_energy_floor = true; return e_floor; }
        else if (ehat_trial > e_max) { used_energy_max = true; return e_max; }
        return ehat_trial;
    }
    double operator()(double mu)    // eq. 44
    {
        const double x = x_mu(mu);
        const double rbarsq = rbarsq_mu(mu, x);
        const double qbar = qbar_mu(mu, x);
        const double vhatsq = vhatsq_mu(mu, rbarsq);
        const double iWhat = iWhat_mu(vhatsq);
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
    double aux_func(double mu) const    // eq. 49
    {
        const double x = 1.0 / (1.0 + mu * bsq);
        const double rbarsq = x * (rsq * x + mu * (1.0 + x) * rbsq);
        return mu * std::sqrt(1.0 + rbarsq) - 1.0;
    }
};

// Illinois false position on [zm, zp] (kastaun.hpp:305-331 and 343-368); returns the last iterate
// and the iteration count at exit (max_iterations when it did not converge)
template <typename F>
static double illinois(F&& f, double zm, double zp, int max_iterations, double tol, int& iter)
{
    double fm = f(zm), fp = f(zp);
    int iterations = max_iterations;
    if ((std::fabs(zm - zp) < tol) || ((std::fabs(fm) + std::fabs(fp)) < 2.0 * tol)) iterations = -1;
    double z = 0.5 * (zm + zp);
    for (iter = 0; iter < iterations; ++iter) {
        z = (zm * fp - zp * fm) / (fp - fm);
        const double fz = f(z);
        if ((std::fabs(zm - zp) < tol) || (std::fabs(fz) < tol)) break;
        if (fz * fp < 0.0) { zm = zp; fm = fp; zp = z; fp = fz; }
        else { fm = 0.5 * fm; zp = z; fp = fz; }
    }
    return z;
}

static int u_to_p_kastaun(const Block& B, const double* U, double* P, int j, int i, int loc, int max_iterations,
                          double tol)
{
    const Prescription& fl = myfloors(B, j, i);
    const double gam = B.c.gam;
    const double alpha = 1. / std::sqrt(-B.Gcon(loc, j, i, 0, 0));
    const double a_over_g = alpha / B.Gdet(loc, j, i);
    const double D = U[0] * a_over_g;
    const double D_fl = kmax(D, fl.rho_min_const);
    const double Qcov[4] = {(U[1] - U[0]) * a_over_g, U[2] * a_over_g, U[3] * a_over_g, U[4] * a_over_g};
    const double ncov[4] = {-alpha, 0., 0., 0.};
    double ncon[4];
    B.raise(ncov, ncon, j, i, loc);
    const double q = (-dot4(Qcov, ncon) - D) / D;
    const double rcov[3] = {U[2] / U[0], U[3] / U[0], U[4] / U[0]};
    double g[4][4];
    for (int mu = 0; mu < 4; ++mu) for (int nu = 0; nu < 4; ++nu) g[mu][nu] = B.Gcon(loc, j, i, mu, nu);
    double rcon[3];
    for (int a = 0; a < 3; ++a)        // gamma^ij = g^ij - g^0i g^0j / g^00 (kastaun.hpp:250-262)
        rcon[a] = ((g[a+1][1] - g[0][a+1]*g[0][1]/g[0][0])*rcov[0] +
                   (g[a+1][2] - g[0][a+1]*g[0][2]/g[0][0])*rcov[1] +
                   (g[a+1][3] - g[0][a+1]*g[0][3]/g[0][0])*rcov[2]);
    double rsq = 0.0;
    for (int a = 0; a < 3; ++a) rsq += rcon[a] * rcov[a];
    double bsq = 0.0, bsq_rpsq = 0.0, rbsq = 0.0, bdotr = 0.0, bu[3] = {0.0, 0.0, 0.0};
    if (B.nv > 5) {
        const double sD = 1.0 / std::sqrt(D_fl);
        for (int a = 0; a < 3; ++a) {
            bu[a] = (U[5 + a] * a_over_g) * sD;
            bdotr += bu[a] * rcov[a];
        }
        for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) bsq += B.Gcov(loc, j, i, a + 1, b + 1) * bu[a] * bu[b];
        bsq = kmax(0.0, bsq);
        rbsq = bdotr * bdotr;
        bsq_rpsq = bsq * rsq - rbsq;
    }
    const double zsq = rsq;
    const double v0sq = kmin(zsq / (1.0 + zsq), 1.0 - 1.0 / (fl.gamma_max * fl.gamma_max));
    KastaunResidual res{D, q, bsq, bsq_rpsq, rsq, rbsq, v0sq, gam, fl.rho_min_const, fl.u_min_const / D_fl,
                        fl.gamma_max, fl.u_over_rho_max};
    int iter = 0;
    const double zb = illinois([&](double z) { return res.aux_func(z); }, 0., 1., max_iterations, tol, iter);
    const double mu = illinois([&](double z) { return res(z); }, 0., zb, max_iterations, tol, iter);
    if (iter == max_iterations) return max_iter;
    const double x = res.x_mu(mu);
    const double rbarsq = res.rbarsq_mu(mu, x);
    const double vsq = res.vhatsq_mu(mu, rbarsq);
    const double iW = res.iWhat_mu(vsq);
    const double W = 1. / iW;
    P[0] = res.rhohat_mu(iW);
    const double qbar = res.qbar_mu(mu, x);
    P[1] = res.ehat_mu(mu, qbar, rbarsq, vsq, W) * P[0];
    for (int a = 0; a < 3; ++a) P[2 + a] = W * mu * x * (rcon[a] + mu * bdotr * bu[a]);
    int fflag = 0;
    if (res.used_density_floor) fflag |= FF_INVERTER_RHO;
    if (res.used_energy_floor) fflag |= FF_INVERTER_U;
    if (res.used_gamma_max) fflag |= FF_INVERTER_GAMMA;
    if (res.used_energy_max) fflag |= FF_INVERTER_U_MAX;
    return fflag;
}

// Inverter::u_to_p dispatch on inverter/type (inverter.cpp:54-64)
static int u_to_p(const Block& B, const double* U, double* P, int j, int i, int loc, int max_iterations, double tol)
{
    if (B.c.inverter == 1) return u_to_p_kastaun(B, U, P, j, i, loc, max_iterations, tol);
    return u_to_p_onedw(B, U, P, j, i, loc, max_iterations, tol);
}

// ---------------------------------------------------------------- state helpers
struct Fields {
    std::vector<double> F[3], cmax[3], cmin[3];
    void alloc(const Block& B)
    {
        for (int d = 0; d < 3; ++d) {
            F[d].assign((size_t)B.nv*B.N, 0.);
            cmax[d].assign(B.N, 0.);
            cmin[d].assign(B.N, 0.);
        }
    }
};

static inline void load_cell(const Block& B, const double* A, size_t c, double* out)
{
    for (int p = 0; p < B.nv; ++p) out[p] = A[(size_t)p*B.N + c];
}
static inline void store_cell(const Block& B, double* A, size_t c, const double* in, int nvars)
{
    for (int p = 0; p < nvars; ++p) A[(size_t)p*B.N + c] = in[p];
}

// Inverter::BlockUtoP + B_FluxCT::BlockUtoP over a range (inverter.cpp:131-182, b_flux_ct.cpp:196-217)
static void block_utop(const Block& B, const double* U, double* P, double* pflag, double* fflag,
                       int ks, int ke, int js, int je, int is, int ie)
{
#pragma omp parallel for collapse(2) schedule(dynamic, 4)
    for (int k = ks; k <= ke; ++k) for (int j = js; j <= je; ++j) for (int i = is; i <= ie; ++i) {
        const size_t c = B.id(k, j, i);
        double Uc[8], Pc[8];
        load_cell(B, U, c, Uc);
        load_cell(B, P, c, Pc);
        const int pf = u_to_p(B, Uc, Pc, j, i, center, B.c.iter_max, B.c.err_tol);
        store_cell(B, P, c, Pc, 5);
        pflag[c] = pf % 32;
        fflag[c] = (pf / 32) * 32;
    }
    if (B.nv > 5) {
        for (int v = 0; v < 3; ++v)
        for (int k = ks; k <= ke; ++k) for (int j = js; j <= je; ++j) for (int i = is; i <= ie; ++i) {
            const size_t c = B.id(k, j, i);
            P[(size_t)(5 + v)*B.N + c] = U[(size_t)(5 + v)*B.N + c] / B.Gdet(center, j, i);
        }
    }
}

// floors.cpp:215-229 and floors_impl.hpp:45-128
static void apply_grmhd_floors(const Block& B, double* P, double* U, double* pflag, double* fflag,
                               int ks, int ke, int js, int je, int is, int ie)
{
    const size_t N = B.N;
    std::vector<double> rhofl(N, 0.), ufl(N, 0.);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = ks; k <= ke; ++k) for (int j = js; j <= je; ++j) for (int i = is; i <= ie; ++i) {
        const size_t c = B.id(k, j, i);
        double Pc[8];
        load_cell(B, P, c, Pc);
        double rf, uf;
        const int ff = determine_floors(B, Pc, j, i, rf, uf);
        fflag[c] = (int)fflag[c] | ff;
        rhofl[c] = rf; ufl[c] = uf;
    }
#pragma omp parallel for collapse(2) schedule(dynamic, 4)
    for (int k = ks; k <= ke; ++k) for (int j = js; j <= je; ++j) for (int i = is; i <= ie; ++i) {
        const size_t c = B.id(k, j, i);
        if ((int)fflag[c]) {
            double Pc[8], Uc[8];
            load_cell(B, P, c, Pc);
            load_cell(B, U, c, Uc);
            const int pf = apply_floors_frame(B, Pc, Uc, j, i, rhofl[c], ufl[c]);
            if (pf) pflag[c] = pf;
            apply_ceilings(B, Pc, j, i);
            store_cell(B, P, c, Pc, 5);
            store_cell(B, U, c, Uc, 5);
            p_to_u_mhd_cell(B, P, U, c, j, i);
        }
    }
}

// fixup.cpp:47-156.  Neighbours are read inside [ks..ke] x [js..je] x [is..ie] (the physical range).
static void fix_utop(const Block& B, double* P, double* U, const double* pflag,
                     int ks, int ke, int js, int je, int is, int ie)
{
    if (!B.c.fix_average_neighbors && !B.c.fix_atmosphere) return;
    const size_t N = B.N;
    for (int k = ks; k <= ke; ++k) for (int j = js; j <= je; ++j) for (int i = is; i <= ie; ++i) {
        const size_t c = B.id(k, j, i);
        if ((int)pflag[c] > 0) {
            double wsum = 0., sum[5] = {0.};
            if (B.c.fix_average_neighbors) {
                for (int n = -1; n <= 1; n++) for (int m = -1; m <= 1; m++) for (int l = -1; l <= 1; l++) {
                    const int ii = i + l, jj = j + m, kk = k + n;
                    if (ii < is || ii > ie || jj < js || jj > je || kk < ks || kk > ke) continue;
                    const size_t cn = B.id(kk, jj, ii);
                    if (!((int)pflag[cn] > 0)) {
                        const double w = 1./(std::abs(l) + std::abs(m) + std::abs(n) + 1);
                        wsum += w;
                        for (int p = 0; p < 5; ++p) sum[p] += w * P[(size_t)p*N + cn];
                    }
                }
            }
            for (int p = 0; p < 5; ++p) P[(size_t)p*N + c] = (wsum < 1.e-10) ? 0. : sum[p]/wsum;
        }
    }
    for (int k = ks; k <= ke; ++k) for (int j = js; j <= je; ++j) for (int i = is; i <= ie; ++i) {
        const size_t c = B.id(k, j, i);
        if ((int)pflag[c] > 0) {
            double Pc[8];
            load_cell(B, P, c, Pc);
            // floors_functions.hpp:356-367 (global form) -- identical arithmetic to the local form
            apply_geo_floors_local(B, Pc, j, i);
            store_cell(B, P, c, Pc, 5);
            // grmhd_functions.hpp:325-353 (GRMHD::p_to_u): rho, u, uvec only
            p_to_u_mhd_cell(B, P, U, c, j, i);
        }
    }
}

// ---------------------------------------------------------------- boundaries
// Periodic: Parthenon internal sync.  Outflow/reflecting: Parthenon BoundaryFunction (unvendored):
// outflow copies the last interior zone; reflecting mirrors about the face and flips the sign of
// the vector component normal to it.  KHARMA applies these to the fluid primitives (rho, u, uvec)
// and the conserved field B_U, then sets B_P = B_U/gdet (boundaries.cpp:369-589).
static void periodic_fill(const Block& B, double* A, int nvars, int dir)
{
    for (int p = 0; p < nvars; ++p) {
        double* q = A + (size_t)p*B.N;
        for (int k = 0; k < B.n3; ++k) for (int j = 0; j < B.n2; ++j) for (int i = 0; i < B.n1; ++i) {
            int ii = i, jj = j, kk = k;
            if (dir == 1) { if (i >= B.is && i <= B.ie) continue; ii = (i < B.is) ? i + B.c.nx1 : i - B.c.nx1; }
            if (dir == 2) { if (j >= B.js && j <= B.je) continue; jj = (j < B.js) ? j + B.c.nx2 : j - B.c.nx2; }
            if (dir == 3) { if (k >= B.ks && k <= B.ke) continue; kk = (k < B.ks) ? k + B.c.nx3 : k - B.c.nx3; }
            q[B.id(k, j, i)] = q[B.id(kk, jj, ii)];
        }
    }
}
// boundaries.hpp:101-136
static void check_inflow(const Block& B, double* P, size_t c, int j, int i, bool inner)
{
    double uvec[3], ucon[4];
    for (int v = 0; v < 3; ++v) uvec[v] = P[(size_t)(2 + v)*B.N + c];
    {
        double Ptmp[8] = {0, 0, uvec[0], uvec[1], uvec[2], 0, 0, 0};
        const double gamma = lorentz_calc(B, Ptmp, j, i, center);
        const double alpha = 1. / std::sqrt(-B.Gcon(center, j, i, 0, 0));
        ucon[0] = gamma / alpha;
        for (int v = 0; v < 3; ++v) ucon[v+1] = uvec[v] - gamma * alpha * B.Gcon(center, j, i, 0, v+1);
    }
    if (((ucon[1] > 0.) && inner) || ((ucon[1] < 0.) && !inner)) {
        double Ptmp[8] = {0, 0, uvec[0], uvec[1], uvec[2], 0, 0, 0};
        double gamma = lorentz_calc(B, Ptmp, j, i, center);
        for (int v = 0; v < 3; ++v) uvec[v] /= gamma;
        const double alpha = 1. / std::sqrt(-B.Gcon(center, j, i, 0, 0));
        const double beta1 = B.Gcon(center, j, i, 0, 1) * alpha * alpha;
        uvec[0] = beta1 / alpha;
        const double vsq = B.Gcov(center, j, i, 1, 1) * uvec[0] * uvec[0] +
                           B.Gcov(center, j, i, 2, 2) * uvec[1] * uvec[1] +
                           B.Gcov(center, j, i, 3, 3) * uvec[2] * uvec[2] +
                           2. * (B.Gcov(center, j, i, 1, 2) * uvec[0] * uvec[1] +
                                 B.Gcov(center, j, i, 1, 3) * uvec[0] * uvec[2] +
                                 B.Gcov(center, j, i, 2, 3) * uvec[1] * uvec[2]);
        // clip() result discarded in the reference (boundaries.hpp:129)
        gamma = 1./std::sqrt(1. - vsq);
        for (int v = 0; v < 3; ++v) uvec[v] *= gamma;
        for (int v = 0; v < 3; ++v) P[(size_t)(2 + v)*B.N + c] = uvec[v];
    }
}
// One physical face: P (fluid primitives, vars 0-4) and U_B (vars 5-7 of U); emhd: also the scalar
// primitives q~, dP~ (slots 8, 9), copied as the density is (no sign change)
static void physical_face(const Block& B, double* P, double* U, int face, bool emhd = false)
{
    const int bdir = face / 2 + 1;
    const bool binner = (face % 2) == 0;
    const int type = B.c.bc[face];
    const size_t N = B.N;
    // boundary domain: ghost zones in bdir, all zones in the other directions
    int i0 = 0, i1 = B.n1 - 1, j0 = 0, j1 = B.n2 - 1, k0 = 0, k1 = B.n3 - 1;
    int ref, offset;
    if (bdir == 1) { if (binner) { i0 = 0; i1 = B.is - 1; ref = B.is; } else { i0 = B.ie + 1; i1 = B.n1 - 1; ref = B.ie; } }
    else if (bdir == 2) { if (binner) { j0 = 0; j1 = B.js - 1; ref = B.js; } else { j0 = B.je + 1; j1 = B.n2 - 1; ref = B.je; } }
    else { if (binner) { k0 = 0; k1 = B.ks - 1; ref = B.ks; } else { k0 = B.ke + 1; k1 = B.n3 - 1; ref = B.ke; } }
    offset = 2 * ref + (binner ? -1 : 1);
    for (int k = k0; k <= k1; ++k) for (int j = j0; j <= j1; ++j) for (int i = i0; i <= i1; ++i) {
        const size_t c = B.id(k, j, i);
        int kk = k, jj = j, ii = i;
        if (type == BC_OUTFLOW) {
            if (bdir == 1) ii = ref; else if (bdir == 2) jj = ref; else kk = ref;
        } else {
            if (bdir == 1) ii = offset - i; else if (bdir == 2) jj = offset - j; else kk = offset - k;
        }
        // transmitting polar faces (one_block_transmit.cpp:116-134): half-way round in x3, u^2, u^3,
        // B^2, B^3 inverted
        const bool transmit = type == BC_TRANSMIT;
        if (transmit) kk = ((k - B.ks + B.c.nx3 / 2) % B.c.nx3) + B.ks;
        const size_t s = B.id(kk, jj, ii);
        for (int p = 0; p < 5; ++p) {
            const bool flip = ((type == BC_REFLECT) && (p == 1 + bdir)) || (transmit && (p == 3 || p == 4));
            P[(size_t)p*N + c] = (flip ? -1.0 : 1.0) * P[(size_t)p*N + s];
        }
        if (emhd)
            for (int p = 8; p < 10; ++p) P[(size_t)p*N + c] = P[(size_t)p*N + s];
        if (B.nv > 5)
            for (int v = 0; v < 3; ++v) {
                const bool flip = ((type == BC_REFLECT) && (v == bdir - 1)) || (transmit && v >= 1);
                U[(size_t)(5 + v)*N + c] = (flip ? -1.0 : 1.0) * U[(size_t)(5 + v)*N + s];
            }
    }
    const bool inflow = (face == 0 && B.c.check_inflow_inner_x1) || (face == 1 && B.c.check_inflow_outer_x1);
    if (inflow)
        for (int k = k0; k <= k1; ++k) for (int j = j0; j <= j1; ++j) for (int i = i0; i <= i1; ++i)
            check_inflow(B, P, B.id(k, j, i), j, i, binner);
}
// Fill all ghost zones: physical faces in the order Parthenon applies them (x1, x2, then the
// fix_corner re-application of inner x1: boundaries.cpp:538-559), then periodic directions.
// emhd: P and U hold the 10 slots of the EMHD state (the scalar slots q~, dP~ filled as well)
static void apply_boundaries(const Block& B, double* P, double* U, bool emhd = false)
{
    const int nvars = emhd ? 10 : B.nv;
    // periodic directions first, so physical faces see filled corners exactly as after a sync
    for (int d = 1; d <= B.ndim; ++d)
        if (B.c.bc[2*(d-1)] == BC_PERIODIC) { periodic_fill(B, P, nvars, d); periodic_fill(B, U, nvars, d); }
    for (int face = 0; face < 2*B.ndim; ++face) {
        if (!phys_face(B.c.bc[face])) continue;
        physical_face(B, P, U, face, emhd);
        if (face == 3 && B.c.fix_corner_inner && phys_face(B.c.bc[0])) physical_face(B, P, U, 0, emhd);
    }
    for (int d = 1; d <= B.ndim; ++d)
        if (B.c.bc[2*(d-1)] == BC_PERIODIC) { periodic_fill(B, P, nvars, d); periodic_fill(B, U, nvars, d); }
    // B_P = B_U/gdet in the ghost zones (BoundaryUtoP of B_FluxCT)
    if (B.nv > 5)
        for (int k = 0; k < B.n3; ++k) for (int j = 0; j < B.n2; ++j) for (int i = 0; i < B.n1; ++i) {
            if (i >= B.is && i <= B.ie && j >= B.js && j <= B.je && k >= B.ks && k <= B.ke) continue;
            const size_t c = B.id(k, j, i);
            for (int v = 0; v < 3; ++v) P[(size_t)(5 + v)*B.N + c] = U[(size_t)(5 + v)*B.N + c] / B.Gdet(center, j, i);
        }
}

// ---------------------------------------------------------------- timestep and diagnostics
// grmhd.cpp:294-339 (minimum of the zone timestep over the interior, before cfl and clipping)
static double min_ndt(const Block& B, const Fields& f)
{
    double m = std::numeric_limits<double>::max();
#pragma omp parallel for collapse(2) reduction(min:m)
    for (int k = B.ks; k <= B.ke; ++k) for (int j = B.js; j <= B.je; ++j) for (int i = B.is; i <= B.ie; ++i) {
        const size_t c = B.id(k, j, i);
        const double ndt_zone = 1.0 / (1 / (B.c.dx1 / kmax(f.cmax[0][c], f.cmin[0][c])) +
                                       1 / (B.c.dx2 / kmax(f.cmax[1][c], f.cmin[1][c])) +
                                       1 / (B.c.dx3 * 1 / kmax(f.cmax[2][c], f.cmin[2][c])));
        if (!std::isnan(ndt_zone) && (ndt_zone < m)) m = ndt_zone;
    }
    return m;
}
// b_flux_ct.cpp:566-607 and b_flux_ct_functions.hpp:52-75
static double max_divb(const Block& B, const double* U, int avoid_inner, int avoid_outer)
{
    if (B.ndim < 2) return 0.;
    const size_t N = B.N;
    const double* B1 = U + 5*N; const double* B2 = U + 6*N; const double* B3 = U + 7*N;
    const size_t sj = B.n1, sk = (size_t)B.n1*B.n2;
    const bool do3 = B.ndim > 2;
    double mx = 0.;
    for (int k = B.ks; k <= B.ke + (B.ndim > 2); ++k)
    for (int j = B.js; j <= B.je + 1; ++j)
    for (int i = B.is + avoid_inner; i <= B.ie + !avoid_outer; ++i) {
        const size_t c = B.id(k, j, i);
        const double norm = do3 ? 0.25 : 0.5;
        double term1 = B1[c] - B1[c-1] + B1[c-sj] - B1[c-sj-1];
        double term2 = B2[c] - B2[c-sj] + B2[c-1] - B2[c-sj-1];
        double term3 = 0.;
        if (do3) {
            term1 += B1[c-sk] + B1[c-sk-sj] - B1[c-sk-1] - B1[c-sk-sj-1];
            term2 += B2[c-sk] + B2[c-sk-1] - B2[c-sk-sj] - B2[c-sk-sj-1];
            term3 = B3[c] + B3[c-sj] + B3[c-1] + B3[c-sj-1] - B3[c-sk] - B3[c-sk-sj] - B3[c-sk-1] - B3[c-sk-sj-1];
        }
        const double d = std::fabs(norm*term1/B.c.dx1 + norm*term2/B.c.dx2 + norm*term3/B.c.dx3);
        if (d > mx) mx = d;
    }
    return mx;
}

// ---------------------------------------------------------------- one RK2 stage
// Parthenon "rk2" low-storage integrator (unvendored): gam0 = {0, 1/2}, gam1 = {1, 1/2}, beta = {1, 1/2}.
static const double RK_GAM0[2] = {0.0, 0.5}, RK_GAM1[2] = {1.0, 0.5}, RK_BETA[2] = {1.0, 0.5};

// Full-domain ghost refresh + lock-step P->U, shared by both drivers after the UtoP/floors/fixup region
static void finish_stage(const Block& B, double* P, double* U)
{
    apply_boundaries(B, P, U);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < B.n3; ++k) for (int j = 0; j < B.n2; ++j) for (int i = 0; i < B.n1; ++i)
        p_to_u_cell(B, P, U, B.id(k, j, i), j, i);      // Flux::MeshPtoU(entire), flux.cpp:317-322
}

// ---------------------------------------------------------------- first-order flux correction
// KHARMADriver::AddFOFC (kharma_driver.cpp:292-337), Flux::MarkFOFC and Flux::FOFC (fofc.cpp:45-226),
// run between the flux calculation and FixFlux.  A guess of the stage result from the high-order
// fluxes marks the zones where it would hit floors (or lie within eh_buffer of the horizon, or in
// the polar rows); every face bordering a marked zone then gets the donor-cell LLF flux.
//  * the guess divergence covers the interior plus 3 zones (kharma_driver.cpp:306-307) and uses the
//    flux arrays as they stand: faces the flux calculation does not cover hold zeros or the values a
//    previous correction left there, as in the reference;
//  * the guess inversion starts from the stage's primitives (the reference's guess container holds
//    whatever its previous inversion left, a history this restatement does not keep);
//  * periodic directions take the flags of their images (the flag's boundary sync).
static void fofc_correct(const Block& B, Fields& f, int s, double dt, const double* P_s, const double* U_s,
                         const double* U_0)
{
    const size_t N = B.N, nv = B.nv;
    const double g0 = RK_GAM0[s], g1 = RK_GAM1[s], bdt = RK_BETA[s] * dt;
    const double a1 = B.c.dx2*B.c.dx3, a2 = B.c.dx1*B.c.dx3, a3 = B.c.dx1*B.c.dx2;
    const double vol = B.c.dx1*B.c.dx2*B.c.dx3;
    const size_t sj = B.n1, sk = (size_t)B.n1*B.n2;
    const int h2 = B.ndim > 1, h3 = B.ndim > 2;
    // zones whose flags a corrected face reads: interior +-2 (+-0 along periodic directions, whose
    // ghost flags come from their images)
    const int per1 = B.c.bc[0] == BC_PERIODIC, per2 = B.c.bc[2] == BC_PERIODIC, per3 = B.c.bc[4] == BC_PERIODIC;
    const int i0 = B.is - (per1 ? 0 : 2), i1 = B.ie + (per1 ? 0 : 2);
    const int j0 = B.js - (per2 ? 0 : 2*h2), j1 = B.je + (per2 ? 0 : 2*h2);
    const int k0 = B.ks - (per3 ? 0 : 2*h3), k1 = B.ke + (per3 ? 0 : 2*h3);
    std::vector<int> flag(N, 0);
    const double r_mark = B.c.r_horizon + B.c.fofc_eh_buffer;
#pragma omp parallel for collapse(2) schedule(dynamic, 4)
    for (int k = k0; k <= k1; ++k) for (int j = j0; j <= j1; ++j) for (int i = i0; i <= i1; ++i) {
        const size_t c = B.id(k, j, i);
        double Ug[8], Pg[8], dudt[8];
        for (size_t p = 0; p < nv; ++p) {
            const size_t pc = p*N + c;
            double du = (a1 * f.F[0][pc + 1] - a1 * f.F[0][pc]);
            if (B.ndim >= 2) du += a2 * f.F[1][pc + sj] - a2 * f.F[1][pc];
            if (B.ndim == 3) du += a3 * f.F[2][pc + sk] - a3 * f.F[2][pc];
            dudt[p] = -du / vol;
            Pg[p] = P_s[pc];
        }
        // fofc/use_source_term: the guess also takes the geometric source of P_s
        // (kharma_driver.cpp:308-312, over the entire block)
        if (B.c.fofc_use_source_term && !B.C.cart_minkowski()) {
            double new_du[4];
            geo_source_cell(B, Pg, j, i, new_du);
            for (int v = 0; v < 4; ++v) dudt[1 + v] += new_du[v];
        }
        for (size_t p = 0; p < nv; ++p) {
            const size_t pc = p*N + c;
            double x = g0 * U_s[pc] + g1 * U_0[pc];
            Ug[p] = 1.0 * x + bdt * dudt[p];
        }
        if (nv > 5) for (int v = 0; v < 3; ++v) Pg[5 + v] = Ug[5 + v] / B.Gdet(center, j, i);
        const int pf = u_to_p(B, Ug, Pg, j, i, center, B.c.iter_max, B.c.err_tol);
        int ff = (pf / 32) * 32;
        if (B.c.floors_on) {
            double rf, uf;
            ff |= determine_floors(B, Pg, j, i, rf, uf);
        }
        const bool eh = B.C.spherical() && B.rcen[(size_t)j*B.n1 + i] < r_mark;
        flag[c] = (ff != 0 || eh) ? 1 : 0;
    }
    if (B.C.spherical() && B.c.fofc_polar_cells > 0 && B.ndim > 1) {
        for (int face = 2; face <= 3; ++face) {
            if (!phys_face(B.c.bc[face])) continue;
            const int js_ = (face == 2) ? B.js : B.je - B.c.fofc_polar_cells + 1;
            const int je_ = (face == 2) ? B.js + B.c.fofc_polar_cells - 1 : B.je;
            for (int k = 0; k < B.n3; ++k) for (int j = js_; j <= je_; ++j) for (int i = 0; i < B.n1; ++i)
                flag[B.id(k, j, i)] = 1;
        }
    }
    for (int d = 1; d <= B.ndim; ++d) {
        if (B.c.bc[2*(d-1)] != BC_PERIODIC) continue;
        std::vector<double> tmp(flag.begin(), flag.end());
        periodic_fill(B, tmp.data(), 1, d);
        for (size_t x = 0; x < N; ++x) flag[x] = (int)tmp[x];
    }
    // donor-cell LLF fluxes on faces bordering a marked zone, faces over the interior +-1 (fofc.cpp:144-221)
    for (int dir = 1; dir <= B.ndim; ++dir) {
        const int loc = dir - 1;
        const ptrdiff_t st = (dir == 1) ? 1 : ((dir == 2) ? (ptrdiff_t)sj : (ptrdiff_t)sk);
        const int fi1 = kmin(B.ie + 1 + (dir == 1), B.n1 - 1), fi0 = kmax(B.is - 1, dir == 1 ? 1 : 0);
        const int fj0 = h2 ? kmax(B.js - 1, dir == 2 ? 1 : 0) : B.js, fj1 = h2 ? kmin(B.je + 1 + (dir == 2), B.n2 - 1) : B.je;
        const int fk0 = h3 ? kmax(B.ks - 1, dir == 3 ? 1 : 0) : B.ks, fk1 = h3 ? kmin(B.ke + 1 + (dir == 3), B.n3 - 1) : B.ke;
#pragma omp parallel for collapse(2) schedule(static)
        for (int k = fk0; k <= fk1; ++k) for (int j = fj0; j <= fj1; ++j) for (int i = fi0; i <= fi1; ++i) {
            const size_t c = B.id(k, j, i);
            if (!(flag[c] || flag[c - st])) continue;
            double Pl[8], Pr[8];
            for (size_t p = 0; p < nv; ++p) { Pl[p] = P_s[p*N + c - st]; Pr[p] = P_s[p*N + c]; }
            FourVectors Dl, Dr;
            double Ul[8], Fl[8], Ur[8], Fr[8], cmaxL, cminL, cmaxR, cminR;
            calc_4vecs(B, Pl, nv > 5, j, i, loc, Dl);
            prim_to_flux(B, Pl, Dl, j, i, 0, Ul, loc);
            prim_to_flux(B, Pl, Dl, j, i, dir, Fl, loc);
            vchar(B, Pl, Dl, j, i, loc, dir, cmaxL, cminL);
            calc_4vecs(B, Pr, nv > 5, j, i, loc, Dr);
            prim_to_flux(B, Pr, Dr, j, i, 0, Ur, loc);
            prim_to_flux(B, Pr, Dr, j, i, dir, Fr, loc);
            vchar(B, Pr, Dr, j, i, loc, dir, cmaxR, cminR);
            // fofc/use_glf: the global (speed of light) Lax-Friedrichs speeds on replaced faces (fofc.cpp:200-205)
            const double cmax = B.c.fofc_use_glf ? 1. : kmax(kmax(0., cmaxL), cmaxR);
            const double cmin = B.c.fofc_use_glf ? 1. : -kmin(kmin(0., cminL), cminR);
            f.cmax[dir-1][c] = cmax;
            f.cmin[dir-1][c] = cmin;
            for (size_t p = 0; p < nv; ++p) f.F[dir-1][p*N + c] = llf(Fl[p], Fr[p], cmax, cmin, Ul[p], Ur[p]);
        }
    }
}

// FixUtoP as a stage runs it (inverter.hpp:83-89, fixup.cpp:47-156) over the physical range: periodic
// ghosts of P and pflag are filled first so that they serve as neighbours, and across exchange faces
// the neighbour's values in the ghost zones are valid neighbours (their flags are the caller's; zero
// unless it exchanges them)
static void stage_fix_utop(const Block& B, double* P_n, double* U_n, double* pflag)
{
    int ks = B.ks, ke = B.ke, js = B.js, je = B.je, is = B.is, ie = B.ie;
    for (int d = 1; d <= B.ndim; ++d)
        if (B.c.bc[2*(d-1)] == BC_PERIODIC) {
            periodic_fill(B, P_n, 5, d);
            periodic_fill(B, pflag, 1, d);
            if (d == 1) { is = 0; ie = B.n1 - 1; }
            if (d == 2) { js = 0; je = B.n2 - 1; }
            if (d == 3) { ks = 0; ke = B.n3 - 1; }
        }
    if (B.c.bc[0] == BC_EXCHANGE) is = 0;
    if (B.c.bc[1] == BC_EXCHANGE) ie = B.n1 - 1;
    if (B.ndim > 1 && B.c.bc[2] == BC_EXCHANGE) js = 0;
    if (B.ndim > 1 && B.c.bc[3] == BC_EXCHANGE) je = B.n2 - 1;
    if (B.ndim > 2 && B.c.bc[4] == BC_EXCHANGE) ks = 0;
    if (B.ndim > 2 && B.c.bc[5] == BC_EXCHANGE) ke = B.n3 - 1;
    fix_utop(B, P_n, U_n, pflag, ks, ke, js, je, is, ie);
}

// One stage.  P_s/U_s: stage-start state; U_0: step-start conserved state; outputs P_n/U_n.
static void stage(const Block& B, Fields& f, int s, double dt,
                  const double* P_s, const double* U_s, const double* U_0,
                  double* P_n, double* U_n, double* pflag, double* fflag)
{
    const size_t N = B.N, NV = (size_t)B.nv*N;
    // 1. fluxes (kharma_driver.cpp:203-290)
    for (int d = 1; d <= B.ndim; ++d)
        get_flux(B, d, P_s, f.F[d-1].data(), f.cmax[d-1].data(), f.cmin[d-1].data());
    // 1b. first-order flux correction (kharma_step.cpp:168-173), before FixFlux
    if (B.c.fofc) fofc_correct(B, f, s, dt, P_s, U_s, U_0);
    // 2. FixFlux: B_FluxCT then Boundaries (kharma_package.cpp:43-56; the order does not change results)
    double* F[3] = {f.F[0].data(), f.F[1].data(), f.F[2].data()};
    if (B.nv > 5) {
        if (B.c.fix_polar_flux && B.C.spherical()) {
            if (phys_face(B.c.bc[2])) zero_boundary_flux_x2(B, F[0], F[1], F[2], true);
            if (phys_face(B.c.bc[3])) zero_boundary_flux_x2(B, F[0], F[1], F[2], false);
        }
        flux_ct(B, F[0], F[1], F[2]);
    }
    boundaries_fix_flux(B, F);
    // 3-4. dU/dt = -div F + geometric source (kharma_driver.hpp:208-231, flux.cpp:395-444)
    std::vector<double> dudt(NV, 0.);
    flux_divergence(B, F, dudt.data());
    add_geo_source(B, P_s, dudt.data());
    // 5. U_n = gam0 U_s + gam1 U_0 ; U_n = 1.0 U_n + (beta dt) dU/dt (Parthenon WeightedSumData, all zones)
    const double g0 = RK_GAM0[s], g1 = RK_GAM1[s], bdt = RK_BETA[s] * dt;
#pragma omp parallel for schedule(static)
    for (size_t x = 0; x < NV; ++x) U_n[x] = g0 * U_s[x] + g1 * U_0[x];
#pragma omp parallel for schedule(static)
    for (size_t x = 0; x < NV; ++x) U_n[x] = 1.0 * U_n[x] + bdt * dudt[x];
    // copy P_s -> P_n as the inversion guess (kharma_driver.cpp:380-384; fluid prims only)
    std::memcpy(P_n, P_s, 5*N*sizeof(double));
    // 7-8. UtoP and floors on the interior (periodic ghosts are exact images and are refreshed below)
    for (size_t x = 0; x < N; ++x) { pflag[x] = 0; fflag[x] = 0; }
    block_utop(B, U_n, P_n, pflag, fflag, B.ks, B.ke, B.js, B.je, B.is, B.ie);
    if (B.c.floors_on) apply_grmhd_floors(B, P_n, U_n, pflag, fflag, B.ks, B.ke, B.js, B.je, B.is, B.ie);
    // 9. FixUtoP over the physical range
    stage_fix_utop(B, P_n, U_n, pflag);
    // 10-11. boundaries, then U = U(P) over the entire block
    finish_stage(B, P_n, U_n);
}

// ---------------------------------------------------------------- B_CT (b_ct/b_ct.cpp)
// Face field arrays Bf[3][N]: sqrt(-g) B^d on the x_d faces, face i = left face of zone i.  2D and 3D
// blocks with periodic or exchange faces; only the interior faces [is, ie+1] (along their own
// direction) are state.
static const int CT_BS99 = 1, CT_GS05_0 = 2, CT_GS05_C = 3;

// B_CT::BlockUtoP for one zone (b_ct.cpp:172-181)
static void ct_zone_b(const Block& B, const double* Bf, int k, int j, int i, double Bp[3])
{
    const size_t N = B.N, c = B.id(k, j, i);
    const double* F1 = Bf; const double* F2 = Bf + N; const double* F3 = Bf + 2*N;
    Bp[0] = (F1[c] / B.Gdet(face1, j, i) + F1[c + 1] / B.Gdet(face1, j, i + 1)) / 2;
    Bp[1] = (B.ndim > 1) ? (F2[c] / B.Gdet(face2, j, i) + F2[c + B.n1] / B.Gdet(face2, j + 1, i)) / 2
                         : F2[c] / B.Gdet(face2, j, i);
    Bp[2] = (B.ndim > 2) ? (F3[c] / B.Gdet(face3, j, i) + F3[c + (size_t)B.n1*B.n2] / B.Gdet(face3, j, i)) / 2
                         : F3[c] / B.Gdet(face3, j, i);
}

// B_CT::CalculateEMF (b_ct.cpp:262-410) into emf[3][N] (E1, E2, E3 at the edges of zone (k,j,i)'s
// lower corner lines) over [is, ie+1] x [js, je+1] x [ks, ke(+1 in 3D)]
static void ct_calculate_emf(const Block& B, double* F[3], const double* P, double* emf)
{
    const size_t N = B.N, sj = B.n1, sk = (size_t)B.n1*B.n2;
    const size_t V1 = 5*N, V2 = 6*N, V3 = 7*N;
    const int scheme = B.c.ct_scheme;
    const int h3 = B.ndim > 2;
    std::vector<double> emfc;
    if (scheme != CT_BS99) {
        // zone-centred EMF (b_ct.cpp:331-345) over the interior +-1
        emfc.assign(3*N, 0.);
        for (int k = B.ks - h3; k <= B.ke + h3; ++k) for (int j = B.js - 1; j <= B.je + 1; ++j)
        for (int i = B.is - 1; i <= B.ie + 1; ++i) {
            const size_t c = B.id(k, j, i);
            double Pc[8];
            load_cell(B, P, c, Pc);
            FourVectors D;
            calc_4vecs(B, Pc, true, j, i, center, D);
            const double gdet = B.Gdet(center, j, i);
            emfc[c]       = (D.bcon[2]*D.ucon[3] - D.bcon[3]*D.ucon[2]) * gdet;
            emfc[N + c]   = (D.bcon[3]*D.ucon[1] - D.bcon[1]*D.ucon[3]) * gdet;
            emfc[2*N + c] = (D.bcon[1]*D.ucon[2] - D.bcon[2]*D.ucon[1]) * gdet;
        }
    }
    const double* f1 = F[0]; const double* f2 = F[1]; const double* f3 = F[2];
    auto ec = [&](int v, size_t x) { return emfc[v*N + x]; };
    for (int k = B.ks; k <= B.ke + h3; ++k) for (int j = B.js; j <= B.je + 1; ++j) for (int i = B.is; i <= B.ie + 1; ++i) {
        const size_t c = B.id(k, j, i);
        double e1, e2, e3;
        if (B.ndim > 2) {
            e1 = 0.25*(-f2[V3 + c - sk] - f2[V3 + c] + f3[V2 + c - sj] + f3[V2 + c]);
            e2 = 0.25*(-f3[V1 + c - 1] - f3[V1 + c] + f1[V3 + c - sk] + f1[V3 + c]);
            e3 = 0.25*(-f1[V2 + c - sj] - f1[V2 + c] + f2[V1 + c - 1] + f2[V1 + c]);
        } else {
            e1 = -f2[V3 + c];
            e2 = f1[V3 + c];
            e3 = 0.25*(-f1[V2 + c - sj] - f1[V2 + c] + f2[V1 + c - 1] + f2[V1 + c]);
        }
        if (scheme == CT_GS05_0) {
            if (B.ndim > 2) {
                e1 = 2 * e1 - 0.25*(ec(0, c) + ec(0, c - sj) + ec(0, c - sj) + ec(0, c - sk - sj));
                e2 = 2 * e2 - 0.25*(ec(1, c) + ec(1, c - 1) + ec(1, c - sk) + ec(1, c - sk - 1));
            }
            e3 = 2 * e3 - 0.25*(ec(2, c) + ec(2, c - 1) + ec(2, c - sj) + ec(2, c - sj - 1));
        } else if (scheme == CT_GS05_C) {
            if (B.ndim > 2) {
                const double e1_l3 = (f2[c - sk] >= 0.0) ? f3[V2 + c - sj] - ec(0, c - sk - sj) : f3[V2 + c] - ec(0, c - sk);
                const double e1_r3 = (f2[c] >= 0.0) ? f3[V2 + c - sj] - ec(0, c - sj) : f3[V2 + c] - ec(0, c);
                const double e1_l2 = (f3[c - sj] >= 0.0) ? -f2[V3 + c - sk] - ec(0, c - sk - sj) : -f2[V3 + c] - ec(0, c - sj);
                const double e1_r2 = (f3[c] >= 0.0) ? -f2[V3 + c - sk] - ec(0, c - sk) : -f2[V3 + c] - ec(0, c);
                e1 += 0.25*(e1_l3 + e1_r3 + e1_l2 + e1_r2);
                const double e2_l3 = (f1[c - sk] >= 0.0) ? -f3[V1 + c - 1] - ec(1, c - sk - 1) : -f3[V1 + c] - ec(1, c - sk);
                const double e2_r3 = (f1[c] >= 0.0) ? -f3[V1 + c - 1] - ec(1, c - 1) : -f3[V1 + c] - ec(1, c);
                const double e2_l1 = (f3[c - 1] >= 0.0) ? f1[V3 + c - sk] - ec(1, c - sk - 1) : f1[V3 + c] - ec(1, c - 1);
                const double e2_r1 = (f3[c] >= 0.0) ? f1[V3 + c - sk] - ec(1, c - sk) : f1[V3 + c] - ec(1, c);
                e2 += 0.25*(e2_l3 + e2_r3 + e2_l1 + e2_r1);
            }
            const double e3_l2 = (f1[c - sj] >= 0.0) ? f2[V1 + c - 1] - ec(2, c - sj - 1) : f2[V1 + c] - ec(2, c - sj);
            const double e3_r2 = (f1[c] >= 0.0) ? f2[V1 + c - 1] - ec(2, c - 1) : f2[V1 + c] - ec(2, c);
            const double e3_l1 = (f2[c - 1] >= 0.0) ? -f1[V2 + c - sj] - ec(2, c - sj - 1) : -f1[V2 + c] - ec(2, c - 1);
            const double e3_r1 = (f2[c] >= 0.0) ? -f1[V2 + c - sj] - ec(2, c - sj) : -f1[V2 + c] - ec(2, c);
            e3 += 0.25*(e3_l2 + e3_r2 + e3_l1 + e3_r1);
        }
        emf[c] = e1; emf[N + c] = e2; emf[2*N + c] = e3;
    }
}

// B_CT::AddSource (b_ct.cpp:412-470) and the face RK combination (WeightedSumDataFace twice)
static void ct_update_faces(const Block& B, const double* emf, int s, double dt, const double* Bs, const double* B0,
                            double* Bn)
{
    const size_t N = B.N, sj = B.n1, sk = (size_t)B.n1*B.n2;
    const double g0 = RK_GAM0[s], g1 = RK_GAM1[s], bdt = RK_BETA[s] * dt;
    const double L1 = B.c.dx1, L2 = B.c.dx2, L3 = B.c.dx3;
    const bool d3 = B.ndim > 2;
    auto E = [&](int v, size_t x) { return emf[v*N + x]; };
    for (int k = B.ks; k <= B.ke + d3; ++k) for (int j = B.js; j <= B.je + 1; ++j) for (int i = B.is; i <= B.ie + 1; ++i) {
        const size_t c = B.id(k, j, i);
        if (j <= B.je && k <= B.ke) {
            double db = (-L3 * E(2, c + sj) + L3 * E(2, c));
            if (d3) db += (L2 * E(1, c + sk) - L2 * E(1, c));
            db /= (L2 * L3);
            const double x = g0 * Bs[c] + g1 * B0[c];
            Bn[c] = 1.0 * x + bdt * db;
        }
        if (i <= B.ie && k <= B.ke) {
            double db = (L3 * E(2, c + 1) - L3 * E(2, c));
            if (d3) db += (-L1 * E(0, c + sk) + L1 * E(0, c));
            db /= (L1 * L3);
            const double x = g0 * Bs[N + c] + g1 * B0[N + c];
            Bn[N + c] = 1.0 * x + bdt * db;
        }
        if (i <= B.ie && j <= B.je) {
            const double db = (-L2 * E(1, c + 1) + L2 * E(1, c) + L1 * E(0, c + sj) - L1 * E(0, c)) / (L1 * L2);
            const double x = g0 * Bs[2*N + c] + g1 * B0[2*N + c];
            Bn[2*N + c] = 1.0 * x + bdt * db;
        }
    }
}

// ---- B_CT at physical faces (boundaries.cpp:186-207 defaults, 432-490; b_ct_boundaries.cpp:40-262)
// Reflecting faces zero the EMFs on the edges lying in the domain face (zero_EMF), before the face
// update.  After the stage, each physical face (x1 faces, x2 faces, then inner x1 again with
// fix_corner) fills the face field's ghost layers: tangential components copy as zones do
// (outflow: the first interior layer; reflecting: the mirror zone, no sign change), the normal
// component is the reflected face vector (reflect_face_vector: zero on the domain face, minus the
// mirror face beyond it) or, on outflow faces, is rebuilt layer by layer outward from the domain face
// so that every zone it closes has zero divergence (clean_face_B, DestructiveBoundaryClean).  The
// ghost zones then take B from their faces (B_CT::BlockUtoP over the boundary domain).  The arrays
// hold faces 0..n-1 per direction (face n, the top of the last ghost layer, is not stored): the
// cleaning leaves the last transverse ghost layer as copied, and the last ghost zone layer takes its
// normal B from its one stored face; with ng >= 4 neither reaches an interior flux.
static void ct_zero_boundary_emf(const Block& B, double* emf)
{
    const size_t N = B.N;
    for (int face = 0; face < 2*B.ndim; ++face) {
        if (B.c.bc[face] == BC_TRANSMIT) {
            // average_EMF (b_ct_boundaries.cpp:64-186) on a transmitting X2 face: E3 zero on the polar
            // face (spherical coordinates: the edges have no length), E1 replaced by its average over
            // the interior x3 edges (3D; in 2D E1 is left alone).  The reference's team reduction has
            // no fixed order; the sum here runs over k upwards.
            const int jf = (face == 2) ? B.js : B.je + 1;
            if (B.C.spherical())
                for (int k = 0; k < B.n3; ++k) for (int i = 0; i < B.n1; ++i) emf[2*N + B.id(k, jf, i)] = 0.;
            if (B.ndim > 2)
                for (int i = 0; i < B.n1; ++i) {
                    double sum = 0.;
                    for (int k = B.ks; k <= B.ke; ++k) sum += emf[B.id(k, jf, i)];
                    const double av = sum / (B.ke + 1 - B.ks);
                    for (int k = 0; k < B.n3; ++k) emf[B.id(k, jf, i)] = av;
                }
            continue;
        }
        if (B.c.bc[face] != BC_REFLECT) continue;
        const int bdir = face / 2 + 1;
        const bool binner = (face % 2) == 0;
        const int f = (bdir == 1) ? (binner ? B.is : B.ie + 1) : (bdir == 2) ? (binner ? B.js : B.je + 1)
                                                                            : (binner ? B.ks : B.ke + 1);
        for (int k = 0; k < B.n3; ++k) for (int j = 0; j < B.n2; ++j) for (int i = 0; i < B.n1; ++i) {
            const int x = (bdir == 1) ? i : (bdir == 2) ? j : k;
            if (x != f) continue;
            for (int v = 0; v < 3; ++v)
                if (v != bdir - 1) emf[(size_t)v*N + B.id(k, j, i)] = 0.;
        }
    }
}

static void ct_face_boundary(const Block& B, double* Bf, int face)
{
    const size_t N = B.N;
    const int bdir = face / 2 + 1;
    const bool binner = (face % 2) == 0;
    const int type = B.c.bc[face];
    const int n[3] = {B.n1, B.n2, B.n3};
    const int s = (bdir == 1) ? B.is : (bdir == 2) ? B.js : B.ks;
    const int e = (bdir == 1) ? B.ie : (bdir == 2) ? B.je : B.ke;
    const int nb = n[bdir - 1];
    const int f = binner ? s : e + 1;                       // the domain face
    auto at = [&](int v, int k, int j, int i) -> double& { return Bf[(size_t)v*N + B.id(k, j, i)]; };
    auto idx = [&](int k, int j, int i) { return (bdir == 1) ? i : (bdir == 2) ? j : k; };
    auto moved = [&](int k, int j, int i, int x) {
        if (bdir == 1) i = x; else if (bdir == 2) j = x; else k = x;
        return B.id(k, j, i);
    };
    // tangential components: zone-like ghost layers (Parthenon's outflow / reflect)
    for (int v = 0; v < 3; ++v) {
        if (v == bdir - 1 || type == BC_TRANSMIT) continue;
        for (int k = 0; k < B.n3; ++k) for (int j = 0; j < B.n2; ++j) for (int i = 0; i < B.n1; ++i) {
            const int x = idx(k, j, i);
            if (binner ? x >= s : x <= e) continue;
            const int src = (type == BC_OUTFLOW) ? (binner ? s : e) : (binner ? 2*s - 1 - x : 2*e + 1 - x);
            at(v, k, j, i) = Bf[(size_t)v*N + moved(k, j, i, src)];
        }
    }
    const int v = bdir - 1;
    if (type == BC_TRANSMIT) {
        // OneBlockTransmit on the face field (one_block_transmit.cpp:60-143, X2 faces): the mirror
        // face half-way round in x3; F2 and F3 inverted, F2 zero on the polar face itself
        const int nx3 = B.c.nx3;
        auto ki_of = [&](int k) { return ((k - B.ks + nx3 / 2) % nx3) + B.ks; };
        for (int k = 0; k < B.n3; ++k) for (int j = 0; j < B.n2; ++j) for (int i = 0; i < B.n1; ++i) {
            const int ki = ki_of(k);
            if (ki < 0 || ki >= B.n3) continue;
            if (binner ? j < s : j > e) {                  // F1 and F3: zone-like layers
                const int ji = binner ? 2*s - 1 - j : 2*e + 1 - j;
                at(0, k, j, i) = Bf[B.id(ki, ji, i)];
                at(2, k, j, i) = -Bf[2*N + B.id(ki, ji, i)];
            }
            if (binner ? j <= f : j >= f) {                // F2: the polar face and beyond
                const int ji = 2*f - j;
                if (ji < 0 || ji >= nb) continue;
                at(1, k, j, i) = (j == f) ? 0. : -Bf[N + B.id(ki, ji, i)];
            }
        }
        return;
    }
    if (type == BC_REFLECT) {
        // reflect_face_vector (boundaries.cpp:458-479): zero on the domain face, minus the mirror face
        for (int k = 0; k < B.n3; ++k) for (int j = 0; j < B.n2; ++j) for (int i = 0; i < B.n1; ++i) {
            const int x = idx(k, j, i);
            if (binner ? x > f : x < f) continue;
            const int m = 2*f - x;
            if (m < 0 || m >= nb) continue;
            at(v, k, j, i) = (x == f) ? 0. : -Bf[(size_t)v*N + moved(k, j, i, m)];
        }
        return;
    }
    // outflow: Parthenon's copy of the domain face into the ghost faces, then clean_face_B
    for (int k = 0; k < B.n3; ++k) for (int j = 0; j < B.n2; ++j) for (int i = 0; i < B.n1; ++i) {
        const int x = idx(k, j, i);
        if (binner ? x >= f : x <= f) continue;
        at(v, k, j, i) = Bf[(size_t)v*N + moved(k, j, i, f)];
    }
    // DestructiveBoundaryClean (b_ct_boundaries.cpp:190-262): from the domain face outward, each face
    // closes the zone between it and the previous one with zero divergence
    const double A1 = B.c.dx2 * B.c.dx3, A2 = B.c.dx1 * B.c.dx3, A3 = B.c.dx1 * B.c.dx2;
    const int osign = binner ? -1 : 1;
    const double nsign = (double)(-(-osign));
    const int d3 = B.ndim > 2;
    for (int layer = 0; layer < nb; ++layer) {
        const int x = binner ? f - layer : f + layer;
        if (x < 0 || x > nb - 1) break;
        const int lf = binner ? x + 1 : x - 1, lc = binner ? x : x - 1;
        if (bdir == 1) {
            for (int k = 0; k < B.n3 - d3; ++k) for (int j = 0; j < B.n2 - 1; ++j) {
                double nf = nsign * at(0, k, j, lf) * A1 - (at(1, k, j + 1, lc) * A2 - at(1, k, j, lc) * A2);
                if (d3) nf -= at(2, k + 1, j, lc) * A3 - at(2, k, j, lc) * A3;
                at(0, k, j, x) = (double)osign * nf / A1;
            }
        } else if (bdir == 3) {
            // X3 faces (b_ct_boundaries.cpp:249-268), layers along k over the face plane (the
            // reference's loop takes its k range from the face's i bounds, which only its intent, the
            // k layers, can mean)
            for (int j = 0; j < B.n2 - 1; ++j) for (int i = 0; i < B.n1 - 1; ++i) {
                const double nf = nsign * at(2, lf, j, i) * A3 - (at(0, lc, j, i + 1) * A1 - at(0, lc, j, i) * A1)
                                  - (at(1, lc, j + 1, i) * A2 - at(1, lc, j, i) * A2);
                at(2, x, j, i) = (double)osign * nf / A3;
            }
        } else {
            for (int k = 0; k < B.n3 - d3; ++k) for (int i = 0; i < B.n1 - 1; ++i) {
                double nf = nsign * at(1, k, lf, i) * A2 - (at(0, k, lc, i + 1) * A1 - at(0, k, lc, i) * A1);
                if (d3) nf -= at(2, k + 1, lc, i) * A3 - at(2, k, lc, i) * A3;
                at(1, k, x, i) = (double)osign * nf / A2;
            }
        }
    }
}

// Ghost zones of the physical directions: B from the faces, sqrt(-g) B as conserved B
static void ct_ghost_zone_b(const Block& B, const double* Bf, double* P, double* U)
{
    const size_t N = B.N;
    const bool ph1 = phys_face(B.c.bc[0]), ph2 = B.ndim > 1 && phys_face(B.c.bc[2]);
    const bool ph3 = B.ndim > 2 && phys_face(B.c.bc[4]);
    for (int k = 0; k < B.n3; ++k) for (int j = 0; j < B.n2; ++j) for (int i = 0; i < B.n1; ++i) {
        const bool gi = i < B.is || i > B.ie, gj = j < B.js || j > B.je, gk = k < B.ks || k > B.ke;
        if (!((gi && ph1) || (gj && ph2) || (gk && ph3))) continue;
        if ((gi && !ph1) || (gj && !ph2) || (gk && !ph3)) continue;     // periodic images fill these
        double Bp[3];
        const size_t c = B.id(k, j, i);
        const double* F1 = Bf; const double* F2 = Bf + N; const double* F3 = Bf + 2*N;
        Bp[0] = (i == B.n1 - 1) ? F1[c] / B.Gdet(face1, j, i)
                                : (F1[c] / B.Gdet(face1, j, i) + F1[c + 1] / B.Gdet(face1, j, i + 1)) / 2;
        Bp[1] = (B.ndim > 1 && j < B.n2 - 1) ? (F2[c] / B.Gdet(face2, j, i) + F2[c + B.n1] / B.Gdet(face2, j + 1, i)) / 2
                                             : F2[c] / B.Gdet(face2, j, i);
        Bp[2] = (B.ndim > 2 && k < B.n3 - 1) ? (F3[c] / B.Gdet(face3, j, i) + F3[c + (size_t)B.n1*B.n2] / B.Gdet(face3, j, i)) / 2
                                             : F3[c] / B.Gdet(face3, j, i);
        for (int v = 0; v < 3; ++v) {
            P[(size_t)(5 + v)*N + c] = Bp[v];
            U[(size_t)(5 + v)*N + c] = Bp[v] * B.Gdet(center, j, i);
        }
    }
}

// The ghost zones of a B_CT block with physical faces: faces first, then the zone boundaries as
// apply_boundaries fills them, with the zone B of the physical directions' ghost zones from the faces
// (before the periodic images are taken again)
static bool ct_has_physical(const Block& B)
{
    for (int face = 0; face < 2*B.ndim; ++face) if (phys_face(B.c.bc[face])) return true;
    return false;
}
static void ct_apply_boundaries(const Block& B, double* P, double* U, double* Bf)
{
    for (int face = 0; face < 2*B.ndim; ++face) {
        if (!phys_face(B.c.bc[face])) continue;
        ct_face_boundary(B, Bf, face);
        if (face == 3 && B.c.fix_corner_inner && phys_face(B.c.bc[0])) ct_face_boundary(B, Bf, 0);
    }
    apply_boundaries(B, P, U);
    ct_ghost_zone_b(B, Bf, P, U);
    for (int d = 1; d <= B.ndim; ++d)
        if (B.c.bc[2*(d-1)] == BC_PERIODIC) { periodic_fill(B, P, B.nv, d); periodic_fill(B, U, B.nv, d); }
}

// One RK stage with B_CT (kharma_step.cpp:163-214, use_b_ct): fluxes, FixFlux without flux-CT, EMFs,
// face update, the cell update, the zone B (and sqrt(-g) B) from the new faces, inversion, floors,
// fixups, boundaries and P->U as stage() does
static void ct_stage(const Block& B, Fields& f, int s, double dt, const double* P_s, const double* U_s,
                     const double* U_0, const double* Bs, const double* B0, double* P_n, double* U_n, double* Bn,
                     double* pflag, double* fflag)
{
    const size_t N = B.N, NV = (size_t)B.nv*N;
    for (int d = 1; d <= B.ndim; ++d)
        get_flux(B, d, P_s, f.F[d-1].data(), f.cmax[d-1].data(), f.cmin[d-1].data());
    double* F[3] = {f.F[0].data(), f.F[1].data(), f.F[2].data()};
    boundaries_fix_flux(B, F);
    std::vector<double> emf(3*N, 0.);
    ct_calculate_emf(B, F, P_s, emf.data());
    ct_zero_boundary_emf(B, emf.data());
    ct_update_faces(B, emf.data(), s, dt, Bs, B0, Bn);
    std::vector<double> dudt(NV, 0.);
    flux_divergence(B, F, dudt.data());
    add_geo_source(B, P_s, dudt.data());
    const double g0 = RK_GAM0[s], g1 = RK_GAM1[s], bdt = RK_BETA[s] * dt;
    for (size_t x = 0; x < NV; ++x) U_n[x] = g0 * U_s[x] + g1 * U_0[x];
    for (size_t x = 0; x < NV; ++x) U_n[x] = 1.0 * U_n[x] + bdt * dudt[x];
    // the zone B follows the faces (cons.B is derived, not updated by its flux divergence)
    for (int k = B.ks; k <= B.ke; ++k) for (int j = B.js; j <= B.je; ++j) for (int i = B.is; i <= B.ie; ++i) {
        double Bp[3];
        ct_zone_b(B, Bn, k, j, i, Bp);
        const size_t c = B.id(k, j, i);
        for (int v = 0; v < 3; ++v) U_n[(size_t)(5 + v)*N + c] = Bp[v] * B.Gdet(center, j, i);
    }
    // inversion guess and the ghost shell (exchange faces keep theirs; periodic ones are refreshed)
    if (P_n != P_s) std::memcpy(P_n, P_s, NV*sizeof(double));
    for (size_t x = 0; x < N; ++x) { pflag[x] = 0; fflag[x] = 0; }
    block_utop(B, U_n, P_n, pflag, fflag, B.ks, B.ke, B.js, B.je, B.is, B.ie);
    for (int k = B.ks; k <= B.ke; ++k) for (int j = B.js; j <= B.je; ++j) for (int i = B.is; i <= B.ie; ++i) {
        double Bp[3];
        ct_zone_b(B, Bn, k, j, i, Bp);
        for (int v = 0; v < 3; ++v) P_n[(size_t)(5 + v)*N + B.id(k, j, i)] = Bp[v];
    }
    if (B.c.floors_on) apply_grmhd_floors(B, P_n, U_n, pflag, fflag, B.ks, B.ke, B.js, B.je, B.is, B.ie);
    stage_fix_utop(B, P_n, U_n, pflag);
    if (!ct_has_physical(B)) { finish_stage(B, P_n, U_n); return; }
    ct_apply_boundaries(B, P_n, U_n, Bn);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < B.n3; ++k) for (int j = 0; j < B.n2; ++j) for (int i = 0; i < B.n1; ++i)
        p_to_u_cell(B, P_n, U_n, B.id(k, j, i), j, i);
}

// ======================================================================== EMHD and the implicit solve
// Extended GRMHD (emhd/) and the per-zone Newton solve (implicit/).  Zone state for these
// functions is a 10-slot array: rho, u, u1..u3, B1..B3 (slots 0-7 as above), q~ (8), dP~ (9).
// Field arrays are [10][N] in the same slot order.
static const int IQ = 8, IDP = 9, NVE = 10;

enum Closure { CL_CONSTANT = 0, CL_SOUNDSPEED = 1, CL_KAPPA_ETA = 2, CL_TORUS = 3 };   // emhd.hpp:58
struct EmhdParams {            // emhd.hpp:60-84 plus the package switches of emhd.cpp:60-72, 118-125
    int32_t type, higher_order_terms, feedback, conduction, viscosity, stability_limits;
    double tau, conduction_alpha, viscosity_alpha, kappa, eta;
};
struct ImplicitParams {        // implicit.cpp:99-119 (jacobian: 0 finite difference, 1 exact)
    int32_t min_nonlinear_iter, max_nonlinear_iter, use_qr, linesearch, max_linesearch_iter, jacobian;
    double jacobian_delta, rootfind_tol, linesearch_eps, linesearch_lambda;
};
enum { SOLVE_CONVERGED = 0, SOLVE_FAIL = 1, SOLVE_BEYOND_TOL = 2, SOLVE_BACKTRACK = 3 };   // implicit.hpp:63-69

// The implicitly evolved variables in the reference's pack order (Implicit::GetOrderedNames,
// implicit.cpp:64-83: implicit-flagged first): rho, u, uvec, then q and dP when present.
static int implicit_map(const EmhdParams& ep, int map[7])
{
    int n = 0;
    for (int p = 0; p < 5; ++p) map[n++] = p;
    if (ep.conduction) map[n++] = IQ;
    if (ep.viscosity) map[n++] = IDP;
    return n;
}

// Forward-mode dual number with NDIR tangent directions.  The oracle's exact Jacobian is the
// residual below evaluated on Dual inputs seeded with unit vectors; the value part performs
// the same IEEE operations as the plain double evaluation.
static const int NDIR = 7;
struct Dual {
    double v, d[NDIR];
    Dual() : v(0.) { for (int k = 0; k < NDIR; ++k) d[k] = 0.; }
    Dual(double x) : v(x) { for (int k = 0; k < NDIR; ++k) d[k] = 0.; }
};
static inline Dual operator+(const Dual& a, const Dual& b) { Dual r(a.v + b.v); for (int k = 0; k < NDIR; ++k) r.d[k] = a.d[k] + b.d[k]; return r; }
static inline Dual operator-(const Dual& a, const Dual& b) { Dual r(a.v - b.v); for (int k = 0; k < NDIR; ++k) r.d[k] = a.d[k] - b.d[k]; return r; }
static inline Dual operator-(const Dual& a) { Dual r(-a.v); for (int k = 0; k < NDIR; ++k) r.d[k] = -a.d[k]; return r; }
static inline Dual operator*(const Dual& a, const Dual& b)
{ Dual r(a.v * b.v); for (int k = 0; k < NDIR; ++k) r.d[k] = a.d[k]*b.v + a.v*b.d[k]; return r; }
static inline Dual operator/(const Dual& a, const Dual& b)
{ Dual r(a.v / b.v); for (int k = 0; k < NDIR; ++k) r.d[k] = (a.d[k]*b.v - a.v*b.d[k]) / (b.v*b.v); return r; }
static inline Dual operator+(const Dual& a, double b) { Dual r(a); r.v = a.v + b; return r; }
static inline Dual operator+(double a, const Dual& b) { Dual r(b); r.v = a + b.v; return r; }
static inline Dual operator-(const Dual& a, double b) { Dual r(a); r.v = a.v - b; return r; }
static inline Dual operator-(double a, const Dual& b) { Dual r(a - b.v); for (int k = 0; k < NDIR; ++k) r.d[k] = -b.d[k]; return r; }
static inline Dual operator*(const Dual& a, double b) { Dual r(a.v * b); for (int k = 0; k < NDIR; ++k) r.d[k] = a.d[k]*b; return r; }
static inline Dual operator*(double a, const Dual& b) { Dual r(a * b.v); for (int k = 0; k < NDIR; ++k) r.d[k] = a*b.d[k]; return r; }
static inline Dual operator/(const Dual& a, double b) { Dual r(a.v / b); for (int k = 0; k < NDIR; ++k) r.d[k] = a.d[k]/b; return r; }
static inline Dual operator/(double a, const Dual& b)
{ Dual r(a / b.v); for (int k = 0; k < NDIR; ++k) r.d[k] = -a*b.d[k]/(b.v*b.v); return r; }
static inline Dual& operator+=(Dual& a, const Dual& b) { a = a + b; return a; }
static inline Dual& operator-=(Dual& a, const Dual& b) { a = a - b; return a; }
static inline Dual& operator*=(Dual& a, const Dual& b) { a = a * b; return a; }
static inline Dual& operator+=(Dual& a, double b) { a = a + b; return a; }
static inline Dual& operator-=(Dual& a, double b) { a = a - b; return a; }
static inline Dual& operator*=(Dual& a, double b) { a = a * b; return a; }
static inline double tval(double x) { return x; }
static inline double tval(const Dual& x) { return x.v; }
static inline double tsqrt(double x) { return std::sqrt(x); }
static inline Dual tsqrt(const Dual& a)
{ Dual r(std::sqrt(a.v)); for (int k = 0; k < NDIR; ++k) r.d[k] = a.d[k] / (2. * r.v); return r; }
// m::max(x, c) with a constant c: derivative of the selected branch
template <class T> static inline T tmax(const T& x, double c) { return (tval(x) < c) ? T(c) : x; }

template <class T> struct FV { T ucon[4], ucov[4], bcon[4], bcov[4]; };
template <class T> static inline T tdot(const T* a, const T* b) { return a[0]*b[0] + a[1]*b[1] + a[2]*b[2] + a[3]*b[3]; }

// GRMHD::calc_ucon at the zone centre (grmhd_functions.hpp:121-133, 282-291)
template <class T>
static void calc_ucon_t(const Block& B, const T* P, int j, int i, T ucon[4])
{
    const int loc = center;
    const T qsq = B.Gcov(loc, j, i, 1, 1) * P[2] * P[2] +
                  B.Gcov(loc, j, i, 2, 2) * P[3] * P[3] +
                  B.Gcov(loc, j, i, 3, 3) * P[4] * P[4] +
                  2. * (B.Gcov(loc, j, i, 1, 2) * P[2] * P[3] +
                        B.Gcov(loc, j, i, 1, 3) * P[2] * P[4] +
                        B.Gcov(loc, j, i, 2, 3) * P[3] * P[4]);
    const T gamma = tsqrt(1. + qsq);
    const double alpha = 1. / std::sqrt(-B.Gcon(loc, j, i, 0, 0));
    ucon[0] = gamma / alpha;
    for (int v = 0; v < 3; ++v) ucon[v+1] = P[2 + v] - gamma * alpha * B.Gcon(loc, j, i, 0, v+1);
}
// GRCoordinates::lower at the centre (gr_coordinates.hpp:227-232)
template <class T>
static void lower_t(const Block& B, const T* vcon, T* vcov, int j, int i)
{
    for (int mu = 0; mu < 4; ++mu) vcov[mu] = T(0.);
    for (int mu = 0; mu < 4; ++mu) for (int nu = 0; nu < 4; ++nu) vcov[mu] += B.Gcov(center, j, i, mu, nu) * vcon[nu];
}
// GRMHD::calc_4vecs at the centre with B (grmhd_functions.hpp:225-246)
template <class T>
static void calc_4vecs_t(const Block& B, const T* P, int j, int i, FV<T>& D)
{
    calc_ucon_t(B, P, j, i, D.ucon);
    lower_t(B, D.ucon, D.ucov, j, i);
    D.bcon[0] = T(0.);
    for (int v = 0; v < 3; ++v) D.bcon[0] += P[5 + v] * D.ucov[v+1];
    for (int v = 0; v < 3; ++v) D.bcon[v+1] = (P[5 + v] + D.bcon[0] * D.ucon[v+1]) / D.ucon[0];
    lower_t(B, D.bcon, D.bcov, j, i);
}

// EMHD::set_parameters, scalar form (emhd.hpp:179-261)
static void emhd_set_parameters(const Block& B, const EmhdParams& ep, double gam, double rho, double u,
                                double qtilde, double dPtilde, double bsq, int j, int i,
                                double& tau, double& chi_e, double& nu_e)
{
    if (ep.type == CL_CONSTANT) {
        tau = ep.tau;
        chi_e = ep.conduction_alpha;
        nu_e = ep.viscosity_alpha;
    } else if (ep.type == CL_SOUNDSPEED) {
        const double cs2 = (gam * (gam - 1.) * u) / (rho + (gam * u));
        tau = ep.tau;
        chi_e = ep.conduction_alpha * cs2 * tau;
        nu_e = ep.viscosity_alpha * cs2 * tau;
    } else if (ep.type == CL_KAPPA_ETA) {
        tau = ep.tau;
        chi_e = ep.kappa / kmax(rho, SMALL);
        nu_e = ep.eta / kmax(rho, SMALL);
    } else {
        const double r = B.rcen[(size_t)j*B.n1 + i];
        const double tau_dyn = std::sqrt(r*r*r);
        tau = tau_dyn;
        const double pg = (gam - 1.) * u;
        const double Theta = pg / rho;
        const double cs2 = clip(gam * pg / (rho + (gam * u)), SMALL, 0./0.);
        const double lambda = 0.01;
        {
            const double q = (ep.higher_order_terms)
                ? qtilde * std::sqrt(rho * ep.conduction_alpha * cs2 * Theta * Theta) : qtilde;
            const double q_max = ep.conduction_alpha * rho * cs2 * std::sqrt(cs2);
            const double q_ratio = std::fabs(q) / q_max;
            const double inv_exp_g = std::exp(-(q_ratio - 1.) / lambda);
            const double f_fmin = inv_exp_g / (inv_exp_g + 1.) + 1.e-5;
            tau = kmin(tau, f_fmin * tau_dyn);
        }
        {
            const double dP = (ep.higher_order_terms)
                ? dPtilde * std::sqrt(rho * ep.viscosity_alpha * cs2 * Theta) : dPtilde;
            const double dP_comp_ratio = kmax(pg - 2./3. * dP, SMALL) / kmax(pg + 1./3. * dP, SMALL);
            const double dP_max = (dP > 0.) ? kmin(0.5 * bsq * dP_comp_ratio, 1.49 * pg / 1.07)
                                            : kmax(-bsq, -2.99 * pg / 1.07);
            const double dP_ratio = std::fabs(dP) / (std::fabs(dP_max) + SMALL);
            const double inv_exp_g = std::exp((1. - dP_ratio) / lambda);
            const double f_fmin = inv_exp_g / (inv_exp_g + 1.) + 1.e-5;
            tau = kmin(tau, f_fmin * tau_dyn);
        }
        const double max_alpha = (1 - cs2) / (2 * cs2 + 1.e-12);
        chi_e = kmin(max_alpha, ep.conduction_alpha) * cs2 * tau;
        nu_e = kmin(max_alpha, ep.viscosity_alpha) * cs2 * tau;
    }
}
// EMHD::set_parameters on a zone's primitives (emhd.hpp:262-287)
static void emhd_set_parameters_P(const Block& B, const EmhdParams& ep, double gam, const double* P, int j, int i,
                                  double& tau, double& chi_e, double& nu_e)
{
    FV<double> D;
    calc_4vecs_t(B, P, j, i, D);
    const double bsq = kmax(tdot(D.bcon, D.bcov), SMALL);
    const double qtilde = ep.conduction ? P[IQ] : 0.;
    const double dPtilde = ep.viscosity ? P[IDP] : 0.;
    emhd_set_parameters(B, ep, gam, P[0], P[1], qtilde, dPtilde, bsq, j, i, tau, chi_e, nu_e);
}
// EMHD::convert_prims_to_q_dP (emhd.hpp:313-332)
template <class T>
static void convert_prims_to_q_dP_t(const T& q_tilde, const T& dP_tilde, const T& rho, const T& Theta,
                                    const T& cs2, const EmhdParams& ep, T& q, T& dP)
{
    q = q_tilde;
    if (ep.higher_order_terms) {
        if (ep.type == CL_KAPPA_ETA) q *= tsqrt(ep.kappa * Theta * Theta / ep.tau);
        else                         q *= tsqrt(rho * ep.conduction_alpha * cs2 * Theta * Theta);
    }
    dP = dP_tilde;
    if (ep.higher_order_terms) {
        if (ep.type == CL_KAPPA_ETA) dP *= tsqrt(ep.eta * Theta / ep.tau);
        else                         dP *= tsqrt(rho * ep.viscosity_alpha * cs2 * Theta);
    }
}
// Flux::calc_tensor with the EMHD / GRMHD branches (flux_functions.hpp:80-107, emhd.hpp:296-309,
// grmhd_functions.hpp:142-155)
template <class T>
static void calc_tensor_t(const EmhdParams& ep, double gam, const T* P, const FV<T>& D, int dir, T Tm[4])
{
    if ((ep.conduction || ep.viscosity) && ep.feedback) {
        const T qtilde = ep.conduction ? P[IQ] : T(0.);
        const T dPtilde = ep.viscosity ? P[IDP] : T(0.);
        const T Theta = (gam - 1) * P[1] / P[0];
        const T cs2 = gam * (gam - 1) * P[1] / (P[0] + gam * P[1]);
        T q, dP;
        convert_prims_to_q_dP_t(qtilde, dPtilde, P[0], Theta, cs2, ep, q, dP);
        const T pgas = (gam - 1) * P[1];
        const T bsq = tmax(tdot(D.bcon, D.bcov), SMALL);
        const T b_mag = tsqrt(bsq);
        const T eta = pgas + P[0] + P[1] + bsq;
        const T ptot = pgas + 0.5 * bsq;
        for (int mu = 0; mu < 4; ++mu)
            Tm[mu] = eta * D.ucon[dir] * D.ucov[mu] + ptot * (double)(dir == mu) - D.bcon[dir] * D.bcov[mu]
                   + (q / b_mag) * ((D.ucon[dir] * D.bcov[mu]) + (D.bcon[dir] * D.ucov[mu]))
                   - dP * ((D.bcon[dir] * D.bcov[mu] / bsq) - (1./3.) * ((double)(dir == mu) + D.ucon[dir] * D.ucov[mu]));
    } else {
        const T pgas = (gam - 1) * P[1];
        const T bsq = tdot(D.bcon, D.bcov);
        const T eta = pgas + P[0] + P[1] + bsq;
        const T ptot = pgas + 0.5 * bsq;
        for (int mu = 0; mu < 4; ++mu)
            Tm[mu] = eta * D.ucon[dir] * D.ucov[mu] + ptot * (double)(dir == mu) - D.bcon[dir] * D.bcov[mu];
    }
}
// Flux::prim_to_flux for the 10-slot state at the centre (flux_functions.hpp:180-232)
template <class T>
static void prim_to_flux_t(const Block& B, const EmhdParams& ep, double gam, const T* P, const FV<T>& D,
                           int j, int i, int dir, T* flux)
{
    const double gdet = B.Gdet(center, j, i);
    flux[0] = P[0] * D.ucon[dir] * gdet;
    T Tm[4];
    calc_tensor_t(ep, gam, P, D, dir, Tm);
    flux[1] = Tm[0] * gdet + flux[0];
    flux[2] = Tm[1] * gdet;
    flux[3] = Tm[2] * gdet;
    flux[4] = Tm[3] * gdet;
    if (dir == 0) {
        for (int v = 0; v < 3; ++v) flux[5 + v] = P[5 + v] * gdet;
    } else {
        for (int v = 0; v < 3; ++v) flux[5 + v] = (D.bcon[v+1] * D.ucon[dir] - D.bcon[dir] * D.ucon[v+1]) * gdet;
    }
    if (ep.conduction) flux[IQ] = P[IQ] * D.ucon[dir] * gdet;
    if (ep.viscosity) flux[IDP] = P[IDP] * D.ucon[dir] * gdet;
}
// EMHD::implicit_sources (emhd_sources.hpp:52-63)
template <class T>
static void implicit_sources_t(const Block& B, const EmhdParams& ep, const T* P, double tau, int j, int i,
                               T& dUq, T& dUdP)
{
    if (ep.conduction) dUq = -B.Gdet(center, j, i) * (P[IQ] / tau);
    if (ep.viscosity) dUdP = -B.Gdet(center, j, i) * (P[IDP] / tau);
}
// EMHD::time_derivative_sources (emhd_sources.hpp:69-128); P_new is the trial state
template <class T>
static void time_derivative_sources_t(const Block& B, const EmhdParams& ep, const T* P_new, const double* P_old,
                                      const double* P, double tau, double chi_e, double nu_e,
                                      const FV<double>& D, double gam, double dt, int j, int i, T& dUq, T& dUdP)
{
    const bool ho = ep.higher_order_terms;
    const double bsq = kmax(tdot(D.bcon, D.bcov), SMALL);
    const double mag_b = std::sqrt(bsq);
    double ucon_o[4], ucov_old[4];
    T ucon_n[4], ucov_new[4];
    calc_ucon_t(B, P_old, j, i, ucon_o);
    lower_t(B, ucon_o, ucov_old, j, i);
    calc_ucon_t(B, P_new, j, i, ucon_n);
    lower_t(B, ucon_n, ucov_new, j, i);
    T dt_ucov[4];
    for (int mu = 0; mu < 4; ++mu) dt_ucov[mu] = (ucov_new[mu] - ucov_old[mu]) / dt;
    T div_ucon = T(0.);
    for (int mu = 0; mu < 4; ++mu) div_ucon += B.Gcon(center, j, i, 0, mu) * dt_ucov[mu];
    const T Theta_new = tmax((gam-1) * P_new[1] / P_new[0], SMALL);
    const double Theta_old = kmax((gam-1) * P_old[1] / P_old[0], SMALL);
    const T dt_Theta = (Theta_new - Theta_old) / dt;
    const double rho = P[0];
    const double Theta = (gam-1) * P[1] / P[0];
    if (ep.conduction) {
        const double qtilde = P[IQ];
        T q0 = -rho * chi_e * (D.bcon[0] / mag_b) * dt_Theta;
        for (int mu = 0; mu < 4; ++mu) q0 -= rho * chi_e * (D.bcon[mu] / mag_b) * Theta * D.ucon[0] * dt_ucov[mu];
        T q0_tilde = q0;
        if (ho) q0_tilde *= (chi_e != 0) ? std::sqrt(tau / (chi_e * rho * Theta * Theta)) : 0.0;
        dUq = B.Gdet(center, j, i) * (q0_tilde / tau);
        if (ho) dUq += B.Gdet(center, j, i) * (qtilde / 2.) * div_ucon;
    }
    if (ep.viscosity) {
        const double dPtilde = P[IDP];
        T dP0 = -rho * nu_e * div_ucon;
        for (int mu = 0; mu < 4; ++mu) dP0 += 3. * rho * nu_e * (D.bcon[0] * D.bcon[mu] / bsq) * dt_ucov[mu];
        T dP0_tilde = dP0;
        if (ho) dP0_tilde *= (nu_e != 0) ? std::sqrt(tau / (nu_e * rho * Theta)) : 0.0;
        dUdP = B.Gdet(center, j, i) * (dP0_tilde / tau);
        if (ho) dUdP += B.Gdet(center, j, i) * (dPtilde / 2.) * div_ucon;
    }
}
// Implicit::calc_residual (implicit.hpp:139-200).  Pi/Ui: full-step initial state; Ps: sub-step
// initial state; src: flux divergence plus explicit sources; dUi: implicit sources of Pi.
template <class T>
static void calc_residual_t(const Block& B, const EmhdParams& ep, double gam, const T* Pt, const double* Pi,
                            const double* Ui, const double* Ps, const double* src, const double* dUi,
                            int nf, const int* map, int j, int i, double dt, T* res)
{
    T Utmp[NVE];
    FV<T> Dt;
    calc_4vecs_t(B, Pt, j, i, Dt);
    prim_to_flux_t(B, ep, gam, Pt, Dt, j, i, 0, Utmp);
    for (int ip = 0; ip < nf; ++ip) res[ip] = (Utmp[map[ip]] - Ui[map[ip]]) / dt - src[map[ip]];
    if (ep.conduction || ep.viscosity) {
        T throwaway;
        T& rq = ep.conduction ? res[5] : throwaway;
        T& rdP = ep.viscosity ? res[ep.conduction ? 6 : 5] : throwaway;
        double tau, chi_e, nu_e;
        emhd_set_parameters_P(B, ep, gam, Ps, j, i, tau, chi_e, nu_e);
        FV<double> D;
        calc_4vecs_t(B, Ps, j, i, D);
        T dUq = T(0.), dUdP = T(0.);
        implicit_sources_t(B, ep, Pt, tau, j, i, dUq, dUdP);
        if (ep.conduction) rq -= 0.5*(dUq + dUi[IQ]);
        if (ep.viscosity) rdP -= 0.5*(dUdP + dUi[IDP]);
        emhd_set_parameters_P(B, ep, gam, Ps, j, i, tau, chi_e, nu_e);
        time_derivative_sources_t(B, ep, Pt, Pi, Ps, tau, chi_e, nu_e, D, gam, dt, j, i, dUq, dUdP);
        rq -= dUq;
        rdP -= dUdP;
        rq *= tau;
        rdP *= tau;
        if (ep.higher_order_terms) {
            const double rho = Ps[0], uu = Ps[1];
            const double Theta = (gam - 1.) * uu / rho;
            rq *= (chi_e != 0) ? std::sqrt(rho * chi_e * tau * Theta * Theta) / tau : 1.;
            rdP *= (nu_e != 0) ? std::sqrt(rho * nu_e * tau * Theta) / tau : 1.;
        }
    }
}
// Implicit sources of the full-step initial state, with tau from the sub-step state
// (implicit.cpp:294-305)
static void implicit_dU(const Block& B, const EmhdParams& ep, double gam, const double* Pfull, const double* Psub,
                        int j, int i, double* dUi)
{
    dUi[IQ] = 0.; dUi[IDP] = 0.;
    if (ep.conduction || ep.viscosity) {
        double tau, chi_e, nu_e;
        emhd_set_parameters_P(B, ep, gam, Psub, j, i, tau, chi_e, nu_e);
        implicit_sources_t(B, ep, Pfull, tau, j, i, dUi[IQ], dUi[IDP]);
    }
}
// Implicit::calc_jacobian, forward differences (implicit.hpp:208-255).  Ps_ is modified and restored.
static void calc_jacobian_fd(const Block& B, const EmhdParams& ep, double gam, double delta, double* Psol,
                             const double* Pi, const double* Ui, const double* Ps, const double* src,
                             const double* dUi, int nf, const int* map, int j, int i, double dt,
                             double* J, double* res)
{
    calc_residual_t<double>(B, ep, gam, Psol, Pi, Ui, Ps, src, dUi, nf, map, j, i, dt, res);
    double rsave[7], Psave[NVE];
    for (int ip = 0; ip < nf; ++ip) rsave[ip] = res[ip];
    for (int p = 0; p < NVE; ++p) Psave[p] = Psol[p];
    for (int col = 0; col < nf; ++col) {
        const int pc = map[col];
        if (std::fabs(Psave[pc]) < (0.5 * delta)) Psol[pc] = Psave[pc] + delta;
        else Psol[pc] = (1 + delta) * Psave[pc];
        calc_residual_t<double>(B, ep, gam, Psol, Pi, Ui, Ps, src, dUi, nf, map, j, i, dt, res);
        for (int row = 0; row < nf; ++row)
            J[row*nf + col] = (res[row] - rsave[row]) / (Psol[pc] - Psave[pc] + SMALL);
        Psol[pc] = Psave[pc];
    }
    for (int ip = 0; ip < nf; ++ip) res[ip] = rsave[ip];
}
// Exact Jacobian of the same residual (not in the reference, whose Jacobian is only by finite
// differences): forward mode over the nf implicit primitives.
static void calc_jacobian_exact(const Block& B, const EmhdParams& ep, double gam, const double* Psol,
                                const double* Pi, const double* Ui, const double* Ps, const double* src,
                                const double* dUi, int nf, const int* map, int j, int i, double dt,
                                double* J, double* res)
{
    Dual Pt[NVE], r[7];
    for (int p = 0; p < NVE; ++p) Pt[p] = Dual(Psol[p]);
    for (int col = 0; col < nf; ++col) Pt[map[col]].d[col] = 1.;
    calc_residual_t<Dual>(B, ep, gam, Pt, Pi, Ui, Ps, src, dUi, nf, map, j, i, dt, r);
    for (int row = 0; row < nf; ++row) {
        res[row] = r[row].v;
        for (int col = 0; col < nf; ++col) J[row*nf + col] = r[row].d[col];
    }
}
// Linear solve J x = b by Householder QR with column pivoting, then Q^T b, back substitution
// and the inverse permutation: KokkosBatched SerialQR (unblocked, with pivots), SerialApplyQ
// (left, transpose), SerialTrsv (upper, non-unit) and SerialApplyPivot (left, backward) as
// called at implicit.cpp:374-383 (external/kokkos-kernels, KokkosBatched_QR_Serial_Internal.hpp,
// _Householder_Serial_Internal.hpp, _ApplyHouseholder_Serial_Internal.hpp,
// _ApplyQ_Serial_Internal.hpp, _Trsv_Serial_Internal.hpp, _ApplyPivot_Internal.hpp,
// _FindAmax_Internal.hpp).  A is row-major n x n and is overwritten by the factorisation.
static void qr_solve(int n, double* A, double* b)
{
    double tau[7], norm[7], w[7];
    int piv[7];
    for (int c = 0; c < n; ++c) {
        norm[c] = 0.;
        for (int r = 0; r < n; ++r) norm[c] += A[r*n + c] * A[r*n + c];
    }
    for (int k = 0; k < n; ++k) {
        int p = 0;
        double mx = norm[k];
        for (int c = 1; c < n - k; ++c) if (norm[k + c] > mx) { mx = norm[k + c]; p = c; }
        piv[k] = p;
        if (p != 0) {
            std::swap(norm[k], norm[k + p]);
            for (int r = 0; r < n; ++r) std::swap(A[r*n + k], A[r*n + k + p]);
        }
        const int m2 = n - k - 1;
        double& chi1 = A[k*n + k];
        double nx2 = 0.;
        for (int r = 0; r < m2; ++r) { const double x = A[(k+1+r)*n + k]; nx2 += x * x; }
        if (nx2 == 0.) {
            chi1 = -chi1;
            tau[k] = 0.5;
        } else {
            const double nchi1 = std::fabs(chi1);
            const double nx = std::sqrt(nx2 + nchi1 * nchi1);
            const double alpha = (chi1 < 0 ? 1. : -1.) * nx;
            const double cma = chi1 - alpha;
            const double inv = 1. / cma;
            for (int r = 0; r < m2; ++r) A[(k+1+r)*n + k] *= inv;
            const double cma2 = cma * cma;
            tau[k] = 0.5 + 0.5 * (nx2 / cma2);
            chi1 = alpha;
        }
        const double inv_tau = 1. / tau[k];
        for (int c = 0; c < m2; ++c) {
            double t = A[k*n + k+1+c];
            for (int r = 0; r < m2; ++r) t += A[(k+1+r)*n + k] * A[(k+1+r)*n + k+1+c];
            w[c] = t * inv_tau;
        }
        for (int c = 0; c < m2; ++c) A[k*n + k+1+c] -= w[c];
        for (int c = 0; c < m2; ++c) for (int r = 0; r < m2; ++r) A[(k+1+r)*n + k+1+c] -= A[(k+1+r)*n + k] * w[c];
        for (int c = 0; c < m2; ++c) norm[k+1+c] -= A[k*n + k+1+c] * A[k*n + k+1+c];
    }
    for (int k = 0; k < n; ++k) {
        const int m2 = n - k - 1;
        const double inv_tau = 1. / tau[k];
        double t = b[k];
        for (int r = 0; r < m2; ++r) t += A[(k+1+r)*n + k] * b[k+1+r];
        const double wk = t * inv_tau;
        b[k] -= wk;
        for (int r = 0; r < m2; ++r) b[k+1+r] -= A[(k+1+r)*n + k] * wk;
    }
    for (int p = n - 1; p >= 0; --p) {
        b[p] = b[p] / A[p*n + p];
        for (int r = 0; r < p; ++r) b[r] -= A[r*n + p] * b[p];
    }
    for (int k = n - 1; k >= 0; --k) if (piv[k] != 0) std::swap(b[k], b[k + piv[k]]);
}
// The use_qr = false path: KokkosBatched SerialLU (no pivoting, diagonal nudged by tiny = SMALL)
// followed by the upper-triangular solve only, exactly as implicit.cpp:387-401 calls them.
static void lu_solve(int n, double* A, double* b)
{
    for (int p = 0; p < n; ++p) {
        const double a_real = A[p*n + p];
        A[p*n + p] += -SMALL * (double)(a_real < 0);
        A[p*n + p] += SMALL * (double)(a_real >= 0);
        const double a11 = A[p*n + p];
        for (int r = 0; r < n - p - 1; ++r) {
            A[(p+1+r)*n + p] /= a11;
            for (int c = 0; c < n - p - 1; ++c) A[(p+1+r)*n + p+1+c] -= A[(p+1+r)*n + p] * A[p*n + p+1+c];
        }
    }
    for (int p = n - 1; p >= 0; --p) {
        b[p] = b[p] / A[p*n + p];
        for (int r = 0; r < p; ++r) b[r] -= A[r*n + p] * b[p];
    }
}
static inline void load10(const double* A, size_t N, size_t c, double* out)
{
    for (int p = 0; p < NVE; ++p) out[p] = A[(size_t)p*N + c];
}
// One Newton iteration of Implicit::Step for one zone (implicit.cpp:286-522: the jacobian,
// solve and set-step kernels in sequence).  Psol is the zone's solver state, read and written.
static void implicit_zone_iteration(const Block& B, const EmhdParams& ep, const ImplicitParams& ip, double gam,
                                    const double* Pf, const double* Uf, const double* Ps, const double* S,
                                    double* Psol, double& solve_norm, double& solve_fail, double dt, int j, int i)
{
    int map[7];
    const int nf = implicit_map(ep, map);
    if (solve_fail == SOLVE_FAIL) return;
    solve_fail = SOLVE_CONVERGED;
    double dUi[NVE] = {0};
    implicit_dU(B, ep, gam, Pf, Ps, j, i, dUi);
    double J[49], res[7], delta[7];
    if (ip.jacobian == 1) calc_jacobian_exact(B, ep, gam, Psol, Pf, Uf, Ps, S, dUi, nf, map, j, i, dt, J, res);
    else calc_jacobian_fd(B, ep, gam, ip.jacobian_delta, Psol, Pf, Uf, Ps, S, dUi, nf, map, j, i, dt, J, res);
    for (int q = 0; q < nf; ++q) delta[q] = -res[q];
    if (ip.use_qr) qr_solve(nf, J, delta);
    else lu_solve(nf, J, delta);
    // implicit_set_step (implicit.cpp:426-521)
    double Pls[NVE];
    for (int p = 0; p < NVE; ++p) Pls[p] = Psol[p];
    double lambda = ip.linesearch_lambda;
    if ((Psol[0] + lambda*delta[0] < 0.) || (Psol[1] + lambda*delta[1] < 0.)) {
        solve_fail = SOLVE_BACKTRACK;
        lambda = 0.1;
    }
    if ((Psol[0] + lambda*delta[0] < 0.) || (Psol[1] + lambda*delta[1] < 0.)) {
        solve_fail = SOLVE_FAIL;
        for (int q = 0; q < nf; ++q) Psol[map[q]] = Ps[map[q]];
        return;
    }
    if (ip.linesearch) {
        solve_norm = 0.;
        for (int q = 0; q < nf; ++q) solve_norm += res[q]*res[q];
        solve_norm = std::sqrt(solve_norm);
        const double f0 = 0.5 * solve_norm;
        const double fprime0 = -2. * f0;
        for (int it = 0; it < ip.max_linesearch_iter; it++) {
            for (int q = 0; q < nf; ++q) Pls[map[q]] = Psol[map[q]] + (lambda * delta[q]);
            calc_residual_t<double>(B, ep, gam, Pls, Pf, Uf, Ps, S, dUi, nf, map, j, i, dt, res);
            solve_norm = 0.;
            for (int q = 0; q < nf; ++q) solve_norm += res[q]*res[q];
            solve_norm = std::sqrt(solve_norm);
            const double f1 = 0.5 * solve_norm;
            const int condition = f1 > (f0 * (1. - ip.linesearch_eps * lambda) + SMALL);
            const double denom = (f1 - f0 - (fprime0 * lambda)) * condition + (1 - condition);
            const double lambda_new = -fprime0 * lambda * lambda / denom * 0.5;
            lambda = lambda * (1 - condition) + (condition * lambda_new);
            if (condition == 0) break;
        }
    }
    for (int q = 0; q < nf; ++q) Psol[map[q]] += lambda * delta[q];
    calc_residual_t<double>(B, ep, gam, Psol, Pf, Uf, Ps, S, dUi, nf, map, j, i, dt, res);
    solve_norm = 0;
    for (int q = 0; q < nf; ++q) solve_norm += res[q]*res[q];
    solve_norm = std::sqrt(solve_norm);
    if (std::isnan(solve_norm)) {
        solve_fail = SOLVE_FAIL;
        for (int q = 0; q < nf; ++q) Psol[map[q]] = Ps[map[q]];
    } else if (solve_norm > ip.rootfind_tol) {
        solve_fail = SOLVE_BEYOND_TOL;
    }
}
// Implicit::Step over the block interior (implicit.cpp:159-571).  Arrays are [10][N].  Returns
// the number of Newton iterations taken; maxnorm[iter-1] receives each iteration's maximum
// solve_norm (the reduction of implicit.cpp:527-534; NaN norms are skipped as Kokkos::Max does).
static int implicit_step(const Block& B, const EmhdParams& ep, const ImplicitParams& ip, double gam,
                         const double* Pf, const double* Uf, const double* Ps, const double* S, double* Psol,
                         double* solve_norm, double* solve_fail, double dt, double* maxnorm)
{
    const size_t N = B.N;
    int iters = 0;
    for (int iter = 1; iter <= ip.max_nonlinear_iter; ++iter) {
        iters = iter;
#pragma omp parallel for collapse(2) schedule(static)
        for (int k = B.ks; k <= B.ke; ++k) for (int j = B.js; j <= B.je; ++j) for (int i = B.is; i <= B.ie; ++i) {
            const size_t c = B.id(k, j, i);
            double pf[NVE], uf[NVE], ps[NVE], s[NVE], psol[NVE];
            load10(Pf, N, c, pf); load10(Uf, N, c, uf); load10(Ps, N, c, ps); load10(S, N, c, s);
            load10(Psol, N, c, psol);
            implicit_zone_iteration(B, ep, ip, gam, pf, uf, ps, s, psol, solve_norm[c], solve_fail[c], dt, j, i);
            for (int p = 0; p < NVE; ++p) Psol[(size_t)p*N + c] = psol[p];
        }
        double m = -std::numeric_limits<double>::max();
        for (int k = B.ks; k <= B.ke; ++k) for (int j = B.js; j <= B.je; ++j) for (int i = B.is; i <= B.ie; ++i) {
            const double v = solve_norm[B.id(k, j, i)];
            if (v > m) m = v;
        }
        if (maxnorm) maxnorm[iter - 1] = m;
        if (iter >= ip.min_nonlinear_iter && m < ip.rootfind_tol) break;
    }
    return iters;
}
// Implicit::FixSolve (fix_solve.cpp:44-130) over the entire block.  Neighbours are read from the
// state before this pass (the reference reads them while other failed zones are being replaced).
static void fix_solve(const Block& B, const EmhdParams& ep, double gam, double* P, double* U, const double* solve_fail)
{
    int map[7];
    const int nf = implicit_map(ep, map);
    const size_t N = B.N;
    std::vector<double> P0(P, P + (size_t)NVE*N);
    auto failed = [](double s) { return (int)s == SOLVE_FAIL; };
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < B.n3; ++k) for (int j = 0; j < B.n2; ++j) for (int i = 0; i < B.n1; ++i) {
        const size_t c = B.id(k, j, i);
        if (!failed(solve_fail[c])) continue;
        double wsum = 0., wsum_x = 0., sum[7] = {0.}, sum_x[7] = {0.};
        for (int n = -1; n <= 1; n++) for (int m = -1; m <= 1; m++) for (int l = -1; l <= 1; l++) {
            const int ii = i + l, jj = j + m, kk = k + n;
            if (ii < 0 || ii >= B.n1 || jj < 0 || jj >= B.n2 || kk < 0 || kk >= B.n3) continue;
            const double w = 1./(std::abs(l) + std::abs(m) + std::abs(n) + 1);
            const size_t cn = B.id(kk, jj, ii);
            if (!failed(solve_fail[cn])) {
                wsum += w;
                for (int q = 0; q < nf; ++q) sum[q] += w * P0[(size_t)map[q]*N + cn];
            }
            wsum_x += w;
            for (int q = 0; q < nf; ++q) sum_x[q] += w * P0[(size_t)map[q]*N + cn];
        }
        if (wsum < 1.e-10) { for (int q = 0; q < nf; ++q) P[(size_t)map[q]*N + c] = sum_x[q]/wsum_x; }
        else               { for (int q = 0; q < nf; ++q) P[(size_t)map[q]*N + c] = sum[q]/wsum; }
    }
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < B.n3; ++k) for (int j = 0; j < B.n2; ++j) for (int i = 0; i < B.n1; ++i) {
        const size_t c = B.id(k, j, i);
        if (!failed(solve_fail[c])) continue;
        double Pc[NVE], Uc[NVE];
        load10(P, N, c, Pc);
        FV<double> D;
        calc_4vecs_t(B, Pc, j, i, D);
        prim_to_flux_t(B, ep, gam, Pc, D, j, i, 0, Uc);
        for (int p = 0; p < NVE; ++p)
            if (p < 8 || (p == IQ && ep.conduction) || (p == IDP && ep.viscosity)) U[(size_t)p*N + c] = Uc[p];
    }
}
// Flux::p_to_u for the 10-slot state over the entire block (flux_functions.hpp:343-352)
static void emhd_ptou(const Block& B, const EmhdParams& ep, double gam, const double* P, double* U)
{
    const size_t N = B.N;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 0; k < B.n3; ++k) for (int j = 0; j < B.n2; ++j) for (int i = 0; i < B.n1; ++i) {
        const size_t c = B.id(k, j, i);
        double Pc[NVE], Uc[NVE];
        load10(P, N, c, Pc);
        FV<double> D;
        calc_4vecs_t(B, Pc, j, i, D);
        prim_to_flux_t(B, ep, gam, Pc, D, j, i, 0, Uc);
        for (int p = 0; p < NVE; ++p)
            if (p < 8 || (p == IQ && ep.conduction) || (p == IDP && ep.viscosity)) U[(size_t)p*N + c] = Uc[p];
    }
}
// KReconstruction::slope_limit<linear_mc> (reconstruction.hpp:781-798)
static inline double slope_mc(double x1, double x2, double x3, double dx)
{
    const double Dqm = 2 * (x2 - x1) / dx;
    const double Dqp = 2 * (x3 - x2) / dx;
    const double Dqc = 0.5 * (x3 - x1) / dx;
    if (Dqm * Dqp <= 0) return 0;
    if ((std::fabs(Dqm) < std::fabs(Dqp)) && (std::fabs(Dqm) < std::fabs(Dqc))) return Dqm;
    else if (std::fabs(Dqp) < std::fabs(Dqc)) return Dqp;
    return Dqc;
}
// EMHD::AddSource: explicit conduction and viscosity sources added to dUdt over the interior
// (emhd.cpp:288-397, gradients by EMHD::gradient_calc<linear_mc>, emhd_utils.hpp:55-79)
static void emhd_add_source(const Block& B, const EmhdParams& ep, double gam, const double* P, double* dUdt)
{
    if (!(ep.conduction || ep.viscosity)) return;
    const size_t N = B.N;
    // temporaries ucov and Theta over the interior plus a one-zone halo in active directions
    std::vector<double> Tmp((size_t)5*N, 0.);
    const int il = B.is - 1, ih = B.ie + 1;
    const int jl = (B.ndim > 1) ? B.js - 1 : B.js, jh = (B.ndim > 1) ? B.je + 1 : B.je;
    const int kl = (B.ndim > 2) ? B.ks - 1 : B.ks, kh = (B.ndim > 2) ? B.ke + 1 : B.ke;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = kl; k <= kh; ++k) for (int j = jl; j <= jh; ++j) for (int i = il; i <= ih; ++i) {
        const size_t c = B.id(k, j, i);
        double Pc[NVE], ucon[4], ucov[4];
        load10(P, N, c, Pc);
        calc_ucon_t(B, Pc, j, i, ucon);
        lower_t(B, ucon, ucov, j, i);
        for (int mu = 0; mu < 4; ++mu) Tmp[(size_t)mu*N + c] = ucov[mu];
        Tmp[4*N + c] = kmax((gam - 1) * Pc[1] / Pc[0], SMALL);
    }
    const size_t sj = B.n1, sk = (size_t)B.n1*B.n2;
    const bool do_2d = B.ndim > 1, do_3d = B.ndim > 2;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = B.ks; k <= B.ke; ++k) for (int j = B.js; j <= B.je; ++j) for (int i = B.is; i <= B.ie; ++i) {
        const size_t c = B.id(k, j, i);
        double Pc[NVE];
        load10(P, N, c, Pc);
        double tau, chi_e, nu_e;
        emhd_set_parameters_P(B, ep, gam, Pc, j, i, tau, chi_e, nu_e);
        FV<double> D;
        calc_4vecs_t(B, Pc, j, i, D);
        const double bsq = kmax(tdot(D.bcon, D.bcov), SMALL);
        auto slope = [&](int var, int dir) {
            const double* T = &Tmp[(size_t)var*N];
            if (dir == 1) return slope_mc(T[c - 1], T[c], T[c + 1], B.c.dx1);
            if (dir == 2) return slope_mc(T[c - sj], T[c], T[c + sj], B.c.dx2);
            return slope_mc(T[c - sk], T[c], T[c + sk], B.c.dx3);
        };
        double grad_ucov[4][4], grad_Theta[4];
        for (int mu = 0; mu < 4; ++mu) {
            grad_ucov[0][mu] = 0;
            grad_ucov[1][mu] = slope(mu, 1);
            grad_ucov[2][mu] = do_2d ? slope(mu, 2) : 0.;
            grad_ucov[3][mu] = do_3d ? slope(mu, 3) : 0.;
        }
        const size_t cg = ((size_t)j*B.n1 + i)*64;
        for (int mu = 0; mu < 4; ++mu) for (int nu = 0; nu < 4; ++nu) for (int lam = 0; lam < 4; ++lam)
            grad_ucov[mu][nu] -= B.conn[cg + lam*16 + mu*4 + nu] * Tmp[(size_t)lam*N + c];
        grad_Theta[0] = 0;
        grad_Theta[1] = slope(4, 1);
        grad_Theta[2] = do_2d ? slope(4, 2) : 0.;
        grad_Theta[3] = do_3d ? slope(4, 3) : 0.;
        double div_ucon = 0;
        for (int mu = 0; mu < 4; ++mu) for (int nu = 0; nu < 4; ++nu)
            div_ucon += B.Gcon(center, j, i, mu, nu) * grad_ucov[mu][nu];
        const double rho = Pc[0];
        const double Theta = Tmp[4*N + c];
        const double gdet = B.Gdet(center, j, i);
        if (ep.conduction) {
            const double qtilde = Pc[IQ];
            const double inv_mag_b = 1. / std::sqrt(bsq);
            double q0 = 0;
            for (int mu = 0; mu < 4; ++mu) q0 -= rho * chi_e * (D.bcon[mu] * inv_mag_b) * grad_Theta[mu];
            for (int mu = 0; mu < 4; ++mu) for (int nu = 0; nu < 4; ++nu)
                q0 -= rho * chi_e * (D.bcon[mu] * inv_mag_b) * Theta * D.ucon[nu] * grad_ucov[nu][mu];
            double q0_tilde = q0;
            if (ep.higher_order_terms)
                q0_tilde *= (chi_e != 0) ? std::sqrt(tau / (chi_e * rho * Theta * Theta)) : 0.0;
            dUdt[(size_t)IQ*N + c] += gdet * q0_tilde / tau;
            if (ep.higher_order_terms) dUdt[(size_t)IQ*N + c] += gdet * (qtilde / 2.) * div_ucon;
        }
        if (ep.viscosity) {
            const double dPtilde = Pc[IDP];
            double dP0 = -rho * nu_e * div_ucon;
            for (int mu = 0; mu < 4; ++mu) for (int nu = 0; nu < 4; ++nu)
                dP0 += 3. * rho * nu_e * (D.bcon[mu] * D.bcon[nu] / bsq) * grad_ucov[mu][nu];
            double dP0_tilde = dP0;
            if (ep.higher_order_terms)
                dP0_tilde *= (nu_e != 0) ? std::sqrt(tau / (nu_e * rho * Theta)) : 0.0;
            dUdt[(size_t)IDP*N + c] += gdet * dP0_tilde / tau;
            if (ep.higher_order_terms) dUdt[(size_t)IDP*N + c] += gdet * (dPtilde / 2.) * div_ucon;
        }
    }
}

// ---------------------------------------------------------------- EMHD explicit path and ImEx stage
// The explicit part of the EMHD step: Flux::GetFlux with the EMHD variables present (get_flux.hpp
// with prim_to_flux at the faces, flux_functions.hpp:180-232, and vchar's EMHD signal speeds,
// :368-439), flux-CT, the divergence of every variable, Flux::AddGeoSource with the EMHD stress
// tensor (flux.cpp:395-444 through Flux::calc_tensor, :80-107) and EMHD::AddSource; then the ImEx
// stage of imex_step.cpp:58-356 with the vl2 integrator the implicit package forces
// (implicit.cpp:96): explicit update of B only, B_P = B_U/gdet, the implicit guess copied from the
// sub-step state, Implicit::Step with beta dt, FixSolve, ghost zones, P -> U.
static const double VL2_GAM0[2] = {0.0, 0.0}, VL2_GAM1[2] = {1.0, 1.0}, VL2_BETA[2] = {0.5, 1.0};

static inline FV<double> to_fv(const FourVectors& D)
{
    FV<double> F;
    for (int mu = 0; mu < 4; ++mu) { F.ucon[mu] = D.ucon[mu]; F.ucov[mu] = D.ucov[mu]; F.bcon[mu] = D.bcon[mu]; F.bcov[mu] = D.bcov[mu]; }
    return F;
}
static inline bool emhd_active(const EmhdParams& ep, int p) { return p < 8 || (p == IQ && ep.conduction) || (p == IDP && ep.viscosity); }

// Flux::prim_to_flux at a face location for the 10-slot state
static void emhd_prim_to_flux_loc(const Block& B, const EmhdParams& ep, const double* P, const FourVectors& Dv,
                                  int j, int i, int loc, int dir, double* flux)
{
    const double gam = B.c.gam, gdet = B.Gdet(loc, j, i);
    const FV<double> D = to_fv(Dv);
    flux[0] = P[0] * D.ucon[dir] * gdet;
    double Tm[4];
    calc_tensor_t(ep, gam, P, D, dir, Tm);
    flux[1] = Tm[0] * gdet + flux[0];
    flux[2] = Tm[1] * gdet;
    flux[3] = Tm[2] * gdet;
    flux[4] = Tm[3] * gdet;
    if (dir == 0) {
        for (int v = 0; v < 3; ++v) flux[5 + v] = P[5 + v] * gdet;
    } else {
        for (int v = 0; v < 3; ++v) flux[5 + v] = (D.bcon[v+1] * D.ucon[dir] - D.bcon[dir] * D.ucon[v+1]) * gdet;
    }
    flux[IQ] = ep.conduction ? P[IQ] * D.ucon[dir] * gdet : 0.;
    flux[IDP] = ep.viscosity ? P[IDP] * D.ucon[dir] * gdet : 0.;
}
// vchar with the EMHD-augmented sound speed (flux_functions.hpp:380-403)
static void emhd_vchar(const Block& B, const EmhdParams& ep, const double* P, const FourVectors& D, int j, int i,
                       int loc, int dir, double& cmax, double& cmin)
{
    const double gam = B.c.gam;
    const double ef  = P[0] + gam * P[1];
    const double cs2 = gam * (gam - 1) * P[1] / ef;
    const double bsq = dot4(D.bcon, D.bcov);
    const double va2 = bsq / (bsq + ef);
    const double ccond2 = ep.conduction ? (gam - 1.) * ep.conduction_alpha * cs2 : 0.0;
    const double cvis2 = ep.viscosity ? (4./3.) / (P[0] + (gam * P[1])) * P[0] * ep.viscosity_alpha * cs2 : 0.0;
    const double cs2_emhd = 0.5*(cs2 + ccond2 + std::sqrt(cs2*cs2 + ccond2*ccond2)) + cvis2;
    const double cms2 = cs2_emhd + va2 - cs2_emhd*va2;
    double Bcov[4] = {1., 0., 0., 0.};
    double Acov[4] = {0., 0., 0., 0.}; Acov[dir] = 1.;
    double Acon[4], Bcon[4];
    B.raise(Acov, Acon, j, i, loc);
    B.raise(Bcov, Bcon, j, i, loc);
    const double Asq = dot4(Acon, Acov);
    const double Bsq = dot4(Bcon, Bcov);
    const double Au  = dot4(Acov, D.ucon);
    const double Bu  = dot4(Bcov, D.ucon);
    const double AB  = dot4(Acon, Bcov);
    const double A  = Bu*Bu - (Bsq + Bu*Bu) * cms2;
    const double Bq = 2. * (Au*Bu - (AB + Au*Bu) * cms2);
    const double Cq = Au*Au - (Asq + Au*Au) * cms2;
    const double discr = std::sqrt(kmax(Bq * Bq - 4. * A * Cq, 0.));
    const double vp = -(-Bq + discr) / (2. * A);
    const double vm = -(-Bq - discr) / (2. * A);
    cmax = kmax(vp, vm);
    cmin = kmin(vp, vm);
}
// Face fluxes of the 10-slot state along dir (same face ranges and cmin sign as get_flux)
static void get_flux_emhd(const Block& B, const EmhdParams& ep, int dir, const double* P, double* F,
                          double* cmaxo, double* cmino)
{
    const int loc = dir - 1;
    const int d1 = (dir == 1), d2 = (dir == 2), d3 = (dir == 3);
    const int i0 = B.is - (!d1 ? 1 : 0), i1 = B.ie + 1;
    const int j0 = (B.ndim >= 2) ? B.js - (d2 ? 0 : 1) : B.js, j1 = (B.ndim >= 2) ? B.je + 1 : B.je;
    const int k0 = (B.ndim >= 3) ? B.ks - (d3 ? 0 : 1) : B.ks, k1 = (B.ndim >= 3) ? B.ke + 1 : B.ke;
    const ptrdiff_t st = d1 + (d2 ? B.n1 : 0) + (d3 ? (ptrdiff_t)B.n1*B.n2 : 0);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = k0; k <= k1; ++k) for (int j = j0; j <= j1; ++j) for (int i = i0; i <= i1; ++i) {
        const size_t c = B.id(k, j, i);
        double Pl[NVE] = {0.}, Pr[NVE] = {0.};
        for (int p = 0; p < NVE; ++p) {
            if (!emhd_active(ep, p)) continue;
            const double* q = P + (size_t)p*B.N;
            double l, r;
            recon_zone(B.c.recon, q[c - 3*st], q[c - 2*st], q[c - st], q[c], q[c + st], l, r);
            Pl[p] = r;
            recon_zone(B.c.recon, q[c - 2*st], q[c - st], q[c], q[c + st], q[c + 2*st], l, r);
            Pr[p] = l;
        }
        FourVectors Dl, Dr;
        double Ul[NVE], Fl[NVE], Ur[NVE], Fr[NVE], cmaxL, cminL, cmaxR, cminR;
        calc_4vecs(B, Pl, true, j, i, loc, Dl);
        emhd_prim_to_flux_loc(B, ep, Pl, Dl, j, i, loc, 0, Ul);
        emhd_prim_to_flux_loc(B, ep, Pl, Dl, j, i, loc, dir, Fl);
        emhd_vchar(B, ep, Pl, Dl, j, i, loc, dir, cmaxL, cminL);
        calc_4vecs(B, Pr, true, j, i, loc, Dr);
        emhd_prim_to_flux_loc(B, ep, Pr, Dr, j, i, loc, 0, Ur);
        emhd_prim_to_flux_loc(B, ep, Pr, Dr, j, i, loc, dir, Fr);
        emhd_vchar(B, ep, Pr, Dr, j, i, loc, dir, cmaxR, cminR);
        const double cmax = kmax(kmax(0., cmaxL), cmaxR);
        const double cmin = -kmin(kmin(0., cminL), cminR);
        cmaxo[c] = cmax; cmino[c] = cmin;
        for (int p = 0; p < NVE; ++p)
            F[(size_t)p*B.N + c] = !emhd_active(ep, p) ? 0.
                                 : (B.c.riemann ? hlle(Fl[p], Fr[p], cmax, cmin, Ul[p], Ur[p])
                                                : llf(Fl[p], Fr[p], cmax, cmin, Ul[p], Ur[p]));
    }
}
// FluxDivergence of every active variable, then AddGeoSource with the EMHD tensor and EMHD::AddSource
static void emhd_dudt(const Block& B, const EmhdParams& ep, double* F[3], const double* P, double* dudt)
{
    const size_t N = B.N;
    const double a1 = B.c.dx2*B.c.dx3, a2 = B.c.dx1*B.c.dx3, a3 = B.c.dx1*B.c.dx2;
    const double vol = B.c.dx1*B.c.dx2*B.c.dx3;
    const size_t sj = B.n1, sk = (size_t)B.n1*B.n2;
    const double gam = B.c.gam;
    std::fill(dudt, dudt + (size_t)NVE*N, 0.);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = B.ks; k <= B.ke; ++k) for (int j = B.js; j <= B.je; ++j) for (int i = B.is; i <= B.ie; ++i) {
        const size_t c = B.id(k, j, i);
        for (int p = 0; p < NVE; ++p) {
            if (!emhd_active(ep, p)) continue;
            const size_t pc = (size_t)p*N + c;
            double du = (a1 * F[0][pc + 1] - a1 * F[0][pc]);
            if (B.ndim >= 2) du += a2 * F[1][pc + sj] - a2 * F[1][pc];
            if (B.ndim == 3) du += a3 * F[2][pc + sk] - a3 * F[2][pc];
            dudt[pc] = -du / vol;
        }
        if (!B.C.cart_minkowski()) {
            double Pc[NVE];
            load10(P, N, c, Pc);
            FourVectors Dv;
            calc_4vecs(B, Pc, true, j, i, center, Dv);
            const FV<double> D = to_fv(Dv);
            double Tmu[4] = {0}, new_du[4] = {0};
            for (int mu = 0; mu < 4; ++mu) {
                calc_tensor_t(ep, gam, Pc, D, mu, Tmu);
                for (int nu = 0; nu < 4; ++nu)
                    for (int lam = 0; lam < 4; ++lam)
                        new_du[lam] += Tmu[nu] * B.GdetConn(j, i, nu, lam, mu);
            }
            dudt[1*N + c] += new_du[0];
            for (int v = 0; v < 3; ++v) dudt[(size_t)(2 + v)*N + c] += new_du[1 + v];
        }
    }
    emhd_add_source(B, ep, gam, P, dudt);
}
// Minimum zone timestep from the signal speeds (grmhd.cpp:294-339)
static double min_ndt_from(const Block& B, const std::vector<double> cmax[3], const std::vector<double> cmin[3])
{
    double m = std::numeric_limits<double>::max();
    for (int k = B.ks; k <= B.ke; ++k) for (int j = B.js; j <= B.je; ++j) for (int i = B.is; i <= B.ie; ++i) {
        const size_t c = B.id(k, j, i);
        const double ndt_zone = 1.0 / (1 / (B.c.dx1 / kmax(cmax[0][c], cmin[0][c])) +
                                       1 / (B.c.dx2 / kmax(cmax[1][c], cmin[1][c])) +
                                       1 / (B.c.dx3 * 1 / kmax(cmax[2][c], cmin[2][c])));
        if (!std::isnan(ndt_zone) && (ndt_zone < m)) m = ndt_zone;
    }
    return m;
}
// EMHD::ApplyEMHDLimits / apply_instability_limits (emhd.cpp:399-428, emhd_limits.hpp:55-130) over
// the interior: the heat flux limited to 1.07 rho cs^3 and the pressure anisotropy to the mirror and
// firehose bounds, by scaling q~ and dP~; returns the eflag bits per zone in eflag (HIT_Q_LIMIT 1,
// HIT_DP_MAX_LIMIT 2, HIT_DP_MIN_LIMIT 4).  The reference's closing p_to_u is covered by the stage's
// final P -> U over the whole block.
static void emhd_limits(const Block& B, const EmhdParams& ep, double gam, double* P, double* eflag)
{
    const size_t N = B.N;
    for (int k = B.ks; k <= B.ke; ++k) for (int j = B.js; j <= B.je; ++j) for (int i = B.is; i <= B.ie; ++i) {
        const size_t c = B.id(k, j, i);
        double Pc[NVE];
        for (int v = 0; v < NVE; ++v) Pc[v] = P[(size_t)v*N + c];
        int ef = 0;
        const double rho = Pc[0], uu = Pc[1];
        const double qtilde = ep.conduction ? Pc[IQ] : 0., dPtilde = ep.viscosity ? Pc[IDP] : 0.;
        const double pg = (gam - 1.) * uu;
        const double Theta = pg / rho;
        const double cs = std::sqrt(gam * pg / (rho + (gam * uu)));
        FV<double> D;
        calc_4vecs_t(B, Pc, j, i, D);
        const double bsq = kmax(tdot(D.bcon, D.bcov), SMALL);
        // (the reference also evaluates the closure here; nothing below uses it)
        double q, dP;
        convert_prims_to_q_dP_t(qtilde, dPtilde, rho, Theta, cs*cs, ep, q, dP);
        if (ep.conduction) {
            const double qmax = 1.07 * rho * cs*cs*cs;
            const double max_frac = kmax(std::fabs(q) / qmax, 1.);
            if (std::fabs(q) / qmax > 1.) ef |= 1;
            P[(size_t)IQ*N + c] = Pc[IQ] / max_frac;
        }
        if (ep.viscosity) {
            const double dP_comp_ratio = kmax(pg - 2./3. * dP, SMALL) / kmax(pg + 1./3. * dP, SMALL);
            const double dP_plus = kmin(1.07 * 0.5 * bsq * dP_comp_ratio, 1.49 * pg);
            const double dP_minus = kmax(-1.07 * bsq, -2.99 * pg);
            if (dP > 0. && (dP / dP_plus > 1.)) ef |= 2;
            else if (dP < 0. && (dP / dP_minus > 1.)) ef |= 4;
            if (dP > 0.) P[(size_t)IDP*N + c] = Pc[IDP] * (1. / kmax(dP / dP_plus, 1.));
            else P[(size_t)IDP*N + c] = Pc[IDP] * (1. / kmax(dP / dP_minus, 1.));
        }
        if (eflag) eflag[c] = ef;
    }
}

static bool has_physical_face(const Block& B)
{
    for (int face = 0; face < 2*B.ndim; ++face) if (phys_face(B.c.bc[face])) return true;
    return false;
}

// One ImEx stage (s = 0, 1).  All arrays [10][N]; ghost zones of Pout/Uout start as copies of the
// sub-step state (the guess copy); periodic and physical faces are filled, exchange faces are the
// caller's.  fflag / eflag (optional, [N]): the floor and EMHD-limit bits of the interior zones.
// Returns the Newton iterations; *min_ndt from this stage's fluxes.
static int imex_stage(const Block& B, const EmhdParams& ep, const ImplicitParams& ip, int s, double dt,
                      const double* Pfull, const double* Ufull, const double* Psub, const double* Usub,
                      double* Pout, double* Uout, double* solve_norm, double* solve_fail, double* min_ndt_out,
                      double* fflag = nullptr, double* eflag = nullptr)
{
    const size_t N = B.N, NA = (size_t)NVE*N;
    const double gam = B.c.gam;
    std::vector<double> Fv[3], cmx[3], cmn[3];
    double* F[3];
    for (int d = 0; d < 3; ++d) {
        Fv[d].assign(NA, 0.); cmx[d].assign(N, 0.); cmn[d].assign(N, 0.);
        F[d] = Fv[d].data();
    }
    for (int d = 1; d <= B.ndim; ++d) get_flux_emhd(B, ep, d, Psub, F[d-1], cmx[d-1].data(), cmn[d-1].data());
    if (B.c.fix_polar_flux && B.C.spherical()) {
        if (phys_face(B.c.bc[2])) zero_boundary_flux_x2(B, F[0], F[1], F[2], true);
        if (phys_face(B.c.bc[3])) zero_boundary_flux_x2(B, F[0], F[1], F[2], false);
    }
    flux_ct(B, F[0], F[1], F[2]);
    // KBoundaries::FixFlux on the physical faces: inflow checks on X1, zero polar fluxes of every
    // variable, q~ and dP~ included (boundaries.cpp:611-690)
    boundaries_fix_flux(B, F, NVE);
    std::vector<double> dudt(NA, 0.);
    emhd_dudt(B, ep, F, Psub, dudt.data());
    // solver state: the sub-step state everywhere; explicit update of B over the interior
    std::vector<double> Psol(Psub, Psub + NA), Usol(Usub, Usub + NA);
    const double g0 = VL2_GAM0[s], g1 = VL2_GAM1[s], bdt = VL2_BETA[s] * dt;
    for (int v = 5; v < 8; ++v)
        for (int k = B.ks; k <= B.ke; ++k) for (int j = B.js; j <= B.je; ++j) for (int i = B.is; i <= B.ie; ++i) {
            const size_t x = (size_t)v*N + B.id(k, j, i);
            Usol[x] = g0 * Usub[x] + g1 * Ufull[x];
            Usol[x] = 1.0 * Usol[x] + bdt * dudt[x];
        }
    // B_FluxCT::BlockUtoP over the entire block (b_flux_ct.cpp:172-217)
    for (int v = 5; v < 8; ++v)
        for (int k = 0; k < B.n3; ++k) for (int j = 0; j < B.n2; ++j) for (int i = 0; i < B.n1; ++i) {
            const size_t c = B.id(k, j, i);
            Psol[(size_t)v*N + c] = Usol[(size_t)v*N + c] / B.Gdet(center, j, i);
        }
    const int iters = implicit_step(B, ep, ip, gam, Pfull, Ufull, Psub, dudt.data(), Psol.data(), solve_norm,
                                    solve_fail, bdt, nullptr);
    std::memcpy(Pout, Psol.data(), NA*sizeof(double));
    std::memcpy(Uout, Usol.data(), NA*sizeof(double));
    // Packages::MeshApplyFloors over the interior (imex_step.cpp:269): the GRMHD floors (fluid and
    // drift frames change P only; the U they form is replaced by the stage's final P -> U), then the
    // EMHD package's stability limits
    if (fflag) for (size_t x = 0; x < N; ++x) fflag[x] = 0.;
    if (eflag) for (size_t x = 0; x < N; ++x) eflag[x] = 0.;
    if (B.c.floors_on) {
        std::vector<double> pflag_tmp(N, 0.), fflag_tmp(N, 0.);
        apply_grmhd_floors(B, Pout, Uout, pflag_tmp.data(), fflag ? fflag : fflag_tmp.data(),
                           B.ks, B.ke, B.js, B.je, B.is, B.ie);
    }
    if (ep.stability_limits) emhd_limits(B, ep, gam, Pout, eflag);
    fix_solve(B, ep, gam, Pout, Uout, solve_fail);
    // ApplyBoundaryConditionsOnCoarseOrFineMD (imex_step.cpp:297-298): periodic images and the physical
    // faces of the 10-slot state, B_P from U_B in the ghost zones
    if (has_physical_face(B)) {
        apply_boundaries(B, Pout, Uout, true);
    } else {
        for (int d = 1; d <= B.ndim; ++d)
            if (B.c.bc[2*(d-1)] == BC_PERIODIC) { periodic_fill(B, Pout, NVE, d); periodic_fill(B, Uout, NVE, d); }
    }
    emhd_ptou(B, ep, gam, Pout, Uout);
    if (min_ndt_out) *min_ndt_out = min_ndt_from(B, cmx, cmn);
    return iters;
}

struct Handle {
    Block B;
    Fields f;
    std::vector<double> P1, U1, U0;
};

} // namespace orc

// ======================================================================== C ABI (for the tests)
using namespace orc;
extern "C" {

void* orc_create(const Config* cfg, const CoordSpec* cs)
{
    Handle* h = new Handle();
    h->B.init(*cfg, *cs);
    h->B.build_geometry();
    h->f.alloc(h->B);
    return h;
}
void orc_destroy(void* hp) { delete (Handle*)hp; }

// OpenMP threads of the following parallel regions (the CPU baseline's one-thread run); returns the
// previous maximum
int orc_set_threads(int n)
{
    const int prev = omp_get_max_threads();
    if (n > 0) omp_set_num_threads(n);
    return prev;
}

void orc_get_dims(void* hp, int32_t* dims)
{
    const Block& B = ((Handle*)hp)->B;
    dims[0] = B.n1; dims[1] = B.n2; dims[2] = B.n3; dims[3] = B.ndim;
    dims[4] = B.is; dims[5] = B.ie; dims[6] = B.js; dims[7] = B.je; dims[8] = B.ks; dims[9] = B.ke;
}

// Copy the geometry caches out (GRCoordinates layout) or replace them with caller tables.
void orc_get_geometry(void* hp, double* gcov, double* gcon, double* gdet, double* gdet_conn, double* rcen)
{
    const Block& B = ((Handle*)hp)->B;
    if (gcov) std::memcpy(gcov, B.gcov.data(), B.gcov.size()*sizeof(double));
    if (gcon) std::memcpy(gcon, B.gcon.data(), B.gcon.size()*sizeof(double));
    if (gdet) std::memcpy(gdet, B.gdet.data(), B.gdet.size()*sizeof(double));
    if (gdet_conn) std::memcpy(gdet_conn, B.gdet_conn.data(), B.gdet_conn.size()*sizeof(double));
    if (rcen) std::memcpy(rcen, B.rcen.data(), B.rcen.size()*sizeof(double));
}
void orc_set_geometry(void* hp, const double* gcov, const double* gcon, const double* gdet,
                      const double* gdet_conn, const double* rcen)
{
    Block& B = ((Handle*)hp)->B;
    if (gcov) std::memcpy(B.gcov.data(), gcov, B.gcov.size()*sizeof(double));
    if (gcon) std::memcpy(B.gcon.data(), gcon, B.gcon.size()*sizeof(double));
    if (gdet) std::memcpy(B.gdet.data(), gdet, B.gdet.size()*sizeof(double));
    if (gdet_conn) std::memcpy(B.gdet_conn.data(), gdet_conn, B.gdet_conn.size()*sizeof(double));
    if (rcen) std::memcpy(B.rcen.data(), rcen, B.rcen.size()*sizeof(double));
}

// Flux::GetFlux<recon, dir> on the consumer range; F is [nvar][cells]
void orc_get_flux(void* hp, int dir, const double* P, double* F, double* cmax, double* cmin)
{
    Handle* h = (Handle*)hp;
    get_flux(h->B, dir, P, F, cmax, cmin);
}

// B_FluxCT::FixFlux + KBoundaries::FixFlux on raw fluxes (in place)
void orc_fix_flux(void* hp, double* F1, double* F2, double* F3)
{
    Handle* h = (Handle*)hp;
    const Block& B = h->B;
    double* F[3] = {F1, F2, F3};
    if (B.nv > 5) {
        if (B.c.fix_polar_flux && B.C.spherical()) {
            if (phys_face(B.c.bc[2])) zero_boundary_flux_x2(B, F1, F2, F3, true);
            if (phys_face(B.c.bc[3])) zero_boundary_flux_x2(B, F1, F2, F3, false);
        }
        flux_ct(B, F1, F2, F3);
    }
    boundaries_fix_flux(B, F);
}

// Inverter::BlockUtoP (+ B) over the interior
void orc_utop(void* hp, const double* U, double* P, double* pflag, double* fflag)
{
    const Block& B = ((Handle*)hp)->B;
    block_utop(B, U, P, pflag, fflag, B.ks, B.ke, B.js, B.je, B.is, B.ie);
}
// Floors::ApplyGRMHDFloors over the interior
// Inverter::MeshFixUtoP on a block after its inversion and floors (P, U, pflag as the stage leaves them)
void orc_fix_utop(void* hp, double* P, double* U, double* pflag)
{
    const Block& B = ((Handle*)hp)->B;
    stage_fix_utop(B, P, U, pflag);
}
void orc_floors(void* hp, double* P, double* U, double* pflag, double* fflag)
{
    const Block& B = ((Handle*)hp)->B;
    apply_grmhd_floors(B, P, U, pflag, fflag, B.ks, B.ke, B.js, B.je, B.is, B.ie);
}
// Flux::MeshPtoU over the entire block
void orc_ptou(void* hp, const double* P, double* U)
{
    const Block& B = ((Handle*)hp)->B;
    for (int k = 0; k < B.n3; ++k) for (int j = 0; j < B.n2; ++j) for (int i = 0; i < B.n1; ++i)
        p_to_u_cell(B, P, U, B.id(k, j, i), j, i);
}
void orc_boundaries(void* hp, double* P, double* U)
{
    apply_boundaries(((Handle*)hp)->B, P, U);
}

// One full RK2 step (both stages).  Returns the next dt per SetGlobalTimeStep + EstimateTimestep
// (kharma_driver.cpp:439-460, grmhd.cpp:294-339), and the raw minimum zone timestep.
void orc_step(void* hp, double* P, double* U, double* pflag, double* fflag, double dt,
              double* dt_next, double* min_ndt_out)
{
    Handle* h = (Handle*)hp;
    const Block& B = h->B;
    const size_t NV = (size_t)B.nv*B.N;
    h->P1.assign(NV, 0.); h->U1.assign(NV, 0.); h->U0.assign(U, U + NV);
    // the B primitives of the new state are always rebuilt from B_U; seed the fluid prims copy
    std::memcpy(h->P1.data(), P, NV*sizeof(double));
    stage(B, h->f, 0, dt, P, h->U0.data(), h->U0.data(), h->P1.data(), h->U1.data(), pflag, fflag);
    stage(B, h->f, 1, dt, h->P1.data(), h->U1.data(), h->U0.data(), P, U, pflag, fflag);
    const double mn = min_ndt(B, h->f);
    if (min_ndt_out) *min_ndt_out = mn;
    if (dt_next) {
        // EstimateTimestep: clip(cfl*min, dt_min, max_dt_increase*dt_last); SetGlobalTimeStep: min(2 dt, that)
        const double ndt = clip(mn * B.c.cfl, B.c.dt_min, B.c.max_dt_increase * dt);
        *dt_next = std::min(2.0 * dt, ndt);
    }
}

// One RK2 step with B_CT in place on (P, U, Bf[3][N]); returns the next dt like orc_step
void orc_ct_step(void* hp, double* P, double* U, double* Bf, double* pflag, double* fflag, double dt,
                 double* dt_next, double* min_ndt_out)
{
    Handle* h = (Handle*)hp;
    const Block& B = h->B;
    const size_t NV = (size_t)B.nv*B.N;
    h->P1.assign(P, P + NV); h->U1.assign(NV, 0.); h->U0.assign(U, U + NV);
    std::vector<double> B0(Bf, Bf + 3*B.N), B1(Bf, Bf + 3*B.N);
    ct_stage(B, h->f, 0, dt, P, h->U0.data(), h->U0.data(), B0.data(), B0.data(), h->P1.data(), h->U1.data(),
             B1.data(), pflag, fflag);
    ct_stage(B, h->f, 1, dt, h->P1.data(), h->U1.data(), h->U0.data(), B1.data(), B0.data(), P, U, Bf, pflag, fflag);
    const double mn = min_ndt(B, h->f);
    if (min_ndt_out) *min_ndt_out = mn;
    if (dt_next) {
        const double ndt = clip(mn * B.c.cfl, B.c.dt_min, B.c.max_dt_increase * dt);
        *dt_next = std::min(2.0 * dt, ndt);
    }
}

// Ghost zones of a B_CT block (khb_ct_boundaries): with physical faces the face field's ghost layers
// and the ghost zones' B from them, else the zone boundaries alone
void orc_ct_boundaries(void* hp, double* P, double* U, double* Bf)
{
    const Block& B = ((Handle*)hp)->B;
    if (ct_has_physical(B)) ct_apply_boundaries(B, P, U, Bf);
    else apply_boundaries(B, P, U);
}

// B_CT::BlockUtoP over the interior
void orc_ct_utop(void* hp, const double* Bf, double* P, double* U)
{
    const Block& B = ((Handle*)hp)->B;
    for (int k = B.ks; k <= B.ke; ++k) for (int j = B.js; j <= B.je; ++j) for (int i = B.is; i <= B.ie; ++i) {
        double Bp[3];
        ct_zone_b(B, Bf, k, j, i, Bp);
        const size_t c = B.id(k, j, i);
        for (int v = 0; v < 3; ++v) {
            P[(size_t)(5 + v)*B.N + c] = Bp[v];
            U[(size_t)(5 + v)*B.N + c] = Bp[v] * B.Gdet(center, j, i);
        }
    }
}

// B_CT::DangerousPtoU over the interior faces (the x3 faces of a 2D block: their zone's value)
void orc_ct_faces_from_prims(void* hp, const double* P, double* Bf)
{
    const Block& B = ((Handle*)hp)->B;
    const size_t N = B.N, sj = B.n1, sk = (size_t)B.n1*B.n2;
    const int d3 = B.ndim > 2;
    for (int k = B.ks; k <= B.ke + d3; ++k) for (int j = B.js; j <= B.je + 1; ++j) for (int i = B.is; i <= B.ie + 1; ++i) {
        const size_t c = B.id(k, j, i);
        if (j <= B.je && k <= B.ke) Bf[c] = B.Gdet(face1, j, i) * (P[5*N + c - 1] + P[5*N + c]) / 2;
        if (i <= B.ie && k <= B.ke) Bf[N + c] = B.Gdet(face2, j, i) * (P[6*N + c - sj] + P[6*N + c]) / 2;
        if (i <= B.ie && j <= B.je)
            Bf[2*N + c] = d3 ? B.Gdet(face3, j, i) * (P[7*N + c - sk] + P[7*N + c]) / 2 : B.Gdet(face3, j, i) * P[7*N + c];
    }
}

// max |face divergence| over the interior (b_ct.cpp:499-520)
double orc_ct_max_divb(void* hp, const double* Bf)
{
    const Block& B = ((Handle*)hp)->B;
    const size_t N = B.N, sj = B.n1, sk = (size_t)B.n1*B.n2;
    double m = 0.;
    for (int k = B.ks; k <= B.ke; ++k) for (int j = B.js; j <= B.je; ++j) for (int i = B.is; i <= B.ie; ++i) {
        const size_t c = B.id(k, j, i);
        double du = (Bf[c + 1] - Bf[c]) / B.c.dx1;
        if (B.ndim > 1) du += (Bf[N + c + sj] - Bf[N + c]) / B.c.dx2;
        if (B.ndim > 2) du += (Bf[2*N + c + sk] - Bf[2*N + c]) / B.c.dx3;
        m = std::max(m, std::fabs(du));
    }
    return m;
}

double orc_max_divb(void* hp, const double* U, int avoid_inner, int avoid_outer)
{
    return max_divb(((Handle*)hp)->B, U, avoid_inner, avoid_outer);
}

// Single-cell inversion, for golden/unit tests: U and P are nvar-long arrays at (j,i) of the centre
int orc_utop_cell(void* hp, int j, int i, const double* U, double* P)
{
    const Block& B = ((Handle*)hp)->B;
    return u_to_p(B, U, P, j, i, center, B.c.iter_max, B.c.err_tol);
}

// ---- EMHD explicit fluxes and the ImEx stage
void orc_get_flux_emhd(void* hp, const EmhdParams* ep, int dir, const double* P, double* F, double* cmax, double* cmin)
{
    get_flux_emhd(((Handle*)hp)->B, *ep, dir, P, F, cmax, cmin);
}
int orc_imex_stage(void* hp, const EmhdParams* ep, const ImplicitParams* ip, int stage, double dt,
                   const double* Pfull, const double* Ufull, const double* Psub, const double* Usub,
                   double* Pout, double* Uout, double* solve_norm, double* solve_fail, double* min_ndt)
{
    return imex_stage(((Handle*)hp)->B, *ep, *ip, stage - 1, dt, Pfull, Ufull, Psub, Usub, Pout, Uout,
                      solve_norm, solve_fail, min_ndt);
}
// The same with the floor and EMHD-limit flags of the interior zones ([N] each)
int orc_imex_stage_flags(void* hp, const EmhdParams* ep, const ImplicitParams* ip, int stage, double dt,
                         const double* Pfull, const double* Ufull, const double* Psub, const double* Usub,
                         double* Pout, double* Uout, double* solve_norm, double* solve_fail, double* min_ndt,
                         double* fflag, double* eflag)
{
    return imex_stage(((Handle*)hp)->B, *ep, *ip, stage - 1, dt, Pfull, Ufull, Psub, Usub, Pout, Uout,
                      solve_norm, solve_fail, min_ndt, fflag, eflag);
}

// ---- EMHD and the implicit solve.  All field arrays are [10][N] (slots rho..B3, q, dP).
void orc_get_connection(void* hp, double* conn)
{
    const Block& B = ((Handle*)hp)->B;
    std::memcpy(conn, B.conn.data(), B.conn.size()*sizeof(double));
}
void orc_emhd_ptou(void* hp, const EmhdParams* ep, const double* P, double* U)
{
    const Block& B = ((Handle*)hp)->B;
    emhd_ptou(B, *ep, B.c.gam, P, U);
}
void orc_emhd_add_source(void* hp, const EmhdParams* ep, const double* P, double* dUdt)
{
    const Block& B = ((Handle*)hp)->B;
    emhd_add_source(B, *ep, B.c.gam, P, dUdt);
}
// Residual and Jacobian at the solver state over the interior, as the split "implicit_jacobian"
// kernel stores them (implicit.cpp:286-320): res [nf][N], J [nf*nf][N] (row-major per zone).
void orc_implicit_jacobian(void* hp, const EmhdParams* ep, const ImplicitParams* ip, const double* Pf,
                           const double* Uf, const double* Ps, const double* S, const double* Psol, double dt,
                           double* J, double* res)
{
    const Block& B = ((Handle*)hp)->B;
    const size_t N = B.N;
    int map[7];
    const int nf = implicit_map(*ep, map);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = B.ks; k <= B.ke; ++k) for (int j = B.js; j <= B.je; ++j) for (int i = B.is; i <= B.ie; ++i) {
        const size_t c = B.id(k, j, i);
        double pf[NVE], uf[NVE], ps[NVE], s[NVE], psol[NVE], dUi[NVE] = {0}, Jz[49], rz[7];
        load10(Pf, N, c, pf); load10(Uf, N, c, uf); load10(Ps, N, c, ps); load10(S, N, c, s); load10(Psol, N, c, psol);
        implicit_dU(B, *ep, B.c.gam, pf, ps, j, i, dUi);
        if (ip->jacobian == 1) calc_jacobian_exact(B, *ep, B.c.gam, psol, pf, uf, ps, s, dUi, nf, map, j, i, dt, Jz, rz);
        else calc_jacobian_fd(B, *ep, B.c.gam, ip->jacobian_delta, psol, pf, uf, ps, s, dUi, nf, map, j, i, dt, Jz, rz);
        for (int q = 0; q < nf; ++q) res[(size_t)q*N + c] = rz[q];
        for (int q = 0; q < nf*nf; ++q) J[(size_t)q*N + c] = Jz[q];
    }
}
// Residual only at a trial state (the linesearch call of implicit.cpp:469-473)
void orc_implicit_residual(void* hp, const EmhdParams* ep, const double* Pf, const double* Uf, const double* Ps,
                           const double* S, const double* Ptest, double dt, double* res)
{
    const Block& B = ((Handle*)hp)->B;
    const size_t N = B.N;
    int map[7];
    const int nf = implicit_map(*ep, map);
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = B.ks; k <= B.ke; ++k) for (int j = B.js; j <= B.je; ++j) for (int i = B.is; i <= B.ie; ++i) {
        const size_t c = B.id(k, j, i);
        double pf[NVE], uf[NVE], ps[NVE], s[NVE], pt[NVE], dUi[NVE] = {0}, rz[7];
        load10(Pf, N, c, pf); load10(Uf, N, c, uf); load10(Ps, N, c, ps); load10(S, N, c, s); load10(Ptest, N, c, pt);
        implicit_dU(B, *ep, B.c.gam, pf, ps, j, i, dUi);
        calc_residual_t<double>(B, *ep, B.c.gam, pt, pf, uf, ps, s, dUi, nf, map, j, i, dt, rz);
        for (int q = 0; q < nf; ++q) res[(size_t)q*N + c] = rz[q];
    }
}
// Dense solve of one system with the reference's QR (use_qr = 1) or LU path; A row-major n x n.
void orc_dense_solve(int n, int use_qr, double* A, double* b)
{
    if (use_qr) qr_solve(n, A, b);
    else lu_solve(n, A, b);
}
int orc_implicit_step(void* hp, const EmhdParams* ep, const ImplicitParams* ip, const double* Pf, const double* Uf,
                      const double* Ps, const double* S, double* Psol, double* solve_norm, double* solve_fail,
                      double dt, double* maxnorm)
{
    const Block& B = ((Handle*)hp)->B;
    return implicit_step(B, *ep, *ip, B.c.gam, Pf, Uf, Ps, S, Psol, solve_norm, solve_fail, dt, maxnorm);
}
void orc_fix_solve(void* hp, const EmhdParams* ep, double* P, double* U, const double* solve_fail)
{
    const Block& B = ((Handle*)hp)->B;
    fix_solve(B, *ep, B.c.gam, P, U, solve_fail);
}

} // extern "C"

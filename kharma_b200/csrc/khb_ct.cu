// khb_ct.cu -- B_CT: the face-centred magnetic field package (kharma/b_ct/b_ct.cpp) on sm_100a.
//
// Per stage, after the face fluxes: k_ct_emfc (zone-centred EMF v x B from the stage primitives),
// k_ct_emf (edge EMFs: Balsara-Spicer flux averages plus the Gardiner-Stone corrections), then
// k_ct_faces (face change from the EMF circulation and the RK combination of the face field).  The
// zone pass then takes the zone B from the updated faces (ct_zone_b in khb_kernels.cuh).  EMFs are
// formed in the flux arithmetic FT (FP32 in the FP32-flux form); the face update is FP64.  Blocks are
// 2D or 3D.  Interior faces are the state; every EMF and zone-centred EMF they need lies within the
// flux ranges and the ghost zones.  X1/X2 faces may be physical (outflow, reflecting, or transmitting
// X2 faces): reflecting faces zero the EMFs on their domain-face edges (zero_EMF), transmitting ones
// average them (average_EMF), and after each stage the face field's ghost layers are filled
// (k_ct_face_tangential, k_ct_face_reflect, k_ct_face_outflow with the divergence cleaning,
// k_ct_face_transmit) before the ghost zones take B from their faces (k_ghost_ptou).
#include "khb_internal.hpp"
#include "khb_kernels.cuh"

#include <cstring>
#include <string>

namespace khb {

// Zone-centred EMF (b_ct.cpp:331-345): (b^2 u^3 - b^3 u^2, b^3 u^1 - b^1 u^3, b^1 u^2 - b^2 u^1) sqrt(-g)
template <typename FT>
__global__ void __launch_bounds__(128) k_ct_emfc(Dims d, DevGeom g, khb_fields P, FT* __restrict__ emfc, Box bx)
{
    int i, j, k;
    if (!box_cell(bx, blockIdx.x, i, j, k)) return;
    const long long c = ((long long)k*d.n2 + j)*d.n1 + i;
    ZoneGeom G;
    load_zone_geom(g, j, i, G);
    double Pz[8];
#pragma unroll
    for (int p = 0; p < 8; ++p) Pz[p] = __ldg(P.v[p] + c);
    const double gcon0[4] = {G.gcon[0][0], G.gcon[0][1], G.gcon[0][2], G.gcon[0][3]};
    FourVec<double> D;
    calc_4vecs<double, true>(G.gcov, G.gcon[0][0], gcon0, Pz, D);
    emfc[c]           = (FT)((D.bcon[2]*D.ucon[3] - D.bcon[3]*D.ucon[2]) * G.gdet);
    emfc[d.N + c]     = (FT)((D.bcon[3]*D.ucon[1] - D.bcon[1]*D.ucon[3]) * G.gdet);
    emfc[2*d.N + c]   = (FT)((D.bcon[1]*D.ucon[2] - D.bcon[2]*D.ucon[1]) * G.gdet);
}

// Edge EMFs (b_ct.cpp:262-410).  E1 at (i centre, j face, k face), E2 at (i face, j centre, k face),
// E3 at (i face, j face, k centre); flux(dir, var, zone) = F_dir[var N + zone].
template <typename FT>
__global__ void __launch_bounds__(128) k_ct_emf(Dims d, int scheme, const FT* __restrict__ F1, const FT* __restrict__ F2,
                                                const FT* __restrict__ F3, const FT* __restrict__ emfc, FT* __restrict__ emf,
                                                Box bx)
{
    int i, j, k;
    if (!box_cell(bx, blockIdx.x, i, j, k)) return;
    const long long N = d.N, sj = d.sj, sk = d.sk;
    const long long c = ((long long)k*d.n2 + j)*d.n1 + i;
    const long long V1 = 5*N, V2 = 6*N, V3 = 7*N;
    const FT q = (FT)0.25;
    auto f1 = [&](long long v, long long x) { return __ldg(F1 + v + x); };
    auto f2 = [&](long long v, long long x) { return __ldg(F2 + v + x); };
    auto f3 = [&](long long v, long long x) { return __ldg(F3 + v + x); };
    auto ec = [&](int v, long long x) { return __ldg(emfc + v*N + x); };
    FT e1, e2, e3;
    // Balsara & Spicer: the B fluxes averaged to the edge
    if (d.ndim > 2) {
        e1 = q*(-f2(V3, c - sk) - f2(V3, c) + f3(V2, c - sj) + f3(V2, c));
        e2 = q*(-f3(V1, c - 1) - f3(V1, c) + f1(V3, c - sk) + f1(V3, c));
        e3 = q*(-f1(V2, c - sj) - f1(V2, c) + f2(V1, c - 1) + f2(V1, c));
    } else {
        e1 = -f2(V3, c);
        e2 = f1(V3, c);
        e3 = q*(-f1(V2, c - sj) - f1(V2, c) + f2(V1, c - 1) + f2(V1, c));
    }
    if (scheme == KHB_CT_GS05_0) {
        // twice the face average less the average of the four zone-centred EMFs around the edge
        // (E1's average as b_ct.cpp:354-355 writes it, with the (j-1) zone twice)
        if (d.ndim > 2) {
            e1 = (FT)2 * e1 - q*(ec(0, c) + ec(0, c - sj) + ec(0, c - sj) + ec(0, c - sk - sj));
            e2 = (FT)2 * e2 - q*(ec(1, c) + ec(1, c - 1) + ec(1, c - sk) + ec(1, c - sk - 1));
        }
        e3 = (FT)2 * e3 - q*(ec(2, c) + ec(2, c - 1) + ec(2, c - sj) + ec(2, c - sj - 1));
    } else if (scheme == KHB_CT_GS05_C) {
        // E^c upwinded by the sign of the mass flux (b_ct.cpp:362-406)
        const FT zero = (FT)0;
        if (d.ndim > 2) {
            const FT e1_l3 = (f2(0, c - sk) >= zero) ? f3(V2, c - sj) - ec(0, c - sk - sj) : f3(V2, c) - ec(0, c - sk);
            const FT e1_r3 = (f2(0, c) >= zero)      ? f3(V2, c - sj) - ec(0, c - sj)      : f3(V2, c) - ec(0, c);
            const FT e1_l2 = (f3(0, c - sj) >= zero) ? -f2(V3, c - sk) - ec(0, c - sk - sj) : -f2(V3, c) - ec(0, c - sj);
            const FT e1_r2 = (f3(0, c) >= zero)      ? -f2(V3, c - sk) - ec(0, c - sk)      : -f2(V3, c) - ec(0, c);
            e1 += q*(e1_l3 + e1_r3 + e1_l2 + e1_r2);
            const FT e2_l3 = (f1(0, c - sk) >= zero) ? -f3(V1, c - 1) - ec(1, c - sk - 1) : -f3(V1, c) - ec(1, c - sk);
            const FT e2_r3 = (f1(0, c) >= zero)      ? -f3(V1, c - 1) - ec(1, c - 1)      : -f3(V1, c) - ec(1, c);
            const FT e2_l1 = (f3(0, c - 1) >= zero)  ? f1(V3, c - sk) - ec(1, c - sk - 1) : f1(V3, c) - ec(1, c - 1);
            const FT e2_r1 = (f3(0, c) >= zero)      ? f1(V3, c - sk) - ec(1, c - sk)     : f1(V3, c) - ec(1, c);
            e2 += q*(e2_l3 + e2_r3 + e2_l1 + e2_r1);
        }
        const FT e3_l2 = (f1(0, c - sj) >= zero) ? f2(V1, c - 1) - ec(2, c - sj - 1) : f2(V1, c) - ec(2, c - sj);
        const FT e3_r2 = (f1(0, c) >= zero)      ? f2(V1, c - 1) - ec(2, c - 1)      : f2(V1, c) - ec(2, c);
        const FT e3_l1 = (f2(0, c - 1) >= zero)  ? -f1(V2, c - sj) - ec(2, c - sj - 1) : -f1(V2, c) - ec(2, c - 1);
        const FT e3_r1 = (f2(0, c) >= zero)      ? -f1(V2, c - sj) - ec(2, c - sj)     : -f1(V2, c) - ec(2, c);
        e3 += q*(e3_l2 + e3_r2 + e3_l1 + e3_r1);
    }
    emf[c] = e1;
    emf[N + c] = e2;
    emf[2*N + c] = e3;
}

// Face change from the EMF circulation (b_ct.cpp:412-470; edge lengths and face areas of the uniform
// native grid) and the RK combination Bf_out = 1.0 (gam0 Bf_s + gam1 Bf_0) + beta dt dBf/dt
// (WeightedSumDataFace twice, kharma_driver.cpp:339-387).  One thread per (i, j, k) of
// [is, ie+1] x [js, je+1] x [ks, ke(+1 in 3D)]; each component takes its own face range.
template <typename FT>
__global__ void __launch_bounds__(128) k_ct_faces(Dims d, Phys ph, const FT* __restrict__ emf, khb_fields Bs,
                                                  khb_fields B0, khb_fields Bout, double g0, double g1, double bdt_host,
                                                  const double* dt_dev, double beta, Box bx)
{
    int i, j, k;
    if (!box_cell(bx, blockIdx.x, i, j, k)) return;
    const long long N = d.N, sj = d.sj, sk = d.sk;
    const long long c = ((long long)k*d.n2 + j)*d.n1 + i;
    const double bdt = dt_dev ? beta * __ldg(dt_dev) : bdt_host;
    auto E = [&](int v, long long x) { return (double)__ldg(emf + v*N + x); };
    const double L1 = ph.dx1, L2 = ph.dx2, L3 = ph.dx3;
    const bool d3 = d.ndim > 2;
    if (j <= d.je && k <= d.ke) {
        double db = (-L3 * E(2, c + sj) + L3 * E(2, c));
        if (d3) db += (L2 * E(1, c + sk) - L2 * E(1, c));
        db /= (L2 * L3);
        const double x = g0 * Bs.v[0][c] + g1 * B0.v[0][c];
        Bout.v[0][c] = 1.0 * x + bdt * db;
    }
    if (i <= d.ie && k <= d.ke) {
        double db = (L3 * E(2, c + 1) - L3 * E(2, c));
        if (d3) db += (-L1 * E(0, c + sk) + L1 * E(0, c));
        db /= (L1 * L3);
        const double x = g0 * Bs.v[1][c] + g1 * B0.v[1][c];
        Bout.v[1][c] = 1.0 * x + bdt * db;
    }
    if (i <= d.ie && j <= d.je) {
        const double db = (-L2 * E(1, c + 1) + L2 * E(1, c) + L1 * E(0, c + sj) - L1 * E(0, c)) / (L1 * L2);
        const double x = g0 * Bs.v[2][c] + g1 * B0.v[2][c];
        Bout.v[2][c] = 1.0 * x + bdt * db;
    }
}

// B_CT::BlockUtoP over a box of zones (b_ct.cpp:160-188)
__global__ void __launch_bounds__(128) k_ct_center(Dims d, DevGeom g, khb_fields Bf, khb_fields P, khb_fields U, Box bx)
{
    int i, j, k;
    if (!box_cell(bx, blockIdx.x, i, j, k)) return;
    const long long c = ((long long)k*d.n2 + j)*d.n1 + i;
    const double* const F[3] = {Bf.v[0], Bf.v[1], Bf.v[2]};
    double Bp[3];
    ct_zone_b(d, g, F, c, j, i, Bp);
    const double gdet = __ldg(g.gdet[3] + (long long)j*g.G1 + i);
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        P.v[5 + v][c] = Bp[v];
        U.v[5 + v][c] = Bp[v] * gdet;
    }
}

// B_CT::DangerousPtoU over the interior faces (b_ct.cpp:190-230); the x3 faces of a 2D block hold
// sqrt(-g) B^3 of their zone
__global__ void __launch_bounds__(128) k_ct_from_prims(Dims d, DevGeom g, khb_fields P, khb_fields Bf, Box bx)
{
    int i, j, k;
    if (!box_cell(bx, blockIdx.x, i, j, k)) return;
    const long long c = ((long long)k*d.n2 + j)*d.n1 + i;
    const long long gi = (long long)j*g.G1 + i;
    if (j <= d.je && k <= d.ke)
        Bf.v[0][c] = __ldg(g.gdet[0] + gi) * (P.v[5][c - 1] + P.v[5][c]) / 2;
    if (i <= d.ie && k <= d.ke)
        Bf.v[1][c] = __ldg(g.gdet[1] + gi) * (P.v[6][c - d.sj] + P.v[6][c]) / 2;
    if (i <= d.ie && j <= d.je)
        Bf.v[2][c] = (d.ndim > 2) ? __ldg(g.gdet[2] + gi) * (P.v[7][c - d.sk] + P.v[7][c]) / 2
                                  : __ldg(g.gdet[2] + gi) * P.v[7][c];
}

// max |face divergence| over the interior (face_div, b_ct_functions.hpp:47-56); values >= 0 so the
// maximum is taken over bit patterns
__global__ void __launch_bounds__(128) k_ct_divb(Dims d, Phys ph, khb_fields Bf, unsigned long long* word, Box bx)
{
    int i, j, k;
    double v = 0.;
    if (box_cell(bx, blockIdx.x, i, j, k)) {
        const long long c = ((long long)k*d.n2 + j)*d.n1 + i;
        double du = (Bf.v[0][c + 1] - Bf.v[0][c]) / ph.dx1;
        if (d.ndim > 1) du += (Bf.v[1][c + d.sj] - Bf.v[1][c]) / ph.dx2;
        if (d.ndim > 2) du += (Bf.v[2][c + d.sk] - Bf.v[2][c]) / ph.dx3;
        v = fabs(du);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) atomicMax(word, (unsigned long long)__double_as_longlong(v));
}

// ---- physical faces (boundaries.cpp:186-207 defaults, 432-490; b_ct_boundaries.cpp:40-262)
// Index of the zone / face at position x along bdir and (a, b) across it (a the faster of the two)
__device__ __forceinline__ long long ct_at(const Dims& d, int bdir, int x, int a, int b)
{
    int i, j, k;
    if (bdir == 1) { i = x; j = a; k = b; } else if (bdir == 2) { i = a; j = x; k = b; } else { i = a; j = b; k = x; }
    return ((long long)k*d.n2 + j)*d.n1 + i;
}
__host__ __device__ inline int ct_na(const Dims& d, int bdir) { return (bdir == 1) ? d.n2 : d.n1; }
__host__ __device__ inline int ct_nb(const Dims& d, int bdir) { return (bdir == 3) ? d.n2 : d.n3; }
__host__ __device__ inline int ct_nx(const Dims& d, int bdir) { return (bdir == 1) ? d.n1 : (bdir == 2) ? d.n2 : d.n3; }
__host__ __device__ inline int ct_s(const Dims& d, int bdir) { return (bdir == 1) ? d.is : (bdir == 2) ? d.js : d.ks; }
__host__ __device__ inline int ct_e(const Dims& d, int bdir) { return (bdir == 1) ? d.ie : (bdir == 2) ? d.je : d.ke; }

// zero_EMF (b_ct_boundaries.cpp:40-62): the EMF components in mask (bit v: E(v+1)) on the domain
// face's edges, over the whole face plane
template <typename FT>
__global__ void k_ct_zero_emf(Dims d, int bdir, int f, int mask, FT* emf)
{
    const int na = ct_na(d, bdir), nb = ct_nb(d, bdir);
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)na*nb) return;
    const long long c = ct_at(d, bdir, f, (int)(t % na), (int)(t / na));
#pragma unroll
    for (int v = 0; v < 3; ++v)
        if (mask & (1 << v)) emf[v*d.N + c] = (FT)0;
}

// average_EMF on a transmitting X2 face (b_ct_boundaries.cpp:64-186, 3D): E1 on the polar face
// replaced by its average over the interior x3 edges, summed over k upwards (the reference's team
// reduction has no fixed order), every k set.  One thread per i.
template <typename FT>
__global__ void k_ct_average_emf1(Dims d, int jf, FT* emf)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.n1) return;
    double sum = 0.;
    for (int k = d.ks; k <= d.ke; ++k) sum += (double)emf[((long long)k*d.n2 + jf)*d.n1 + i];
    const double av = sum / (d.ke + 1 - d.ks);
    for (int k = 0; k < d.n3; ++k) emf[((long long)k*d.n2 + jf)*d.n1 + i] = (FT)av;
}

// OneBlockTransmit on the face field (one_block_transmit.cpp:60-143), X2 faces: the mirror face
// half-way round in x3; F1 copied, F3 inverted over the ghost rows, F2 inverted beyond the polar face
// and zero on it.  One thread per (k, row, i) of the rows j < js (or > je) and the polar face row.
__global__ void k_ct_face_transmit(Dims d, khb_fields Bf, int binner)
{
    const int s = d.js, e = d.je, f = binner ? s : e + 1;
    const int rows = binner ? s + 1 : d.n2 - f;                   // ghost rows plus the polar face row
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)rows * d.n1 * d.n3) return;
    const int i = (int)(t % d.n1);
    const long long r = t / d.n1;
    const int l = (int)(r % rows), k = (int)(r / rows);
    const int j = binner ? l : f + l;
    const int ki = ((k - d.ks + d.nx3 / 2) % d.nx3) + d.ks;
    if (ki < 0 || ki >= d.n3) return;
    const long long c = ((long long)k*d.n2 + j)*d.n1 + i;
    if (binner ? j < s : j > e) {
        const int ji = binner ? 2*s - 1 - j : 2*e + 1 - j;
        const long long m = ((long long)ki*d.n2 + ji)*d.n1 + i;
        Bf.v[0][c] = Bf.v[0][m];
        Bf.v[2][c] = -Bf.v[2][m];
    }
    const int ji = 2*f - j;
    if (ji < 0 || ji >= d.n2) return;
    Bf.v[1][c] = (j == f) ? 0. : -Bf.v[1][((long long)ki*d.n2 + ji)*d.n1 + i];
}

// The tangential face components of one face's ghost layers, as zones: outflow copies the first
// interior layer, reflecting the mirror layer (no sign change)
__global__ void k_ct_face_tangential(Dims d, khb_fields Bf, int bdir, int binner, int outflow)
{
    const int na = ct_na(d, bdir), nb = ct_nb(d, bdir);
    const int s = ct_s(d, bdir), e = ct_e(d, bdir);
    const int layers = binner ? s : ct_nx(d, bdir) - 1 - e;
    const long long plane = (long long)na*nb;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2*layers*plane) return;
    const int comp = (int)(t / (layers*plane));
    const long long r = t - comp*(layers*plane);
    const int l = (int)(r / plane);
    const long long q = r - l*plane;
    const int a = (int)(q % na), b = (int)(q / na);
    const int v = (bdir == 1) ? 1 + comp : ((bdir == 2) ? 2*comp : comp);     // the components other than bdir-1
    const int x = binner ? l : e + 1 + l;
    const int src = outflow ? (binner ? s : e) : (binner ? 2*s - 1 - x : 2*e + 1 - x);
    Bf.v[v][ct_at(d, bdir, x, a, b)] = Bf.v[v][ct_at(d, bdir, src, a, b)];
}

// reflect_face_vector (boundaries.cpp:458-479): the normal component zero on the domain face f and
// minus the mirror face beyond it
__global__ void k_ct_face_reflect(Dims d, khb_fields Bf, int bdir, int binner)
{
    const int na = ct_na(d, bdir), nb = ct_nb(d, bdir), nx = ct_nx(d, bdir);
    const int f = binner ? ct_s(d, bdir) : ct_e(d, bdir) + 1;
    const int layers = binner ? f + 1 : nx - f;
    const long long plane = (long long)na*nb;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= layers*plane) return;
    const int l = (int)(t / plane);
    const long long q = t - l*plane;
    const int a = (int)(q % na), b = (int)(q / na);
    const int x = binner ? l : f + l;
    const int m = 2*f - x;
    if (m < 0 || m >= nx) return;
    double* F = Bf.v[bdir - 1];
    F[ct_at(d, bdir, x, a, b)] = (x == f) ? 0. : -F[ct_at(d, bdir, m, a, b)];
}

// Outflow normal component: the domain face copied outward (Parthenon's outflow), then clean_face_B
// (DestructiveBoundaryClean, b_ct_boundaries.cpp:190-262): from the domain face outward each face
// closes the zone between it and the previous face with zero divergence.  One thread per column
// across the face, all layers in order; the cleaning covers the columns whose transverse upper faces
// are stored (all but the last transverse layer).
__global__ void k_ct_face_outflow(Dims d, Phys ph, khb_fields Bf, int bdir, int binner)
{
    const int na = ct_na(d, bdir), nb = ct_nb(d, bdir), nx = ct_nx(d, bdir);
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)na*nb) return;
    const int a = (int)(t % na), b = (int)(t / na);
    const int f = binner ? ct_s(d, bdir) : ct_e(d, bdir) + 1;
    double* Fn = Bf.v[bdir - 1];
    const double ff = Fn[ct_at(d, bdir, f, a, b)];
    if (binner) { for (int x = 0; x < f; ++x) Fn[ct_at(d, bdir, x, a, b)] = ff; }
    else { for (int x = f + 1; x < nx; ++x) Fn[ct_at(d, bdir, x, a, b)] = ff; }
    const int d3 = d.ndim > 2;
    if (a >= na - 1 || b >= nb - ((bdir == 3) ? 1 : d3)) return;
    const double A1 = ph.dx2 * ph.dx3, A2 = ph.dx1 * ph.dx3, A3 = ph.dx1 * ph.dx2;
    const int osign = binner ? -1 : 1;
    const double nsign = (double)(-(-osign));
    if (bdir == 3) {
        // X3 faces (b_ct_boundaries.cpp:249-268): both in-plane components close the zone
        const double* F1 = Bf.v[0];
        const double* F2 = Bf.v[1];
        for (int layer = 0; layer < nx; ++layer) {
            const int x = binner ? f - layer : f + layer;
            if (x < 0 || x > nx - 1) break;
            const int lf = binner ? x + 1 : x - 1, lc = binner ? x : x - 1;
            const long long zc = ct_at(d, 3, lc, a, b);
            const double nf = nsign * Fn[ct_at(d, 3, lf, a, b)] * A3 - (F1[zc + 1] * A1 - F1[zc] * A1)
                              - (F2[zc + d.sj] * A2 - F2[zc] * A2);
            Fn[ct_at(d, 3, x, a, b)] = (double)osign * nf / A3;
        }
        return;
    }
    const double* Ft = Bf.v[(bdir == 1) ? 1 : 0];                 // the other in-plane component
    const double* F3 = Bf.v[2];
    const double At = (bdir == 1) ? A2 : A1, An = (bdir == 1) ? A1 : A2;
    const long long up = (bdir == 1) ? d.sj : 1;                  // its upper face across the column
    for (int layer = 0; layer < nx; ++layer) {
        const int x = binner ? f - layer : f + layer;
        if (x < 0 || x > nx - 1) break;
        const int lf = binner ? x + 1 : x - 1, lc = binner ? x : x - 1;
        const long long zc = ct_at(d, bdir, lc, a, b);
        double nf = nsign * Fn[ct_at(d, bdir, lf, a, b)] * An - (Ft[zc + up] * At - Ft[zc] * At);
        if (d3) nf -= F3[zc + d.sk] * A3 - F3[zc] * A3;
        Fn[ct_at(d, bdir, x, a, b)] = (double)osign * nf / An;
    }
}

namespace {

Box interior_box(const Dims& d) { return make_box(d.is, d.js, d.ks, d.ie - d.is + 1, d.je - d.js + 1, d.ke - d.ks + 1); }

// Faces [is, ie+1] x [js, je+1] x [ks, ke(+1 in 3D)]
Box face_box(const Dims& d)
{
    return make_box(d.is, d.js, d.ks, d.ie - d.is + 2, d.je - d.js + 2, d.ke - d.ks + 1 + (d.ndim > 2));
}

template <typename FT>
void edge_emf(khb_ctx* ctx, const khb_fields& Ps, cudaStream_t st)
{
    const Dims& d = ctx->d;
    FT* emfc = (FT*)ctx->ct_emfc;
    // zone-centred EMFs over the interior +-1 in active directions (the edges' neighbours)
    const int h3 = d.ndim > 2;
    const Box zb = make_box(d.is - 1, d.js - 1, d.ks - h3, d.ie - d.is + 3, d.je - d.js + 3, d.ke - d.ks + 1 + 2*h3);
    if (ctx->ph.ct_scheme != KHB_CT_BS99)
        k_ct_emfc<FT><<<box_blocks(zb), 128, 0, st>>>(d, ctx->g, Ps, emfc, zb);
    const Box eb = face_box(d);
    k_ct_emf<FT><<<box_blocks(eb), 128, 0, st>>>(d, ctx->ph.ct_scheme, (const FT*)ctx->F[0], (const FT*)ctx->F[1],
                                                  (const FT*)ctx->F[2], emfc, (FT*)ctx->emf, eb);
}

} // namespace

int ct_emf(khb_ctx* ctx, const khb_fields& Ps, cudaStream_t st)
{
    if (ctx->fp32) edge_emf<float>(ctx, Ps, st); else edge_emf<double>(ctx, Ps, st);
    ctx->launches += 1 + (ctx->ph.ct_scheme != KHB_CT_BS99);
    const Dims& d = ctx->d;
    for (int face = 0; face < 2 * d.ndim; ++face) {
        if (d.bc[face] == KHB_BC_TRANSMITTING) {
            const int jf = (face == 2) ? d.js : d.je + 1;
            const long long n = (long long)d.n1 * d.n3;
            if (ctx->ph.spherical) {                     // E3 only (component mask 4)
                if (ctx->fp32) k_ct_zero_emf<float><<<blocks_for(n, 128), 128, 0, st>>>(d, 2, jf, 4, (float*)ctx->emf);
                else k_ct_zero_emf<double><<<blocks_for(n, 128), 128, 0, st>>>(d, 2, jf, 4, (double*)ctx->emf);
                ctx->launches += 1;
            }
            if (d.ndim > 2) {
                if (ctx->fp32) k_ct_average_emf1<float><<<blocks_for(d.n1, 128), 128, 0, st>>>(d, jf, (float*)ctx->emf);
                else k_ct_average_emf1<double><<<blocks_for(d.n1, 128), 128, 0, st>>>(d, jf, (double*)ctx->emf);
                ctx->launches += 1;
            }
            continue;
        }
        if (d.bc[face] != KHB_BC_REFLECTING) continue;
        const int bdir = face / 2 + 1, binner = (face % 2) == 0;
        const int f = binner ? ct_s(d, bdir) : ct_e(d, bdir) + 1;
        const long long n = (long long)ct_na(d, bdir) * ct_nb(d, bdir);
        const int mask = 7 & ~(1 << (bdir - 1));        // the two components along the face
        if (ctx->fp32) k_ct_zero_emf<float><<<blocks_for(n, 128), 128, 0, st>>>(d, bdir, f, mask, (float*)ctx->emf);
        else k_ct_zero_emf<double><<<blocks_for(n, 128), 128, 0, st>>>(d, bdir, f, mask, (double*)ctx->emf);
        ctx->launches += 1;
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? KHB_OK : set_error(KHB_ERR_CUDA, std::string("B_CT EMF: ") + cudaGetErrorString(e));
}

// The face field's ghost layers at the physical faces, in Parthenon's order (x1 faces, x2 faces, then
// inner x1 again with fix_corner)
int ct_face_boundaries(khb_ctx* ctx, const khb_fields& Bf, cudaStream_t st)
{
    const Dims& d = ctx->d;
    auto one = [&](int face) {
        const int bdir = face / 2 + 1, binner = (face % 2) == 0;
        if (d.bc[face] == KHB_BC_TRANSMITTING) {
            const int rows = binner ? d.js + 1 : d.n2 - (d.je + 1);
            k_ct_face_transmit<<<blocks_for((long long)rows * d.n1 * d.n3, 128), 128, 0, st>>>(d, Bf, binner);
            ctx->launches += 1;
            return;
        }
        const int outflow = d.bc[face] == KHB_BC_OUTFLOW;
        const long long plane = (long long)ct_na(d, bdir) * ct_nb(d, bdir);
        const int layers = binner ? ct_s(d, bdir) : ct_nx(d, bdir) - 1 - ct_e(d, bdir);
        k_ct_face_tangential<<<blocks_for(2 * layers * plane, 128), 128, 0, st>>>(d, Bf, bdir, binner, outflow);
        if (outflow) {
            k_ct_face_outflow<<<blocks_for(plane, 128), 128, 0, st>>>(d, ctx->ph, Bf, bdir, binner);
        } else {
            const int f = binner ? ct_s(d, bdir) : ct_e(d, bdir) + 1;
            const int nl = binner ? f + 1 : ct_nx(d, bdir) - f;
            k_ct_face_reflect<<<blocks_for(nl * plane, 128), 128, 0, st>>>(d, Bf, bdir, binner);
        }
        ctx->launches += 2;
    };
    for (int face = 0; face < 2 * d.ndim; ++face) {
        if (!phys_face(d.bc[face])) continue;
        one(face);
        if (face == 3 && ctx->cfg.fix_corner_inner && phys_face(d.bc[0])) one(0);
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? KHB_OK : set_error(KHB_ERR_CUDA, std::string("B_CT face boundaries: ") + cudaGetErrorString(e));
}

int ct_face_update(khb_ctx* ctx, int stage, double dt, const khb_fields& Bs, const khb_fields& B0,
                   const khb_fields& Bout, cudaStream_t st)
{
    const Dims& d = ctx->d;
    const int s = stage - 1;
    const Box fb = face_box(d);
    if (ctx->fp32)
        k_ct_faces<float><<<box_blocks(fb), 128, 0, st>>>(d, ctx->ph, (const float*)ctx->emf, Bs, B0, Bout, kRkGam0[s],
                                                          kRkGam1[s], kRkBeta[s] * dt, ctx->dt_active, kRkBeta[s], fb);
    else
        k_ct_faces<double><<<box_blocks(fb), 128, 0, st>>>(d, ctx->ph, (const double*)ctx->emf, Bs, B0, Bout, kRkGam0[s],
                                                           kRkGam1[s], kRkBeta[s] * dt, ctx->dt_active, kRkBeta[s], fb);
    ctx->launches += 1;
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? KHB_OK : set_error(KHB_ERR_CUDA, std::string("B_CT face update: ") + cudaGetErrorString(e));
}

} // namespace khb

using namespace khb;

namespace {
int ct_check(const khb_ctx* ctx, const char* who)
{
    if (!ctx || !ctx->geom_set) return set_error(KHB_ERR_STATE, std::string(who) + ": context without geometry");
    if (ctx->ph.ct_scheme == KHB_CT_NONE) return set_error(KHB_ERR_STATE, std::string(who) + ": block is not B_CT");
    return KHB_OK;
}
bool faces_ok(const khb_fields* f) { return f && f->v[0] && f->v[1] && f->v[2]; }
}

extern "C" {

int khb_ct_utop(khb_ctx* ctx, const khb_fields* Bf, const khb_fields* P, const khb_fields* U, void* stream)
{
    KHB_RANGE("khb_ct_utop");
    int rc;
    if ((rc = ct_check(ctx, "khb_ct_utop"))) return rc;
    if (!faces_ok(Bf) || !P || !U) return set_error(KHB_ERR_ARG, "khb_ct_utop: NULL argument");
    const Box zb = interior_box(ctx->d);
    k_ct_center<<<box_blocks(zb), 128, 0, (cudaStream_t)stream>>>(ctx->d, ctx->g, *Bf, *P, *U, zb);
    ctx->launches += 1;
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? KHB_OK : set_error(KHB_ERR_CUDA, std::string("khb_ct_utop: ") + cudaGetErrorString(e));
}

int khb_ct_faces_from_prims(khb_ctx* ctx, const khb_fields* P, const khb_fields* Bf, void* stream)
{
    KHB_RANGE("khb_ct_faces_from_prims");
    int rc;
    if ((rc = ct_check(ctx, "khb_ct_faces_from_prims"))) return rc;
    if (!faces_ok(Bf) || !P) return set_error(KHB_ERR_ARG, "khb_ct_faces_from_prims: NULL argument");
    const Box fb = face_box(ctx->d);
    k_ct_from_prims<<<box_blocks(fb), 128, 0, (cudaStream_t)stream>>>(ctx->d, ctx->g, *P, *Bf, fb);
    ctx->launches += 1;
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? KHB_OK : set_error(KHB_ERR_CUDA, std::string("khb_ct_faces_from_prims: ") + cudaGetErrorString(e));
}

int khb_ct_max_divb(khb_ctx* ctx, const khb_fields* Bf, double* max_divb_host, void* stream)
{
    KHB_RANGE("khb_ct_max_divb");
    int rc;
    if ((rc = ct_check(ctx, "khb_ct_max_divb"))) return rc;
    if (!faces_ok(Bf) || !max_divb_host) return set_error(KHB_ERR_ARG, "khb_ct_max_divb: NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(ctx->words + 1, 0, sizeof(unsigned long long), st);
    const Box zb = interior_box(ctx->d);
    if (e == cudaSuccess) {
        k_ct_divb<<<box_blocks(zb), 128, 0, st>>>(ctx->d, ctx->ph, *Bf, ctx->words + 1, zb);
        e = cudaGetLastError();
    }
    unsigned long long bits = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bits, ctx->words + 1, sizeof(bits), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return set_error(KHB_ERR_CUDA, std::string("khb_ct_max_divb: ") + cudaGetErrorString(e));
    ctx->launches += 1;
    std::memcpy(max_divb_host, &bits, sizeof(double));
    return KHB_OK;
}

} // extern "C"

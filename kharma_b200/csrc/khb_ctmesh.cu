// khb_ctmesh.cu -- static mesh refinement of B_CT (face-centred field) MHD blocks: the corrections
// between a stage's fluxes and its update, and the ghost exchange after it, across blocks of
// neighbouring levels.  Tables come from the host (kharma_b200/ctmesh.py):
//   k_ctm_flux   coarse face flux of the fluid variables = mean of the 2^(ndim-1) fine fluxes
//   k_ctm_emf    coarse edge EMF = mean of the fine edge EMFs along it (one where the edge is inactive)
//   k_ctm_cell   ghost-zone fluid primitives: copy, restriction (mean of 2^ndim fine zones) or
//                prolongation (minmod slopes, +-1/4), the operators of the hydro mesh
//   k_ctm_face   ghost faces: copy, restriction (mean of the fine faces on the coarse face),
//                prolongation onto faces shared with a coarse face (value plus minmod tangential
//                slopes, +-1/4) and onto faces inside a coarse zone (Olivares et al.'s
//                divergence-preserving operator, b_ct_functions.hpp:151-200)
// after which each block's ghost zones take B from their faces and U = U(P)
// (khb_ct_ghost_from_faces).  The kharma driver's exchange (khb_ctmesh_exchange_cons) moves the
// updated conserved fluid variables and the seed primitives by the same entries, between the update
// and the inversion, then inverts each ghost zone like the interior:
//   k_ctm_cell_cons    ghost-zone U (fluid) and seed P (fluid) by the entries
//   k_ctm_ghost_cell   B and U_B from the faces, inversion, floors, U = U(P) (the zone pass's cell half)
// All blocks have one shape and FP64 fluxes, in any coordinate system: the face field holds
// sqrt(-g) B^i and the EMFs and fluxes their sqrt(-g)-weighted values, so that, as in Parthenon's
// operators, areas and lengths are products of the native zone widths.
#include "khb_internal.hpp"
#include "khb_kernels.cuh"

#include <cstring>
#include <string>
#include <vector>

namespace khb {

struct CtmBlock {
    double* P[8];
    double* Bf[3];
    double* F[3];          // the context's raw face fluxes, [nv][N] per direction
    double* emf;           // the context's edge EMFs, [3][N]
    double dx[3];
};

struct CtmDims {
    int n1, n2, n3, ndim;
    long long N, sj, sk;
};

// What the ghost cell pass of one block reads: the block's shape, metric and physics, and its
// zone-pass arguments (Ps the seeds, Us = Uout the updated state, Pout, flags, Bf the faces)
struct CtmZoneBlock {
    Dims d;
    DevGeom g;
    Phys ph;
    ZoneArgs<double> a;
};

__device__ __forceinline__ double ctm_minmod(double a, double b)
{
    return (a * b > 0.) ? ((fabs(a) < fabs(b)) ? a : b) : 0.;
}

__global__ void __launch_bounds__(128) k_ctm_flux(const CtmBlock* __restrict__ B, CtmDims d, const int* __restrict__ t6,
                                                  long long n)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int* t = t6 + 6 * e;
    const int dir = __ldg(t + 1);
    double* Fc = B[__ldg(t)].F[dir - 1];
    const double* Ff = B[__ldg(t + 3)].F[dir - 1];
    const long long cc = __ldg(t + 2), fc = __ldg(t + 4);
    const long long s1 = (dir == 1) ? d.sj : 1;
    const long long s2 = (dir == 3) ? d.sj : d.sk;
    for (int p = 0; p < 5; ++p) {
        const double* f = Ff + p * d.N + fc;
        Fc[p * d.N + cc] = (d.ndim > 2) ? ((f[0] + f[s1]) + (f[s2] + f[s1 + s2])) * 0.25 : (f[0] + f[s1]) * 0.5;
    }
}

__global__ void __launch_bounds__(128) k_ctm_emf(const CtmBlock* __restrict__ B, CtmDims d, const int* __restrict__ t6,
                                                 long long n)
{
    const long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= n) return;
    const int* t = t6 + 6 * x;
    const int e = __ldg(t + 1);
    const long long cc = __ldg(t + 2), fc = __ldg(t + 4);
    const double* Ef = B[__ldg(t + 3)].emf + e * d.N;
    const long long se = (e == 0) ? 1 : ((e == 1) ? d.sj : d.sk);
    const bool active = e < d.ndim;
    B[__ldg(t)].emf[e * d.N + cc] = active ? (Ef[fc] + Ef[fc + se]) * 0.5 : Ef[fc];
}

// Ghost-zone fluid primitives (entries {dst block, dst zone, op, src block, src zone, aux}: the hydro
// mesh's format; op 0 copy, 1 restriction, 2 prolongation with aux bit a for the + side along a)
__global__ void __launch_bounds__(128) k_ctm_cell(const CtmBlock* __restrict__ B, CtmDims d, const int* __restrict__ t6,
                                                  long long begin, long long end)
{
    const long long e = begin + (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= end) return;
    const int* t = t6 + 6 * e;
    const CtmBlock& D = B[__ldg(t)];
    const CtmBlock& S = B[__ldg(t + 3)];
    const long long cd = __ldg(t + 1), cs = __ldg(t + 4);
    const int op = __ldg(t + 2), aux = __ldg(t + 5);
    const long long st[3] = {1, d.sj, d.sk};
    for (int p = 0; p < 5; ++p) {
        const double* q = S.P[p];
        double v;
        if (op == 0) {
            v = q[cs];
        } else if (op == 1) {
            double r = (q[cs] + q[cs + 1]);
            if (d.ndim > 1) r = r + (q[cs + d.sj] + q[cs + d.sj + 1]);
            if (d.ndim > 2) r = r + ((q[cs + d.sk] + q[cs + d.sk + 1]) + (q[cs + d.sk + d.sj] + q[cs + d.sk + d.sj + 1]));
            v = r * ((d.ndim > 2) ? 0.125 : (d.ndim > 1) ? 0.25 : 0.5);
        } else {
            const double uc = q[cs];
            v = uc;
            for (int a = 0; a < d.ndim; ++a) {
                const double sl = ctm_minmod(uc - q[cs - st[a]], q[cs + st[a]] - uc);
                v += ((aux >> a) & 1) ? 0.25 * sl : -0.25 * sl;
            }
        }
        D.P[p][cd] = v;
    }
}

// The kharma driver's exchange of a B_CT mesh: the fluid part of the updated conserved state (U) and of
// the seed primitives (P) by the entry's operator, into the destination's same arrays
__global__ void __launch_bounds__(128) k_ctm_cell_cons(const CtmBlock* __restrict__ Bu, const CtmBlock* __restrict__ Bs,
                                                       CtmDims d, const int* __restrict__ t6, long long begin,
                                                       long long end)
{
    const long long e = begin + (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= end) return;
    const int* t = t6 + 6 * e;
    const long long cd = __ldg(t + 1), cs = __ldg(t + 4);
    const int op = __ldg(t + 2), aux = __ldg(t + 5);
    const long long st[3] = {1, d.sj, d.sk};
    for (int w = 0; w < 2; ++w) {
        const CtmBlock* B = w ? Bs : Bu;
        const CtmBlock& D = B[__ldg(t)];
        const CtmBlock& S = B[__ldg(t + 3)];
        for (int p = 0; p < 5; ++p) {
            const double* q = S.P[p];
            double v;
            if (op == 0) {
                v = q[cs];
            } else if (op == 1) {
                double r = (q[cs] + q[cs + 1]);
                if (d.ndim > 1) r = r + (q[cs + d.sj] + q[cs + d.sj + 1]);
                if (d.ndim > 2) r = r + ((q[cs + d.sk] + q[cs + d.sk + 1]) + (q[cs + d.sk + d.sj] + q[cs + d.sk + d.sj + 1]));
                v = r * ((d.ndim > 2) ? 0.125 : (d.ndim > 1) ? 0.25 : 0.5);
            } else {
                const double uc = q[cs];
                v = uc;
                for (int a = 0; a < d.ndim; ++a) {
                    const double sl = ctm_minmod(uc - q[cs - st[a]], q[cs + st[a]] - uc);
                    v += ((aux >> a) & 1) ? 0.25 * sl : -0.25 * sl;
                }
            }
            D.P[p][cd] = v;
        }
    }
}

// The ghost zones of the cell entries, each inverted as the zone pass's cell half inverts the
// interior (MeshUtoP and MeshApplyFloors over the entire block, kharma_step.cpp:233-236)
template <int MODE>
__global__ void __launch_bounds__(128) k_ctm_ghost_cell(const CtmZoneBlock* __restrict__ Z, const int* __restrict__ t6,
                                                        long long n)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int* t = t6 + 6 * e;
    const CtmZoneBlock& B = Z[__ldg(t)];
    int k, j, i;
    zone_kji(B.d, __ldg(t + 1), k, j, i);
    zone_body<8, double, MODE>(B.d, B.g, B.ph, B.a, i, j, k);
}

// One term of Olivares' operator (b_ct_functions.hpp, F<diff_face, diff_side, offset>): the
// difference across the coarse zone (2 fine zones along df) of the df-faces, upper half less lower
// half along ds, shifted by one zone along of (-1: none); zero for an inactive df
__device__ __forceinline__ double olv_term(const CtmBlock& D, const CtmDims& d, long long base, int df, int ds, int of,
                                           double area)
{
    if (df >= d.ndim) return 0.;
    const long long st[3] = {1, d.sj, d.sk};
    const long long o = (of >= 0 && of < d.ndim) ? st[of] : 0;
    const long long s = (ds < d.ndim) ? st[ds] : 0;
    const long long f2 = 2 * st[df];
    const double* F = D.Bf[df];
    return F[base + f2 + s + o] * area - F[base + s + o] * area - F[base + f2 + o] * area + F[base + o] * area;
}

// Ghost faces (entries {dst block, d, dst face, op, src block, src face, aux, phase})
__global__ void __launch_bounds__(128) k_ctm_face(const CtmBlock* __restrict__ B, CtmDims d, const int* __restrict__ t8,
                                                  long long begin, long long end)
{
    const long long e = begin + (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= end) return;
    const int* t = t8 + 8 * e;
    const CtmBlock& D = B[__ldg(t)];
    const int fd = __ldg(t + 1), op = __ldg(t + 3), aux = __ldg(t + 6);
    const long long x = __ldg(t + 2), y = __ldg(t + 5);
    const CtmBlock& S = B[__ldg(t + 4)];
    const long long st[3] = {1, d.sj, d.sk};
    // tangential active axes in ascending order
    int ta[2], nt = 0;
    for (int a = 0; a < d.ndim; ++a)
        if (a != fd) ta[nt++] = a;
    double v;
    if (op == 0) {
        v = S.Bf[fd][y];
    } else if (op == 1) {
        const double* f = S.Bf[fd] + y;
        if (nt == 2) v = ((f[0] + f[st[ta[0]]]) + (f[st[ta[1]]] + f[st[ta[0]] + st[ta[1]]])) * 0.25;
        else v = (f[0] + f[st[ta[0]]]) * 0.5;
    } else if (op == 2) {
        const double* q = S.Bf[fd];
        const double uc = q[y];
        v = uc;
        for (int n = 0; n < nt; ++n) {
            const int a = ta[n];
            const double sl = ctm_minmod(uc - q[y - st[a]], q[y + st[a]] - uc);
            v += ((aux >> a) & 1) ? 0.25 * sl : -0.25 * sl;
        }
    } else {
        // ProlongateInternalOlivares on a uniform grid: y is the lowest fine zone of the coarse zone,
        // aux the sub-face element; areas (Volume of a face element, FaceArea) are products of the
        // fine zone widths
        const int me = fd, nxt = (me + 1) % 3, thd = (me + 2) % 3;
        const double dx1 = D.dx[0], dx2 = D.dx[1], dx3 = D.dx[2];
        const double a[3] = {(dx2*dx2 - dx3*dx3) / (dx2*dx2 + dx3*dx3), (dx3*dx3 - dx1*dx1) / (dx3*dx3 + dx1*dx1),
                             (dx1*dx1 - dx2*dx2) / (dx1*dx1 + dx2*dx2)};
        const double cf[4][4] = {{3 + a[nxt], 1 - a[nxt], 3 - a[thd], 1 + a[thd]},
                                 {3 + a[nxt], 1 - a[nxt], 1 + a[thd], 3 - a[thd]},
                                 {1 - a[nxt], 3 + a[nxt], 3 - a[thd], 1 + a[thd]},
                                 {1 - a[nxt], 3 + a[nxt], 1 + a[thd], 3 - a[thd]}};
        const double area[3] = {dx2 * dx3, dx1 * dx3, dx1 * dx2};
        // the sub-face of element el lies (el % 2) zones up along nxt and (el / 2) along thd, which
        // makes the operator divergence-preserving (its coefficient rows pair each sub-face with the
        // halves it borders); the reference's offsets exchange the two, which leaves 3D fine zones
        // with a divergence (2D is the same either way)
        const int el = aux;
        int off[3] = {0, 0, 0};
        off[me] = 1;
        if (nxt < d.ndim) off[nxt] = el % 2;
        if (thd < d.ndim) off[thd] = el / 2;
        const long long tgt = y + off[0] * st[0] + off[1] * st[1] + off[2] * st[2];
        const long long dif = st[me];
        const double V = area[me];
        const double* F = D.Bf[me];
        const double ta_ = olv_term(D, d, y, nxt, me, -1, area[nxt]);
        const double tb_ = olv_term(D, d, y, nxt, me, thd, area[nxt]);
        const double tc_ = olv_term(D, d, y, thd, me, -1, area[thd]);
        const double td_ = olv_term(D, d, y, thd, me, nxt, area[thd]);
        v = (0.5 * (F[tgt - dif] * V + F[tgt + dif] * V) +
             1. / 16 * (cf[el][0] * ta_ + cf[el][1] * tb_ + cf[el][2] * tc_ + cf[el][3] * td_)) / V;
        D.Bf[me][tgt] = v;
        return;
    }
    D.Bf[fd][x] = v;
}

} // namespace khb

using namespace khb;

struct khb_ctmesh {
    std::vector<khb_ctx*> ctx;
    CtmDims d;
    CtmBlock* dev_blocks = nullptr;     // the contexts' flux and EMF scratch (khb_ctmesh_correct)
    // descriptors of each state an exchange has worked on, keyed by the first block's first
    // primitive pointer: uploaded on the first exchange of a state, reused after (no transfer, no
    // host wait, so that later calls can be captured in a CUDA graph)
    struct State {
        std::vector<CtmBlock> host;
        CtmBlock* dev;
    };
    std::vector<State> states;
    std::vector<CtmBlock> host_blocks;
    // the ghost cell pass's descriptors of each (seeds, U, Pout, Bf) set, cached the same way
    struct ZoneState {
        std::vector<CtmZoneBlock> host;
        CtmZoneBlock* dev;
    };
    std::vector<ZoneState> zstates;
    int* cell = nullptr;
    long long n_cell = 0;
    std::vector<long long> cell_ends;   // copies and restrictions, then one phase per destination level
    int* face = nullptr;
    long long n_face = 0;
    std::vector<long long> face_ends;
    int* flux = nullptr;
    long long n_flux = 0;
    int* emf = nullptr;
    long long n_emf = 0;
};

namespace {

int ctm_fail(int code, const std::string& msg) { return khb::set_error(code, msg); }

#define KHB_MCUDA(call)                                                                                        \
    do {                                                                                                       \
        cudaError_t e_ = (call);                                                                               \
        if (e_ != cudaSuccess) return ctm_fail(KHB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

int upload(int** dst, const int32_t* src, long long n, int width)
{
    if (n <= 0) return KHB_OK;
    KHB_MCUDA(cudaMalloc((void**)dst, sizeof(int32_t) * width * (size_t)n));
    KHB_MCUDA(cudaMemcpy(*dst, src, sizeof(int32_t) * width * (size_t)n, cudaMemcpyHostToDevice));
    return KHB_OK;
}

// The descriptors of one state (per block P, Bf; NULL for the scratch-only set) plus the contexts'
// flux and EMF scratch, uploaded synchronously into dev
int upload_blocks(khb_ctmesh* m, const khb_fields* P, const khb_fields* Bf, CtmBlock* dev)
{
    const int n = (int)m->ctx.size();
    for (int b = 0; b < n; ++b) {
        CtmBlock& c = m->host_blocks[b];
        std::memset(&c, 0, sizeof(c));
        const khb_ctx* x = m->ctx[b];
        if (P) for (int p = 0; p < 8; ++p) c.P[p] = P[b].v[p];
        if (Bf) for (int q = 0; q < 3; ++q) c.Bf[q] = Bf[b].v[q];
        for (int q = 0; q < 3; ++q) c.F[q] = (double*)x->F[q];
        c.emf = (double*)x->emf;
        c.dx[0] = x->ph.dx1; c.dx[1] = x->ph.dx2; c.dx[2] = x->ph.dx3;
    }
    KHB_MCUDA(cudaMemcpy(dev, m->host_blocks.data(), sizeof(CtmBlock) * n, cudaMemcpyHostToDevice));
    return KHB_OK;
}

// The device descriptors of state (P, Bf; Bf NULL: P only): uploaded on the first call with these
// pointers, found by comparing the host copies afterwards (no device access)
int state_blocks(khb_ctmesh* m, const khb_fields* P, const khb_fields* Bf, CtmBlock** out)
{
    const int n = (int)m->ctx.size();
    for (auto& s : m->states) {
        bool same = true;
        for (int b = 0; b < n && same; ++b) {
            for (int p = 0; p < 8; ++p) same &= s.host[b].P[p] == P[b].v[p];
            for (int q = 0; q < 3; ++q) same &= s.host[b].Bf[q] == (Bf ? Bf[b].v[q] : nullptr);
        }
        if (same) { *out = s.dev; return KHB_OK; }
    }
    khb_ctmesh::State s;
    s.dev = nullptr;
    KHB_MCUDA(cudaMalloc((void**)&s.dev, sizeof(CtmBlock) * n));
    int rc;
    if ((rc = upload_blocks(m, P, Bf, s.dev))) { cudaFree(s.dev); return rc; }
    s.host = m->host_blocks;
    m->states.push_back(s);
    *out = s.dev;
    return KHB_OK;
}

bool same_fields(const khb_fields& a, const khb_fields& b, int n)
{
    for (int p = 0; p < n; ++p) if (a.v[p] != b.v[p]) return false;
    return true;
}

// The ghost cell pass's descriptors of (P_s, U, P_out, Bf, flags): uploaded on first use, then reused
int zone_blocks(khb_ctmesh* m, const khb_fields* Ps, const khb_fields* U, const khb_fields* Pout, const khb_fields* Bf,
                int32_t* const* pflag, int32_t* const* fflag, CtmZoneBlock** out)
{
    const int n = (int)m->ctx.size();
    for (auto& s : m->zstates) {
        bool same = true;
        for (int b = 0; b < n && same; ++b) {
            const ZoneArgs<double>& a = s.host[b].a;
            same = same_fields(a.Ps, Ps[b], 8) && same_fields(a.Us, U[b], 8) && same_fields(a.Pout, Pout[b], 8) &&
                   a.Bf[0] == Bf[b].v[0] && a.Bf[1] == Bf[b].v[1] && a.Bf[2] == Bf[b].v[2] &&
                   a.pflag == pflag[b] && a.fflag == fflag[b];
        }
        if (same) { *out = s.dev; return KHB_OK; }
    }
    khb_ctmesh::ZoneState s;
    s.host.resize(n);
    for (int b = 0; b < n; ++b) {
        CtmZoneBlock& z = s.host[b];
        std::memset((void*)&z, 0, sizeof(z));
        const khb_ctx* c = m->ctx[b];
        z.d = c->d; z.g = c->g; z.ph = c->ph;
        z.a.Ps = Ps[b]; z.a.Us = U[b]; z.a.U0 = U[b]; z.a.Pout = Pout[b]; z.a.Uout = U[b];
        z.a.pflag = pflag[b]; z.a.fflag = fflag[b];
        for (int q = 0; q < 3; ++q) z.a.Bf[q] = Bf[b].v[q];
        z.a.mode = 0;
    }
    s.dev = nullptr;
    KHB_MCUDA(cudaMalloc((void**)&s.dev, sizeof(CtmZoneBlock) * n));
    cudaError_t e = cudaMemcpy(s.dev, s.host.data(), sizeof(CtmZoneBlock) * n, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { cudaFree(s.dev); return ctm_fail(KHB_ERR_CUDA, std::string("cudaMemcpy: ") + cudaGetErrorString(e)); }
    m->zstates.push_back(s);
    *out = s.dev;
    return KHB_OK;
}

} // namespace

extern "C" {

int khb_ctmesh_create(khb_ctx* const* ctxs, int nblocks, const int32_t* cell, int64_t n_cell,
                      const int64_t* cell_ends, int n_cell_phases, const int32_t* face, int64_t n_face,
                      const int64_t* face_ends, int n_face_phases, const int32_t* flux, int64_t n_flux,
                      const int32_t* emf, int64_t n_emf, khb_ctmesh** out)
{
    if (!ctxs || nblocks < 1 || !out) return ctm_fail(KHB_ERR_ARG, "khb_ctmesh_create: NULL argument");
    *out = nullptr;
    const khb_ctx* c0 = ctxs[0];
    for (int b = 0; b < nblocks; ++b) {
        const khb_ctx* c = ctxs[b];
        if (!c || !c->geom_set) return ctm_fail(KHB_ERR_ARG, "khb_ctmesh_create: a context without geometry");
        if (!c->ph.ct_scheme || c->nv != 8)
            return ctm_fail(KHB_ERR_UNSUPPORTED, "khb_ctmesh_create: B_CT MHD blocks (nvar 8) only");
        if (c->fp32) return ctm_fail(KHB_ERR_UNSUPPORTED, "khb_ctmesh_create: FP64 blocks only");
        if (c->d.n1 != c0->d.n1 || c->d.n2 != c0->d.n2 || c->d.n3 != c0->d.n3 || c->d.ndim != c0->d.ndim)
            return ctm_fail(KHB_ERR_ARG, "khb_ctmesh_create: blocks of one shape only");
        if (c->d.ndim < 2) return ctm_fail(KHB_ERR_UNSUPPORTED, "khb_ctmesh_create: 2D and 3D blocks only");
    }
    if ((n_cell && (!cell || !cell_ends || n_cell_phases < 1)) || (n_face && (!face || !face_ends || n_face_phases < 1)) ||
        (n_flux && !flux) || (n_emf && !emf))
        return ctm_fail(KHB_ERR_ARG, "khb_ctmesh_create: NULL table");
    const long long N = c0->d.N;
    auto bad_block = [&](int b) { return b < 0 || b >= nblocks; };
    for (long long e = 0; e < n_cell; ++e) {
        const int32_t* t = cell + 6 * e;
        if (bad_block(t[0]) || bad_block(t[3]) || t[2] < 0 || t[2] > 2 || t[1] < 0 || t[1] >= N || t[4] < 0 || t[4] >= N)
            return ctm_fail(KHB_ERR_ARG, "khb_ctmesh_create: bad ghost-zone entry");
    }
    for (long long e = 0; e < n_face; ++e) {
        const int32_t* t = face + 8 * e;
        if (bad_block(t[0]) || bad_block(t[4]) || t[1] < 0 || t[1] > 2 || t[3] < 0 || t[3] > 3 || t[2] < 0 || t[2] >= N ||
            t[5] < 0 || t[5] >= N)
            return ctm_fail(KHB_ERR_ARG, "khb_ctmesh_create: bad ghost-face entry");
    }
    for (long long e = 0; e < n_flux; ++e) {
        const int32_t* t = flux + 6 * e;
        if (bad_block(t[0]) || bad_block(t[3]) || t[1] < 1 || t[1] > 3 || t[2] < 0 || t[2] >= N || t[4] < 0 || t[4] >= N)
            return ctm_fail(KHB_ERR_ARG, "khb_ctmesh_create: bad flux entry");
    }
    for (long long e = 0; e < n_emf; ++e) {
        const int32_t* t = emf + 6 * e;
        if (bad_block(t[0]) || bad_block(t[3]) || t[1] < 0 || t[1] > 2 || t[2] < 0 || t[2] >= N || t[4] < 0 || t[4] >= N)
            return ctm_fail(KHB_ERR_ARG, "khb_ctmesh_create: bad EMF entry");
    }
    for (int p = 1; p < n_cell_phases; ++p)
        if (cell_ends[p] < cell_ends[p - 1]) return ctm_fail(KHB_ERR_ARG, "khb_ctmesh_create: cell phases out of order");
    for (int p = 1; p < n_face_phases; ++p)
        if (face_ends[p] < face_ends[p - 1]) return ctm_fail(KHB_ERR_ARG, "khb_ctmesh_create: face phases out of order");
    if ((n_cell_phases > 0 && cell_ends[n_cell_phases - 1] != n_cell) ||
        (n_face_phases > 0 && face_ends[n_face_phases - 1] != n_face))
        return ctm_fail(KHB_ERR_ARG, "khb_ctmesh_create: phase ends do not cover the tables");
    khb_ctmesh* m = new khb_ctmesh();
    m->ctx.assign(ctxs, ctxs + nblocks);
    m->d = CtmDims{c0->d.n1, c0->d.n2, c0->d.n3, c0->d.ndim, N, c0->d.sj, c0->d.sk};
    m->host_blocks.resize(nblocks);
    m->n_cell = n_cell; m->n_face = n_face; m->n_flux = n_flux; m->n_emf = n_emf;
    m->cell_ends.assign(cell_ends, cell_ends + (n_cell ? n_cell_phases : 0));
    m->face_ends.assign(face_ends, face_ends + (n_face ? n_face_phases : 0));
    int rc;
    cudaError_t e = cudaMalloc((void**)&m->dev_blocks, sizeof(CtmBlock) * nblocks);
    if (e != cudaSuccess) { delete m; return ctm_fail(KHB_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e)); }
    if ((rc = upload_blocks(m, nullptr, nullptr, m->dev_blocks)) || (rc = upload(&m->cell, cell, n_cell, 6)) ||
        (rc = upload(&m->face, face, n_face, 8)) ||
        (rc = upload(&m->flux, flux, n_flux, 6)) || (rc = upload(&m->emf, emf, n_emf, 6))) {
        cudaFree(m->dev_blocks); cudaFree(m->cell); cudaFree(m->face); cudaFree(m->flux); cudaFree(m->emf);
        delete m;
        return rc;
    }
    *out = m;
    return KHB_OK;
}

int khb_ctmesh_destroy(khb_ctmesh* m)
{
    if (!m) return KHB_OK;
    for (auto& s : m->states) cudaFree(s.dev);
    for (auto& s : m->zstates) cudaFree(s.dev);
    cudaFree(m->dev_blocks); cudaFree(m->cell); cudaFree(m->face); cudaFree(m->flux); cudaFree(m->emf);
    delete m;
    return KHB_OK;
}

int khb_ctmesh_correct(khb_ctmesh* m, void* stream)
{
    KHB_RANGE("khb_ctmesh_correct");
    if (!m) return ctm_fail(KHB_ERR_ARG, "khb_ctmesh_correct: NULL mesh");
    cudaStream_t st = (cudaStream_t)stream;
    if (m->n_flux) k_ctm_flux<<<blocks_for(m->n_flux, 128), 128, 0, st>>>(m->dev_blocks, m->d, m->flux, m->n_flux);
    if (m->n_emf) k_ctm_emf<<<blocks_for(m->n_emf, 128), 128, 0, st>>>(m->dev_blocks, m->d, m->emf, m->n_emf);
    KHB_MCUDA(cudaGetLastError());
    return KHB_OK;
}

int khb_ctmesh_exchange(khb_ctmesh* m, const khb_fields* P, const khb_fields* Bf, void* stream)
{
    KHB_RANGE("khb_ctmesh_exchange");
    if (!m || !P || !Bf) return ctm_fail(KHB_ERR_ARG, "khb_ctmesh_exchange: NULL argument");
    for (size_t b = 0; b < m->ctx.size(); ++b) {
        for (int p = 0; p < 8; ++p)
            if (!P[b].v[p]) return ctm_fail(KHB_ERR_ARG, "khb_ctmesh_exchange: NULL variable pointer");
        for (int q = 0; q < 3; ++q)
            if (!Bf[b].v[q]) return ctm_fail(KHB_ERR_ARG, "khb_ctmesh_exchange: NULL face field");
    }
    cudaStream_t st = (cudaStream_t)stream;
    int rc;
    CtmBlock* blocks = nullptr;
    if ((rc = state_blocks(m, P, Bf, &blocks))) return rc;
    long long lo = 0;
    for (long long hi : m->cell_ends) {
        if (hi > lo) k_ctm_cell<<<blocks_for(hi - lo, 128), 128, 0, st>>>(blocks, m->d, m->cell, lo, hi);
        lo = hi;
    }
    lo = 0;
    for (long long hi : m->face_ends) {
        if (hi > lo) k_ctm_face<<<blocks_for(hi - lo, 128), 128, 0, st>>>(blocks, m->d, m->face, lo, hi);
        lo = hi;
    }
    KHB_MCUDA(cudaGetLastError());
    return KHB_OK;
}

int khb_ctmesh_exchange_cons(khb_ctmesh* m, const khb_fields* P_s, const khb_fields* U, const khb_fields* P_out,
                             const khb_fields* Bf, int32_t* const* pflag, int32_t* const* fflag, void* stream)
{
    KHB_RANGE("khb_ctmesh_exchange_cons");
    if (!m || !P_s || !U || !P_out || !Bf || !pflag || !fflag)
        return ctm_fail(KHB_ERR_ARG, "khb_ctmesh_exchange_cons: NULL argument");
    for (size_t b = 0; b < m->ctx.size(); ++b) {
        for (int p = 0; p < 8; ++p)
            if (!P_s[b].v[p] || !U[b].v[p] || !P_out[b].v[p])
                return ctm_fail(KHB_ERR_ARG, "khb_ctmesh_exchange_cons: NULL variable pointer");
        for (int q = 0; q < 3; ++q)
            if (!Bf[b].v[q]) return ctm_fail(KHB_ERR_ARG, "khb_ctmesh_exchange_cons: NULL face field");
        if (!pflag[b] || !fflag[b]) return ctm_fail(KHB_ERR_ARG, "khb_ctmesh_exchange_cons: NULL flag array");
    }
    cudaStream_t st = (cudaStream_t)stream;
    int rc;
    CtmBlock *bu = nullptr, *bs = nullptr, *bf = nullptr;
    CtmZoneBlock* zb = nullptr;
    if ((rc = state_blocks(m, U, nullptr, &bu)) || (rc = state_blocks(m, P_s, nullptr, &bs)) ||
        (rc = state_blocks(m, P_out, Bf, &bf)) ||
        (rc = zone_blocks(m, P_s, U, P_out, Bf, pflag, fflag, &zb)))
        return rc;
    long long lo = 0;
    for (long long hi : m->cell_ends) {
        if (hi > lo) k_ctm_cell_cons<<<blocks_for(hi - lo, 128), 128, 0, st>>>(bu, bs, m->d, m->cell, lo, hi);
        lo = hi;
    }
    lo = 0;
    for (long long hi : m->face_ends) {
        if (hi > lo) k_ctm_face<<<blocks_for(hi - lo, 128), 128, 0, st>>>(bf, m->d, m->face, lo, hi);
        lo = hi;
    }
    if (m->n_cell) {
        constexpr int C = M_UTOP | M_FLOORS | M_PTOU | M_BCT | M_GHOSTB;
        if (m->ctx[0]->ph.inverter == KHB_INVERTER_KASTAUN)
            k_ctm_ghost_cell<C | M_KASTAUN><<<blocks_for(m->n_cell, 128), 128, 0, st>>>(zb, m->cell, m->n_cell);
        else
            k_ctm_ghost_cell<C><<<blocks_for(m->n_cell, 128), 128, 0, st>>>(zb, m->cell, m->n_cell);
    }
    KHB_MCUDA(cudaGetLastError());
    return KHB_OK;
}

} // extern "C"

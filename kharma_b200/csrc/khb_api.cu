// khb_api.cu -- host side of libkhb: context, scratch, geometry upload, launches, C ABI.
#include "khb_types.cuh"

#include <cstdio>
#include <cstring>
#include <cmath>
#include <string>
#include <vector>

using namespace khb;

#include "khb_internal.hpp"

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg)
{
    g_err = msg;
    return code;
}

#define KHB_CUDA(call)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return fail(KHB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define KHB_LAUNCHED(ctx)                                                                \
    do {                                                                                 \
        (ctx)->launches++;                                                               \
        cudaError_t e_ = cudaGetLastError();                                             \
        if (e_ != cudaSuccess) return fail(KHB_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e_)); \
    } while (0)

inline cudaStream_t S(void* s) { return (cudaStream_t)s; }

int check_fields(const khb_ctx* ctx, const khb_fields* f, const char* name)
{
    if (!f) return fail(KHB_ERR_ARG, std::string(name) + " is NULL");
    for (int p = 0; p < ctx->nv; ++p)
        if (!f->v[p]) return fail(KHB_ERR_ARG, std::string(name) + " has a NULL variable pointer");
    return KHB_OK;
}

// ------------------------------------------------------------------ fluxes
// k_lo <= k_hi: only the faces whose x3 index lies in [k_lo, k_hi]
int launch_flux(khb_ctx* ctx, int dir, const khb_fields& P, cudaStream_t st, int k_lo = 0, int k_hi = -1)
{
    const Dims& d = ctx->d;
    int lo[3], cnt[3];
    const int s[3] = {d.is, d.js, d.ks}, e[3] = {d.ie, d.je, d.ke};
    for (int a = 0; a < 3; ++a) {
        const bool active = (a + 1) <= d.ndim;
        int hi;
        if (a + 1 == dir) { lo[a] = s[a]; hi = e[a] + 1; }
        else if (active) { lo[a] = s[a] - 1; hi = e[a] + 1; }
        else { lo[a] = s[a]; hi = e[a]; }
        if (a == 2 && k_lo <= k_hi) {
            lo[a] = lo[a] > k_lo ? lo[a] : k_lo;
            hi = hi < k_hi ? hi : k_hi;
            if (hi < lo[a]) return KHB_OK;
        }
        cnt[a] = hi - lo[a] + 1;
    }
    if (ctx->fp32)
        Launch<float>::flux(ctx->cfg.recon, ctx->nv, dir, d, ctx->g, ctx->ph, P, (float*)ctx->F[dir-1],
                            (float*)ctx->ctop[dir-1], lo, cnt, st);
    else
        Launch<double>::flux(ctx->cfg.recon, ctx->nv, dir, d, ctx->g, ctx->ph, P, (double*)ctx->F[dir-1],
                             (double*)ctx->ctop[dir-1], lo, cnt, st);
    KHB_LAUNCHED(ctx);
    return KHB_OK;
}

template <typename FT>
int launch_fix_flux_t(khb_ctx* ctx, const Phys& ph, cudaStream_t st, FT* F1 = nullptr, FT* F2 = nullptr,
                      FT* F3 = nullptr, int nv = 0)
{
    // default: the context's flux arrays; the EMHD stage passes its 10-slot arrays (nv = 10)
    const Dims& d = ctx->d;
    if (!F1) { F1 = (FT*)ctx->F[0]; F2 = (FT*)ctx->F[1]; F3 = (FT*)ctx->F[2]; nv = ctx->nv; }
    if (d.ndim >= 2 && (ph.zero_polar_flux || (nv > 5 && ph.fix_polar_flux))) {
        for (int face = 2; face <= 3; ++face) {
            if (!phys_face(d.bc[face])) continue;
            Launch<FT>::fix_flux_x2(nv, d, ph, F1, F2, F3, face == 2, st);
            KHB_LAUNCHED(ctx);
        }
    }
    if (ph.check_inflow_in && phys_face(d.bc[0])) {
        Launch<FT>::fix_flux_x1(d, F1, 1, st);
        KHB_LAUNCHED(ctx);
    }
    if (ph.check_inflow_out && phys_face(d.bc[1])) {
        Launch<FT>::fix_flux_x1(d, F1, 0, st);
        KHB_LAUNCHED(ctx);
    }
    return KHB_OK;
}

// First-order flux correction of a stage (stage weights from the rk2 tables)
template <typename FT>
void launch_fofc_t(khb_ctx* ctx, int stage, double dt, const khb_fields& Ps, const khb_fields& Us,
                   const khb_fields& U0, cudaStream_t st)
{
    const int s = stage - 1;
    FT* F[3] = {(FT*)ctx->F[0], (FT*)ctx->F[1], (FT*)ctx->F[2]};
    FT* ct[3] = {(FT*)ctx->ctop[0], (FT*)ctx->ctop[1], (FT*)ctx->ctop[2]};
    Launch<FT>::fofc(ctx->nv, ctx->d, ctx->g, ctx->ph, Ps, Us, U0, F, ct, kRkGam0[s], kRkGam1[s], kRkBeta[s] * dt,
                     ctx->dt_active, kRkBeta[s], ctx->fofc_flag, st);
}
int launch_fofc(khb_ctx* ctx, int stage, double dt, const khb_fields& Ps, const khb_fields& Us,
                const khb_fields& U0, cudaStream_t st)
{
    if (!ctx->ph.fofc) return KHB_OK;
    if (ctx->fp32) launch_fofc_t<float>(ctx, stage, dt, Ps, Us, U0, st);
    else launch_fofc_t<double>(ctx, stage, dt, Ps, Us, U0, st);
    KHB_LAUNCHED(ctx);
    return KHB_OK;
}

int launch_fix_flux(khb_ctx* ctx, const Phys& ph, cudaStream_t st)
{
    return ctx->fp32 ? launch_fix_flux_t<float>(ctx, ph, st) : launch_fix_flux_t<double>(ctx, ph, st);
}

// ------------------------------------------------------------------ zone pass
struct ZoneCall {
    khb_fields Ps, Us, U0, Pout, Uout;
    int32_t* pflag;
    int32_t* fflag;
    double g0, g1, bdt;
    const double* dt_dev;       // device timestep (then bdt = beta * dt_dev[0])
    double beta;
    int mode;
};

template <typename FT>
void launch_zone_t(khb_ctx* ctx, const ZoneCall& zc, cudaStream_t st)
{
    ZoneArgs<FT> a;
    a.Ps = zc.Ps; a.Us = zc.Us; a.U0 = zc.U0; a.Pout = zc.Pout; a.Uout = zc.Uout;
    for (int x = 0; x < 3; ++x) { a.F[x] = (const FT*)ctx->F[x]; a.ctop[x] = (const FT*)ctx->ctop[x]; }
    a.pflag = zc.pflag; a.fflag = zc.fflag;
    a.g0 = zc.g0; a.g1 = zc.g1; a.bdt = zc.bdt;
    a.dt_dev = zc.dt_dev; a.beta = zc.beta;
    a.ndt_word = ctx->words;
    a.fail_count = ctx->fail_count;
    a.fail_list = ctx->fail_list;
    a.mode = zc.mode;
    for (int x = 0; x < 3; ++x) a.Bf[x] = ctx->ct_active ? ctx->ct_bf[x] : nullptr;
    Launch<FT>::zone(ctx->nv, ctx->d, ctx->g, ctx->ph, a, st);
}

int launch_zone(khb_ctx* ctx, const ZoneCall& zc_in, cudaStream_t st)
{
    ZoneCall zc = zc_in;
    if ((zc.mode & M_UTOP) && ctx->ph.inverter == KHB_INVERTER_KASTAUN) zc.mode |= M_KASTAUN;
    if (ctx->ct_active && (zc.mode & (M_UPDATE | M_UTOP))) zc.mode |= M_BCT;
    if (ctx->fp32) launch_zone_t<float>(ctx, zc, st); else launch_zone_t<double>(ctx, zc, st);
    KHB_LAUNCHED(ctx);
    return KHB_OK;
}

// ------------------------------------------------------------------ fixups, boundaries
int launch_fixup(khb_ctx* ctx, const khb_fields& P, const khb_fields& U, const int32_t* pflag, cudaStream_t st)
{
    if (!ctx->ph.fix_avg && !ctx->ph.fix_atmo) return KHB_OK;
    LaunchCommon::fixup(ctx->nv, ctx->d, ctx->g, ctx->ph, P, U, pflag, ctx->fail_count, ctx->fail_list, st);
    KHB_LAUNCHED(ctx);
    return KHB_OK;
}

// The interior zones of a block to / from a packed [nv][nx3][nx2][nx1] buffer (unpack: buffer -> P)
__global__ void k_interior_pack(Dims d, khb_fields P, int nv, double* buf, int unpack)
{
    const long long nint = (long long)d.nx1 * d.nx2 * d.nx3;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nint) return;
    const int i = (int)(t % d.nx1);
    const long long r = t / d.nx1;
    const int j = (int)(r % d.nx2), k = (int)(r / d.nx2);
    const long long c = ((long long)(k + d.ks) * d.n2 + (j + d.js)) * d.n1 + (i + d.is);
    for (int p = 0; p < nv; ++p) {
        if (unpack) P.v[p][c] = buf[p * nint + t];
        else buf[p * nint + t] = P.v[p][c];
    }
}

// Bf: a B_CT block's faces; with physical faces their ghost layers are filled first and the ghost
// zones of the physical directions take B from them
// nv_state: 10 for the EMHD state (its scalar slots q~, dP~ copied as the density is), else the
// context's nvar
int launch_boundaries(khb_ctx* ctx, const khb_fields& P, const khb_fields& U, cudaStream_t st,
                      const khb_fields* Bf = nullptr, int nv_state = 0)
{
    const Dims& d = ctx->d;
    const int nv = nv_state ? nv_state : ctx->nv;
    const int nv_ptou = (nv == 10) ? 8 : nv;     // ghost B_P and (GRMHD) U; the EMHD U is formed later
    // the transverse range of a face's pass: the interior, or every zone along a direction with an
    // exchange face (a block of a mesh: its ghost rows hold the neighbours' zones, and Parthenon
    // applies the condition over them after the exchange)
    const bool xj = d.ndim >= 2 && (d.bc[2] == KHB_BC_EXCHANGE || d.bc[3] == KHB_BC_EXCHANGE);
    const bool xk = d.ndim >= 3 && (d.bc[4] == KHB_BC_EXCHANGE || d.bc[5] == KHB_BC_EXCHANGE);
    const int lo_k = xk ? 0 : d.ks;
    const int cnt_k = xk ? d.n3 : d.ke - d.ks + 1;
    // a block of a mesh: B and U = U(P) over the boundary domains of its physical faces only
    int pfaces = 0;
    bool exch = false;
    for (int f = 0; f < 2 * d.ndim; ++f) {
        if (phys_face(d.bc[f])) pfaces |= 1 << f;
        exch = exch || d.bc[f] == KHB_BC_EXCHANGE;
    }
    if (!exch) pfaces = 0;
    bool physical = false;
    int ct_mask = 0;
    if (Bf) {
        // a direction with a physical face on either side (a block of a mesh may have one on one side only)
        if (phys_face(d.bc[0]) || phys_face(d.bc[1])) ct_mask |= 1;
        if (d.ndim >= 2 && (phys_face(d.bc[2]) || phys_face(d.bc[3]))) ct_mask |= 2;
        if (d.ndim >= 3 && (phys_face(d.bc[4]) || phys_face(d.bc[5]))) ct_mask |= 4;
        if (!ct_mask) Bf = nullptr;
        // a block of a mesh: every zone past a physical face takes B from its faces, also where it lies
        // in the ghost rows the exchange filled (B_CT::BlockUtoP over the face's boundary domain)
        else if (exch) ct_mask = 7;
    }
    if (Bf) {
        const int rc = khb::ct_face_boundaries(ctx, *Bf, st);
        if (rc) return rc;
    }
    // X1 faces over the interior j range, then X2 faces over all i, then the corner fix
    for (int face = 0; face < 2; ++face) {
        if (!phys_face(d.bc[face])) continue;
        physical = true;
        LaunchCommon::bc(nv, d, ctx->g, ctx->ph, P, U, face, xj ? 0 : d.js, xj ? d.n2 : d.je - d.js + 1, lo_k, cnt_k, st);
        KHB_LAUNCHED(ctx);
    }
    if (d.ndim >= 2) {
        for (int face = 2; face < 4; ++face) {
            if (!phys_face(d.bc[face])) continue;
            physical = true;
            LaunchCommon::bc(nv, d, ctx->g, ctx->ph, P, U, face, 0, d.n1, lo_k, cnt_k, st);
            KHB_LAUNCHED(ctx);
        }
        if (ctx->cfg.fix_corner_inner && phys_face(d.bc[0]) && phys_face(d.bc[3])) {
            LaunchCommon::bc(nv, d, ctx->g, ctx->ph, P, U, 0, 0, d.n2, lo_k, cnt_k, st);
            KHB_LAUNCHED(ctx);
        }
    }
    if (physical) {
        LaunchCommon::ghost_ptou(nv_ptou, d, ctx->g, ctx->ph, P, U, st, Bf, ct_mask, 0, pfaces);
        KHB_LAUNCHED(ctx);
        if (xk) {
            // the X1/X2 passes also filled the X3 ghost planes' corners
            LaunchCommon::ghost_ptou(nv_ptou, d, ctx->g, ctx->ph, P, U, st, Bf, ct_mask, 3, pfaces);
            KHB_LAUNCHED(ctx);
        }
    }
    // X3 faces last (Parthenon's face order), over the whole (j, i) plane: their ghost planes copy
    // the boundary planes with the X1/X2 ghost zones already filled; then B_P and U = U(P) there
    int kplanes = 0;
    if (d.ndim >= 3) {
        for (int face = 4; face < 6; ++face) {
            if (!phys_face(d.bc[face])) continue;
            kplanes |= 1 << (face - 4);
            LaunchCommon::bc(nv, d, ctx->g, ctx->ph, P, U, face, 0, d.n1 * d.n2, 0, 1, st);
            KHB_LAUNCHED(ctx);
        }
        if (kplanes) {
            LaunchCommon::ghost_ptou(nv_ptou, d, ctx->g, ctx->ph, P, U, st, Bf, ct_mask, kplanes, pfaces);
            KHB_LAUNCHED(ctx);
        }
    }
    int pmask = 0;
    if (d.bc[0] == KHB_BC_PERIODIC) pmask |= 1;
    if (d.ndim >= 2 && d.bc[2] == KHB_BC_PERIODIC) pmask |= 2;
    if (d.ndim >= 3 && d.bc[4] == KHB_BC_PERIODIC) pmask |= 4;
    if (pmask) {
        LaunchCommon::periodic(nv, d, P, U, pmask, st);
        KHB_LAUNCHED(ctx);
    }
    return KHB_OK;
}

// The launches launch_boundaries(ctx, P, U, st) makes (no face field, the context's nvar), appended as
// tasks to the phase each belongs to (phases[0..BOUND_PHASES-1], run in that order): a batch runs each
// phase of all its blocks in one k_bound_tasks launch, with the same work per zone
void boundary_tasks_of(khb_ctx* ctx, const khb_fields& P, const khb_fields& U, std::vector<BoundTask>* phases)
{
    const Dims& d = ctx->d;
    const bool xj = d.ndim >= 2 && (d.bc[2] == KHB_BC_EXCHANGE || d.bc[3] == KHB_BC_EXCHANGE);
    const bool xk = d.ndim >= 3 && (d.bc[4] == KHB_BC_EXCHANGE || d.bc[5] == KHB_BC_EXCHANGE);
    const int lo_k = xk ? 0 : d.ks;
    const int cnt_k = xk ? d.n3 : d.ke - d.ks + 1;
    int pfaces = 0;
    bool exch = false;
    for (int f = 0; f < 2 * d.ndim; ++f) {
        if (phys_face(d.bc[f])) pfaces |= 1 << f;
        exch = exch || d.bc[f] == KHB_BC_EXCHANGE;
    }
    if (!exch) pfaces = 0;
    BoundTask base;
    std::memset((void*)&base, 0, sizeof(base));
    base.d = d; base.g = ctx->g; base.ph = ctx->ph; base.P = P; base.U = U;
    auto bc = [&](int phase, int face, int lo_a, int cnt_a, int lk, int ck) {
        BoundTask t = base;
        t.kind = BOUND_BC; t.face = face; t.lo_a = lo_a; t.cnt_a = cnt_a; t.lo_k = lk; t.cnt_k = ck;
        const int bdir = face / 2 + 1;
        const int ng = (bdir == 1) ? d.is : ((bdir == 2) ? d.js : d.ks);
        t.count = (long long)ng * cnt_a * ck;
        if (t.count > 0) phases[phase].push_back(t);
    };
    auto ghost = [&](int phase, int kplanes) {
        BoundTask t = base;
        t.kind = BOUND_GHOST_PTOU; t.kplanes = kplanes; t.pfaces = pfaces;
        const long long plane = (long long)d.n1 * d.n2;
        const long long per = plane - (long long)(d.ie - d.is + 1) * (d.je - d.js + 1);
        t.count = kplanes ? plane * (((kplanes & 1) ? d.ks : 0) + ((kplanes & 2) ? d.n3 - 1 - d.ke : 0))
                          : per * (d.ke - d.ks + 1);
        if (t.count > 0) phases[phase].push_back(t);
    };
    bool physical = false;
    for (int face = 0; face < 2; ++face) {
        if (!phys_face(d.bc[face])) continue;
        physical = true;
        bc(0, face, xj ? 0 : d.js, xj ? d.n2 : d.je - d.js + 1, lo_k, cnt_k);
    }
    if (d.ndim >= 2) {
        for (int face = 2; face < 4; ++face) {
            if (!phys_face(d.bc[face])) continue;
            physical = true;
            bc(1, face, 0, d.n1, lo_k, cnt_k);
        }
        if (ctx->cfg.fix_corner_inner && phys_face(d.bc[0]) && phys_face(d.bc[3])) bc(2, 0, 0, d.n2, lo_k, cnt_k);
    }
    if (physical) {
        ghost(3, 0);
        if (xk) ghost(4, 3);
    }
    int kplanes = 0;
    if (d.ndim >= 3) {
        for (int face = 4; face < 6; ++face) {
            if (!phys_face(d.bc[face])) continue;
            kplanes |= 1 << (face - 4);
            bc(5, face, 0, d.n1 * d.n2, 0, 1);
        }
        if (kplanes) ghost(6, kplanes);
    }
    int pmask = 0;
    if (d.bc[0] == KHB_BC_PERIODIC) pmask |= 1;
    if (d.ndim >= 2 && d.bc[2] == KHB_BC_PERIODIC) pmask |= 2;
    if (d.ndim >= 3 && d.bc[4] == KHB_BC_PERIODIC) pmask |= 4;
    if (pmask) {
        BoundTask t = base;
        t.kind = BOUND_PERIODIC; t.pmask = pmask;
        t.count = d.N - (long long)(d.ie - d.is + 1) * (d.je - d.js + 1) * (d.ke - d.ks + 1);
        if (t.count > 0) phases[7].push_back(t);
    }
}

size_t ft_size(const khb_ctx* ctx) { return ctx->fp32 ? sizeof(float) : sizeof(double); }

bool has_exchange_face(const Dims& d)
{
    for (int f = 0; f < 2 * d.ndim; ++f)
        if (d.bc[f] == KHB_BC_EXCHANGE) return true;
    return false;
}

// Ghost shell of the stage input carried to the output (blocks with exchange faces only), before
// the zone pass so that the fixups see the neighbour values across exchange faces
int launch_ghost_copy(khb_ctx* ctx, const khb_fields& Ps, const khb_fields& Us, const khb_fields& Pout,
                      const khb_fields& Uout, cudaStream_t st)
{
    if (!has_exchange_face(ctx->d) || (Ps.v[0] == Pout.v[0] && Us.v[0] == Uout.v[0])) return KHB_OK;
    LaunchCommon::ghost_copy(ctx->nv, ctx->d, Ps, Us, Pout, Uout, st);
    KHB_LAUNCHED(ctx);
    return KHB_OK;
}


int zone_pass(khb_ctx* ctx, int stage, double dt, const khb_fields& Ps, const khb_fields& Us,
              const khb_fields& U0, const khb_fields& Pout, const khb_fields& Uout,
              int32_t* pflag, int32_t* fflag, cudaStream_t st)
{
    const int s = stage - 1;
    // failed-zone counter, and on the last stage the timestep minimum (taken over bit patterns,
    // from the pattern of DBL_MAX), reset on the device so that the stage can be graph-captured
    LaunchCommon::stage_reset(ctx->fail_count, stage == 2 ? ctx->words : nullptr, st);
    KHB_LAUNCHED(ctx);
    ZoneCall zc;
    zc.Ps = Ps; zc.Us = Us; zc.U0 = U0; zc.Pout = Pout; zc.Uout = Uout;
    zc.pflag = pflag; zc.fflag = fflag;
    zc.g0 = kRkGam0[s]; zc.g1 = kRkGam1[s]; zc.bdt = kRkBeta[s] * dt;
    zc.dt_dev = ctx->dt_active; zc.beta = kRkBeta[s];
    const int dtm = (stage == 2) ? M_DT : 0;
    // the adjoint's recompute keeps the primitives between the inversion and the floors (the split
    // passes are bitwise the fused one)
    const bool snap = ctx->prefloor_dst && ctx->ph.floors_on;
    if (!ctx->zone_split && !snap) {
        zc.mode = M_ZONE_FUSED | dtm;
        return launch_zone(ctx, zc, st);
    }
    int rc;
    zc.mode = M_UPDATE;
    if ((rc = launch_zone(ctx, zc, st))) return rc;
    zc.Us = Uout;          // the updated conserved state is the inversion's input
    if (ctx->zone_split == 1 && !snap) {
        zc.mode = M_ZONE_CELL | dtm;
        return launch_zone(ctx, zc, st);
    }
    zc.mode = M_UTOP;
    if ((rc = launch_zone(ctx, zc, st))) return rc;
    if (snap)
        for (int p = 0; p < 5; ++p)
            KHB_CUDA(cudaMemcpyAsync(ctx->prefloor_dst + (size_t)p * ctx->d.N, Pout.v[p], sizeof(double) * (size_t)ctx->d.N,
                                     cudaMemcpyDeviceToDevice, st));
    zc.Ps = Pout;          // floors start from the inverted primitives and their flags
    zc.mode = M_ZONE_FLOORS | dtm;
    return launch_zone(ctx, zc, st);
}

int do_stage(khb_ctx* ctx, int stage, double dt, const khb_fields& Ps, const khb_fields& Us,
             const khb_fields& U0, const khb_fields& Pout, const khb_fields& Uout,
             int32_t* pflag, int32_t* fflag, cudaStream_t st)
{
    int rc;
    for (int dir = 1; dir <= ctx->d.ndim; ++dir)
        if ((rc = launch_flux(ctx, dir, Ps, st))) return rc;
    if ((rc = launch_fofc(ctx, stage, dt, Ps, Us, U0, st))) return rc;
    if ((rc = launch_fix_flux(ctx, ctx->ph, st))) return rc;
    if ((rc = launch_ghost_copy(ctx, Ps, Us, Pout, Uout, st))) return rc;
    if ((rc = zone_pass(ctx, stage, dt, Ps, Us, U0, Pout, Uout, pflag, fflag, st))) return rc;
    if ((rc = launch_fixup(ctx, Pout, Uout, pflag, st))) return rc;
    return launch_boundaries(ctx, Pout, Uout, st);
}

// One stage of a B_CT block: fluxes and their fixes, edge EMFs and the face update, then the zone pass
// with the zone B from the new faces (M_BCT), fixups and ghost zones
// The first half of a B_CT stage: face fluxes, their fixes and the edge EMFs, in context scratch
int ct_stage_fluxes(khb_ctx* ctx, const khb_fields& Ps, cudaStream_t st)
{
    int rc;
    for (int dir = 1; dir <= ctx->d.ndim; ++dir)
        if ((rc = launch_flux(ctx, dir, Ps, st))) return rc;
    if ((rc = launch_fix_flux(ctx, ctx->ph, st))) return rc;
    return khb::ct_emf(ctx, Ps, st);
}

// The second half: the face update from the EMFs, the zone pass, fixups and ghost zones
int ct_stage_update(khb_ctx* ctx, int stage, double dt, const khb_fields& Ps, const khb_fields& Us,
                    const khb_fields& U0, const khb_fields& Bs, const khb_fields& B0, const khb_fields& Pout,
                    const khb_fields& Uout, const khb_fields& Bout, int32_t* pflag, int32_t* fflag, cudaStream_t st)
{
    int rc;
    if ((rc = khb::ct_face_update(ctx, stage, dt, Bs, B0, Bout, st))) return rc;
    if ((rc = launch_ghost_copy(ctx, Ps, Us, Pout, Uout, st))) return rc;
    for (int x = 0; x < 3; ++x) ctx->ct_bf[x] = Bout.v[x];
    ctx->ct_active = true;
    rc = zone_pass(ctx, stage, dt, Ps, Us, U0, Pout, Uout, pflag, fflag, st);
    ctx->ct_active = false;
    if (rc) return rc;
    if ((rc = launch_fixup(ctx, Pout, Uout, pflag, st))) return rc;
    // a block of a mesh takes its physical faces after the exchange (khb_ct_boundaries), so that the
    // faces it sends are those of the update, as in the reference's sync before its domain conditions
    if (has_exchange_face(ctx->d)) return KHB_OK;
    return launch_boundaries(ctx, Pout, Uout, st, &Bout);
}

// ct_stage_update in two parts around the kharma driver's exchange of a mesh: part 1 the face update,
// the ghost-shell copy and the update half of the zone pass (U_out: the updated conserved state, its
// B from the new faces); part 2 the cell half (inversion from P_s, floors, U = U(P)) and the fixups
int ct_stage_update_part(khb_ctx* ctx, int part, int stage, double dt, const khb_fields& Ps, const khb_fields& Us,
                         const khb_fields& U0, const khb_fields& Bs, const khb_fields& B0, const khb_fields& Pout,
                         const khb_fields& Uout, const khb_fields& Bout, int32_t* pflag, int32_t* fflag, cudaStream_t st)
{
    const int s = stage - 1;
    int rc;
    ZoneCall zc;
    zc.Ps = Ps; zc.Us = Us; zc.U0 = U0; zc.Pout = Pout; zc.Uout = Uout;
    zc.pflag = pflag; zc.fflag = fflag;
    zc.g0 = kRkGam0[s]; zc.g1 = kRkGam1[s]; zc.bdt = kRkBeta[s] * dt;
    zc.dt_dev = ctx->dt_active; zc.beta = kRkBeta[s];
    for (int x = 0; x < 3; ++x) ctx->ct_bf[x] = Bout.v[x];
    if (part == 1) {
        if ((rc = khb::ct_face_update(ctx, stage, dt, Bs, B0, Bout, st))) return rc;
        if ((rc = launch_ghost_copy(ctx, Ps, Us, Pout, Uout, st))) return rc;
        LaunchCommon::stage_reset(ctx->fail_count, stage == 2 ? ctx->words : nullptr, st);
        KHB_LAUNCHED(ctx);
        zc.mode = M_UPDATE;
    } else {
        zc.Us = Uout;          // the updated conserved state is the inversion's input
        zc.mode = M_ZONE_CELL | ((stage == 2) ? M_DT : 0);
    }
    ctx->ct_active = true;
    rc = launch_zone(ctx, zc, st);
    ctx->ct_active = false;
    if (rc || part == 1) return rc;
    if ((rc = launch_fixup(ctx, Pout, Uout, pflag, st))) return rc;
    if (has_exchange_face(ctx->d)) return KHB_OK;
    return launch_boundaries(ctx, Pout, Uout, st, &Bout);
}

int do_ct_stage(khb_ctx* ctx, int stage, double dt, const khb_fields& Ps, const khb_fields& Us,
                const khb_fields& U0, const khb_fields& Bs, const khb_fields& B0, const khb_fields& Pout,
                const khb_fields& Uout, const khb_fields& Bout, int32_t* pflag, int32_t* fflag, cudaStream_t st)
{
    int rc;
    if ((rc = ct_stage_fluxes(ctx, Ps, st))) return rc;
    return ct_stage_update(ctx, stage, dt, Ps, Us, U0, Bs, B0, Pout, Uout, Bout, pflag, fflag, st);
}

} // namespace

int khb::set_error(int code, const std::string& msg) { return fail(code, msg); }
int khb::ctx_fix_flux(khb_ctx* ctx, cudaStream_t st) { return launch_fix_flux(ctx, ctx->ph, st); }
void khb::boundary_tasks(khb_ctx* ctx, const khb_fields& P, const khb_fields& U, std::vector<BoundTask>* phases)
{
    boundary_tasks_of(ctx, P, U, phases);
}

int khb::ctx_boundaries(khb_ctx* ctx, const khb_fields& P, const khb_fields& U, cudaStream_t st)
{
    return launch_boundaries(ctx, P, U, st);
}

int khb::derive_block(const khb_config* cfg, Dims& d, Phys& ph, const char** why)
{
    if (cfg->nvar != 5 && cfg->nvar != 8) { *why = "nvar must be 5 or 8"; return KHB_ERR_UNSUPPORTED; }
    if (cfg->recon < 0 || cfg->recon > KHB_RECON_MP5) { *why = "unknown reconstruction"; return KHB_ERR_UNSUPPORTED; }
    if (cfg->ng < 3) { *why = "need at least 3 ghost zones"; return KHB_ERR_ARG; }
    if (cfg->nx1 < 1 || cfg->nx2 < 1 || cfg->nx3 < 1) { *why = "bad block size"; return KHB_ERR_ARG; }
    if (cfg->nx2 == 1 && cfg->nx3 > 1) { *why = "x3 active with x2 inactive"; return KHB_ERR_UNSUPPORTED; }
    if (cfg->precision != KHB_PREC_FP64 && cfg->precision != KHB_PREC_FP32_FLUX) {
        *why = "unknown precision";
        return KHB_ERR_UNSUPPORTED;
    }
    for (int x = 0; x < 6; ++x) {
        if (cfg->bc[x] < KHB_BC_PERIODIC || cfg->bc[x] > KHB_BC_TRANSMITTING) { *why = "unknown boundary type"; return KHB_ERR_ARG; }
        if (cfg->bc[x] == KHB_BC_TRANSMITTING) {
            // one_block_transmit.cpp:74-75 and boundaries.cpp:297-301
            if (x != 2 && x != 3) { *why = "transmitting boundaries are X2 faces"; return KHB_ERR_UNSUPPORTED; }
            if (cfg->nx3 < 2 || cfg->nx3 % 2 || cfg->bc[4] != KHB_BC_PERIODIC) {
                *why = "transmitting polar boundaries need a 3D block over all of a periodic x3 (even nx3)";
                return KHB_ERR_UNSUPPORTED;
            }
        }
        const bool active = x < 2 || (x < 4 ? cfg->nx2 > 1 : cfg->nx3 > 1);
        if (cfg->bc[x] == KHB_BC_EXCHANGE && !active) {
            *why = "exchange boundaries are supported on faces of active directions only";
            return KHB_ERR_UNSUPPORTED;
        }
    }
    for (int x = 0; x < 6; x += 2)
        if ((cfg->bc[x] == KHB_BC_PERIODIC) != (cfg->bc[x + 1] == KHB_BC_PERIODIC)) {
            *why = "periodic on one face of a direction only";
            return KHB_ERR_ARG;
        }
    std::memset(&d, 0, sizeof(d));
    std::memset(&ph, 0, sizeof(ph));
    d.nx1 = cfg->nx1; d.nx2 = cfg->nx2; d.nx3 = cfg->nx3;
    d.ndim = 1 + (cfg->nx2 > 1) + (cfg->nx3 > 1);
    d.n1 = cfg->nx1 + 2*cfg->ng;
    d.n2 = (cfg->nx2 > 1) ? cfg->nx2 + 2*cfg->ng : 1;
    d.n3 = (cfg->nx3 > 1) ? cfg->nx3 + 2*cfg->ng : 1;
    d.is = cfg->ng; d.ie = cfg->ng + cfg->nx1 - 1;
    d.js = (cfg->nx2 > 1) ? cfg->ng : 0; d.je = d.js + cfg->nx2 - 1;
    d.ks = (cfg->nx3 > 1) ? cfg->ng : 0; d.ke = d.ks + cfg->nx3 - 1;
    d.N = (long long)d.n1*d.n2*d.n3;
    d.sj = d.n1; d.sk = (long long)d.n1*d.n2;
    for (int x = 0; x < 6; ++x) d.bc[x] = cfg->bc[x];
    ph.gam = cfg->gam;
    ph.riemann = cfg->riemann;
    ph.recon_floors = cfg->recon_floors && cfg->floors_on;
    ph.spherical = cfg->spherical;
    ph.cart_minkowski = cfg->cart_minkowski;
    ph.floors_on = cfg->floors_on;
    ph.frame = cfg->floor_frame;
    ph.iter_max = cfg->iter_max;
    ph.err_tol = cfg->err_tol;
    ph.fix_avg = cfg->fix_average_neighbors;
    ph.fix_atmo = cfg->fix_atmosphere;
    ph.dx1 = cfg->dx1; ph.dx2 = cfg->dx2; ph.dx3 = cfg->dx3;
    ph.zero_polar_flux = cfg->zero_polar_flux;
    ph.fix_polar_flux = cfg->fix_polar_flux && cfg->spherical;
    ph.check_inflow_in = cfg->check_inflow_inner_x1;
    ph.check_inflow_out = cfg->check_inflow_outer_x1;
    if (cfg->inverter != KHB_INVERTER_ONEDW && cfg->inverter != KHB_INVERTER_KASTAUN) {
        *why = "unknown inverter";
        return KHB_ERR_UNSUPPORTED;
    }
    ph.inverter = cfg->inverter;
    ph.fofc = cfg->fofc;
    ph.fofc_polar_cells = cfg->fofc_polar_cells;
    ph.fofc_r_mark = cfg->r_horizon + cfg->fofc_eh_buffer;
    ph.fofc_glf = cfg->fofc_use_glf != 0;
    ph.fofc_source = cfg->fofc_use_source_term != 0;
    if (cfg->fofc && cfg->fofc_polar_cells < 0) { *why = "fofc_polar_cells must be >= 0"; return KHB_ERR_ARG; }
    if (cfg->ct_scheme < KHB_CT_NONE || cfg->ct_scheme > KHB_CT_GS05_C) { *why = "unknown ct_scheme"; return KHB_ERR_ARG; }
    if (cfg->ct_scheme != KHB_CT_NONE) {
        if (cfg->nvar != 8) { *why = "B_CT needs the magnetic field (nvar 8)"; return KHB_ERR_UNSUPPORTED; }
        if (d.ndim < 2) { *why = "B_CT blocks are 2D or 3D"; return KHB_ERR_UNSUPPORTED; }
        bool physical = false;
        for (int f = 0; f < 2 * d.ndim; ++f) {
            if (!phys_face(cfg->bc[f])) continue;
            physical = true;
            // b_ct_boundaries.cpp: outflow (clean_face_B) and reflecting (reflect_face_vector,
            // zero_EMF) faces in every direction, transmitting (average_EMF) X2 faces as for the zones
            if (cfg->bc[f] != KHB_BC_OUTFLOW && cfg->bc[f] != KHB_BC_REFLECTING && cfg->bc[f] != KHB_BC_TRANSMITTING) {
                *why = "B_CT blocks take outflow, reflecting or transmitting faces, periodic or exchange faces otherwise";
                return KHB_ERR_UNSUPPORTED;
            }
        }
        if (physical && cfg->ng < 4) { *why = "B_CT with physical faces needs 4 ghost zones"; return KHB_ERR_UNSUPPORTED; }
        if (cfg->fofc) { *why = "FOFC with B_CT is not supported"; return KHB_ERR_UNSUPPORTED; }
    }
    ph.ct_scheme = cfg->ct_scheme;
    if (cfg->ct_scheme != KHB_CT_NONE) ph.fix_polar_flux = 0;      // B_FluxCT's polar fix; not loaded with B_CT
    ph.recon_extra = (cfg->recon >= KHB_RECON_LINEAR_VL) ? cfg->recon - KHB_RECON_PPM : 0;
    if (cfg->recon_lower < KHB_RECON_LOWER_NONE || cfg->recon_lower > KHB_RECON_LOWER_POLES) {
        *why = "unknown recon_lower";
        return KHB_ERR_ARG;
    }
    if (cfg->recon_lower && cfg->recon != KHB_RECON_WENO5) {
        *why = "lowered reconstruction near edges or poles is a weno5 option";   // flux.cpp:82-83
        return KHB_ERR_ARG;
    }
    ph.weno_lower = cfg->recon_lower;
    if (cfg->recon_fallback && (cfg->recon == KHB_RECON_DONOR_CELL || cfg->recon == KHB_RECON_LINEAR_MC ||
                                cfg->recon == KHB_RECON_PPM)) {
        *why = "reconstruction_fallback applies to the high-order reconstructions";
        return KHB_ERR_UNSUPPORTED;
    }
    if (cfg->recon_fallback && !cfg->floors_on) { *why = "reconstruction_fallback needs floors"; return KHB_ERR_ARG; }
    ph.recon_fallback = cfg->recon_fallback;
    std::memcpy(&ph.fl, &cfg->floors, sizeof(khb_floors));
    std::memcpy(&ph.fl_inner, &cfg->floors_inner, sizeof(khb_floors));
    if (cfg->floor_frame < KHB_FRAME_FLUID || cfg->floor_frame > KHB_FRAME_MIXED_NORMAL_DRIFT) {
        *why = "unknown floor frame";
        return KHB_ERR_ARG;
    }
    ph.frame_switch_r = cfg->frame_switch_r;
    ph.frame_switch_beta = cfg->frame_switch_beta;
    return KHB_OK;
}

// ======================================================================== C ABI
extern "C" {

const char* khb_last_error(void) { return g_err.c_str(); }
int khb_version(void) { return 100; }

int khb_create(const khb_config* cfg, khb_ctx** out)
{
    if (!cfg || !out) return fail(KHB_ERR_ARG, "khb_create: NULL argument");
    *out = nullptr;
    Dims dd;
    Phys pp;
    const char* why = nullptr;
    const int drc = khb::derive_block(cfg, dd, pp, &why);
    if (drc) return fail(drc, why);
    khb_ctx* c = new khb_ctx();
    std::memset((void*)c, 0, sizeof(khb_ctx));
    c->cfg = *cfg;
    c->nv = cfg->nvar;
    c->dbl_max_bits = 0x7FEFFFFFFFFFFFFFull;
    c->fp32 = cfg->precision == KHB_PREC_FP32_FLUX;
    c->d = dd;
    c->ph = pp;
    c->zone_split = 1;
    const Dims& d = c->d;
    const size_t N = (size_t)d.N, fs = ft_size(c);
    auto alloc = [&](void** p, size_t bytes) -> cudaError_t {
        cudaError_t e = cudaMalloc(p, bytes);
        if (e == cudaSuccess) e = cudaMemset(*p, 0, bytes);
        return e;
    };
    cudaError_t e = cudaSuccess;
    for (int x = 0; x < 3 && e == cudaSuccess; ++x) {
        e = alloc(&c->F[x], fs * c->nv * N);
        if (e == cudaSuccess) e = alloc(&c->ctop[x], fs * N);
    }
    if (e == cudaSuccess) e = alloc(&c->emf, fs * 3 * N);
    if (e == cudaSuccess) e = alloc((void**)&c->stageP, sizeof(double) * c->nv * N);
    if (e == cudaSuccess) e = alloc((void**)&c->stageU, sizeof(double) * c->nv * N);
    if (e == cudaSuccess) e = alloc((void**)&c->words, sizeof(unsigned long long) * 4);
    if (e == cudaSuccess) e = alloc((void**)&c->fail_count, sizeof(int) * 4);
    if (e == cudaSuccess) e = alloc((void**)&c->fail_list, sizeof(int) * N);
    if (e == cudaSuccess) e = alloc((void**)&c->imp_words, sizeof(unsigned long long) * IMP_WORDS);
    if (e == cudaSuccess && cfg->fofc) e = alloc((void**)&c->fofc_flag, sizeof(int32_t) * N);
    if (e == cudaSuccess && cfg->ct_scheme) e = alloc(&c->ct_emfc, fs * 3 * N);
    if (e == cudaSuccess && cfg->ct_scheme) e = alloc((void**)&c->ct_stageBf, sizeof(double) * 3 * N);
    // words[3]: the status word of the bounds-checked build (every kernel sees it through Dims)
    if (e == cudaSuccess) c->d.chk = c->words + 3;
    // the memsets above run on the legacy default stream, which the caller's (non-blocking) streams
    // do not wait for: finish them before the context is handed out
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        khb_destroy(c);
        return fail(KHB_ERR_CUDA, std::string("khb_create: ") + cudaGetErrorString(e));
    }
    *out = c;
    return KHB_OK;
}

int khb_destroy(khb_ctx* c)
{
    if (!c) return KHB_OK;
    for (int x = 0; x < 3; ++x) { cudaFree(c->F[x]); cudaFree(c->ctop[x]); }
    cudaFree(c->emf); cudaFree(c->stageP); cudaFree(c->stageU);
    cudaFree(c->words); cudaFree(c->fail_count); cudaFree(c->fail_list);
    cudaFree(c->geo_d); cudaFree(c->geo_f);
    cudaFree(c->conn_d); cudaFree(c->emhd_tmp); cudaFree(c->fix_buf); cudaFree(c->imp_words);
    for (int x = 0; x < 3; ++x) cudaFree(c->F10[x]);
    cudaFree(c->dudt10);
    cudaFree(c->fofc_flag);
    cudaFree(c->dt_state);
    cudaFree(c->adj_buf); cudaFree(c->adj_flags); cudaFree(c->adj_red);
    cudaFree(c->adj_pf); cudaFree(c->adj_s2); cudaFree(c->adj_flags2);
    cudaFree(c->ct_emfc); cudaFree(c->ct_stageBf);
    if (c->gexec) cudaGraphExecDestroy(c->gexec);
    if (c->graph) cudaGraphDestroy(c->graph);
    delete c;
    return KHB_OK;
}

int khb_set_geometry(khb_ctx* ctx, const double* gcov, const double* gcon, const double* gdet,
                     const double* gdet_conn, const double* r_center)
{
    if (!ctx || !gcov || !gcon || !gdet || !gdet_conn || !r_center) return fail(KHB_ERR_ARG, "khb_set_geometry: NULL argument");
    const Dims& d = ctx->d;
    const int G1 = d.n1 + 1, G2 = d.n2 + 1;
    const size_t gs = (size_t)G1*G2;
    // device layout: for loc 0..3: gcov [16][G2][G1], gcon [16][G2][G1], gdet [G2][G1]; then
    // gdet_conn [64][n2][n1] and r_center [n2][n1]
    const size_t per_loc = 33 * gs, n2n1 = (size_t)d.n2*d.n1;
    const size_t total = 4*per_loc + 64*n2n1 + 3*n2n1;
    std::vector<double> h(total);
    std::vector<float> hf(3*per_loc);
    for (int loc = 0; loc < 4; ++loc) {
        double* base = h.data() + loc*per_loc;
        for (size_t x = 0; x < gs; ++x) {
            const size_t src = (size_t)loc*gs + x;
            for (int m = 0; m < 16; ++m) {
                base[m*gs + x] = gcov[src*16 + m];
                base[(16 + m)*gs + x] = gcon[src*16 + m];
            }
            base[32*gs + x] = gdet[src];
        }
        if (loc < 3) for (size_t x = 0; x < per_loc; ++x) hf[loc*per_loc + x] = (float)base[x];
    }
    double* gc = h.data() + 4*per_loc;
    for (size_t x = 0; x < n2n1; ++x)
        for (int m = 0; m < 64; ++m) gc[m*n2n1 + x] = gdet_conn[x*64 + m];
    std::memcpy(h.data() + 4*per_loc + 64*n2n1, r_center, n2n1*sizeof(double));
    // geometric floors per zone centre (floors_functions.hpp:96-104), x3-independent
    double* frho = h.data() + 4*per_loc + 65*n2n1;
    double* fu = frho + n2n1;
    for (size_t x = 0; x < n2n1; ++x) {
        // the inner prescription inside floors_switch_r (floors_functions.hpp:89-90)
        const khb_floors& f = (ctx->cfg.floors.radius_dependent_floors && r_center[x] < ctx->cfg.floors.floors_switch_r)
                                  ? ctx->cfg.floors_inner : ctx->cfg.floors;
        if (ctx->cfg.spherical) {
            const double r = r_center[x];
            const double rhoscal = (f.use_r_char) ? 1. / ((r*r) * (1 + r / f.r_char)) : 1. / std::sqrt(r*r*r);
            const double a = f.rho_min_geom * rhoscal, b = f.u_min_geom * std::pow(rhoscal, ctx->cfg.gam);
            frho[x] = (a < f.rho_min_const) ? f.rho_min_const : a;
            fu[x] = (b < f.u_min_const) ? f.u_min_const : b;
        } else {
            frho[x] = f.rho_min_const;
            fu[x] = f.u_min_const;
        }
    }
    if (!ctx->geo_d) {
        KHB_CUDA(cudaMalloc((void**)&ctx->geo_d, total*sizeof(double)));
        KHB_CUDA(cudaMalloc((void**)&ctx->geo_f, hf.size()*sizeof(float)));
    }
    KHB_CUDA(cudaMemcpy(ctx->geo_d, h.data(), total*sizeof(double), cudaMemcpyHostToDevice));
    KHB_CUDA(cudaMemcpy(ctx->geo_f, hf.data(), hf.size()*sizeof(float), cudaMemcpyHostToDevice));
    // a copy from pageable memory may return before it lands, and kernels on non-blocking streams
    // do not wait for the legacy stream: complete the upload before any kernel can read it
    KHB_CUDA(cudaDeviceSynchronize());
    DevGeom& g = ctx->g;
    g.G1 = G1; g.G2 = G2; g.n1 = d.n1; g.gs = (long long)gs;
    for (int loc = 0; loc < 4; ++loc) {
        g.gcov[loc] = ctx->geo_d + loc*per_loc;
        g.gcon[loc] = ctx->geo_d + loc*per_loc + 16*gs;
        g.gdet[loc] = ctx->geo_d + loc*per_loc + 32*gs;
        if (loc < 3) {
            g.gcov_f[loc] = ctx->geo_f + loc*per_loc;
            g.gcon_f[loc] = ctx->geo_f + loc*per_loc + 16*gs;
            g.gdet_f[loc] = ctx->geo_f + loc*per_loc + 32*gs;
        }
    }
    g.gdet_conn = ctx->geo_d + 4*per_loc;
    g.rcen = ctx->geo_d + 4*per_loc + 64*n2n1;
    g.floor_rho = g.rcen + n2n1;
    g.floor_u = g.rcen + 2*n2n1;
    ctx->geom_set = true;
    return KHB_OK;
}

#define KHB_NEED_GEOM(ctx) do { if (!(ctx)) return fail(KHB_ERR_ARG, "NULL context"); \
    if (!(ctx)->geom_set) return fail(KHB_ERR_STATE, "geometry not set (call khb_set_geometry)"); } while (0)

int khb_get_flux(khb_ctx* ctx, int dir, const khb_fields* P, void* stream)
{
    KHB_RANGE("khb_get_flux");
    KHB_NEED_GEOM(ctx);
    if (dir < 1 || dir > ctx->d.ndim) return fail(KHB_ERR_ARG, "khb_get_flux: dir out of range");
    int rc;
    if ((rc = check_fields(ctx, P, "P"))) return rc;
    return launch_flux(ctx, dir, *P, S(stream));
}

int khb_get_flux_planes(khb_ctx* ctx, int dir, const khb_fields* P, int k_lo, int k_hi, void* stream)
{
    KHB_RANGE("khb_get_flux_planes");
    KHB_NEED_GEOM(ctx);
    if (dir < 1 || dir > ctx->d.ndim) return fail(KHB_ERR_ARG, "khb_get_flux_planes: dir out of range");
    if (k_lo > k_hi) return fail(KHB_ERR_ARG, "khb_get_flux_planes: empty plane range");
    int rc;
    if ((rc = check_fields(ctx, P, "P"))) return rc;
    return launch_flux(ctx, dir, *P, S(stream), k_lo, k_hi);
}

int khb_fofc(khb_ctx* ctx, int stage, double dt, const khb_fields* P_s, const khb_fields* U_s,
             const khb_fields* U_0, void* stream)
{
    KHB_RANGE("khb_fofc");
    KHB_NEED_GEOM(ctx);
    if (stage != 1 && stage != 2) return fail(KHB_ERR_ARG, "khb_fofc: stage must be 1 or 2");
    if (!ctx->ph.fofc) return fail(KHB_ERR_STATE, "khb_fofc: the context was created with fofc off");
    int rc;
    if ((rc = check_fields(ctx, P_s, "P_s")) || (rc = check_fields(ctx, U_s, "U_s")) ||
        (rc = check_fields(ctx, U_0, "U_0"))) return rc;
    return launch_fofc(ctx, stage, dt, *P_s, *U_s, *U_0, S(stream));
}

int khb_fix_flux(khb_ctx* ctx, void* stream)
{
    KHB_RANGE("khb_fix_flux");
    KHB_NEED_GEOM(ctx);
    return launch_fix_flux(ctx, ctx->ph, S(stream));
}

int khb_flux_ct(khb_ctx* ctx, void* stream)
{
    KHB_RANGE("khb_flux_ct");
    KHB_NEED_GEOM(ctx);
    if (ctx->nv < 8 || ctx->d.ndim < 2) return KHB_OK;
    if (ctx->fp32)
        Launch<float>::flux_ct(ctx->d, (float*)ctx->F[0], (float*)ctx->F[1], (float*)ctx->F[2], (float*)ctx->emf, S(stream));
    else
        Launch<double>::flux_ct(ctx->d, (double*)ctx->F[0], (double*)ctx->F[1], (double*)ctx->F[2], (double*)ctx->emf, S(stream));
    ctx->launches++;
    KHB_LAUNCHED(ctx);
    // zero polar fluxes again after the rewrite (KBoundaries::FixFlux acts on the final fluxes)
    if (ctx->ph.zero_polar_flux) {
        Phys ph = ctx->ph;
        ph.fix_polar_flux = 0;
        ph.check_inflow_in = ph.check_inflow_out = 0;
        return launch_fix_flux(ctx, ph, S(stream));
    }
    return KHB_OK;
}

int khb_copy_flux(khb_ctx* ctx, int dir, const khb_fields* F_out, double* ctop_out, void* stream)
{
    if (!ctx || dir < 1 || dir > 3 || !F_out) return fail(KHB_ERR_ARG, "khb_copy_flux: bad argument");
    const long long N = ctx->d.N;
    if (ctx->fp32)
        Launch<float>::copy_flux(N, ctx->nv, (const float*)ctx->F[dir-1], (const float*)ctx->ctop[dir-1], *F_out, ctop_out, S(stream));
    else
        Launch<double>::copy_flux(N, ctx->nv, (const double*)ctx->F[dir-1], (const double*)ctx->ctop[dir-1], *F_out, ctop_out, S(stream));
    KHB_LAUNCHED(ctx);
    return KHB_OK;
}

int khb_update(khb_ctx* ctx, const khb_fields* P_s, const khb_fields* U_s, const khb_fields* U_0,
               double gam0, double gam1, double beta_dt, const khb_fields* U_out, void* stream)
{
    KHB_RANGE("khb_update");
    KHB_NEED_GEOM(ctx);
    int rc;
    if ((rc = check_fields(ctx, P_s, "P_s")) || (rc = check_fields(ctx, U_s, "U_s")) ||
        (rc = check_fields(ctx, U_0, "U_0")) || (rc = check_fields(ctx, U_out, "U_out"))) return rc;
    ZoneCall zc;
    std::memset(&zc, 0, sizeof(zc));
    zc.Ps = *P_s; zc.Us = *U_s; zc.U0 = *U_0; zc.Pout = *P_s; zc.Uout = *U_out;
    zc.g0 = gam0; zc.g1 = gam1; zc.bdt = beta_dt;
    zc.mode = M_UPDATE;
    return launch_zone(ctx, zc, S(stream));
}

int khb_utop(khb_ctx* ctx, const khb_fields* U, const khb_fields* P, int32_t* pflag, int32_t* fflag, void* stream)
{
    KHB_RANGE("khb_utop");
    KHB_NEED_GEOM(ctx);
    int rc;
    if ((rc = check_fields(ctx, U, "U")) || (rc = check_fields(ctx, P, "P"))) return rc;
    if (!pflag || !fflag) return fail(KHB_ERR_ARG, "khb_utop: NULL flags");
    ZoneCall zc;
    std::memset(&zc, 0, sizeof(zc));
    zc.Ps = *P; zc.Us = *U; zc.U0 = *U; zc.Pout = *P; zc.Uout = *U;
    zc.pflag = pflag; zc.fflag = fflag;
    zc.mode = M_UTOP;
    return launch_zone(ctx, zc, S(stream));
}

int khb_apply_floors(khb_ctx* ctx, const khb_fields* P, const khb_fields* U, int32_t* pflag, int32_t* fflag, void* stream)
{
    KHB_RANGE("khb_apply_floors");
    KHB_NEED_GEOM(ctx);
    int rc;
    if ((rc = check_fields(ctx, U, "U")) || (rc = check_fields(ctx, P, "P"))) return rc;
    if (!pflag || !fflag) return fail(KHB_ERR_ARG, "khb_apply_floors: NULL flags");
    ZoneCall zc;
    std::memset(&zc, 0, sizeof(zc));
    zc.Ps = *P; zc.Us = *U; zc.U0 = *U; zc.Pout = *P; zc.Uout = *U;
    zc.pflag = pflag; zc.fflag = fflag;
    zc.mode = M_FLOORS;
    return launch_zone(ctx, zc, S(stream));
}

int khb_fix_utop(khb_ctx* ctx, const khb_fields* P, const khb_fields* U, const int32_t* pflag, void* stream)
{
    KHB_RANGE("khb_fix_utop");
    KHB_NEED_GEOM(ctx);
    int rc;
    if ((rc = check_fields(ctx, U, "U")) || (rc = check_fields(ctx, P, "P"))) return rc;
    if (!pflag) return fail(KHB_ERR_ARG, "khb_fix_utop: NULL pflag");
    // build the failed-zone list from pflag with a no-op zone pass
    KHB_CUDA(cudaMemsetAsync(ctx->fail_count, 0, sizeof(int), S(stream)));
    ZoneCall zc;
    std::memset(&zc, 0, sizeof(zc));
    zc.Ps = *P; zc.Us = *U; zc.U0 = *U; zc.Pout = *P; zc.Uout = *U;
    zc.pflag = const_cast<int32_t*>(pflag); zc.fflag = const_cast<int32_t*>(pflag);
    zc.mode = M_FAILLIST;
    if ((rc = launch_zone(ctx, zc, S(stream)))) return rc;
    return launch_fixup(ctx, *P, *U, pflag, S(stream));
}

int khb_boundaries(khb_ctx* ctx, const khb_fields* P, const khb_fields* U, void* stream)
{
    KHB_RANGE("khb_boundaries");
    KHB_NEED_GEOM(ctx);
    int rc;
    if ((rc = check_fields(ctx, U, "U")) || (rc = check_fields(ctx, P, "P"))) return rc;
    return launch_boundaries(ctx, *P, *U, S(stream));
}

int khb_ptou(khb_ctx* ctx, const khb_fields* P, const khb_fields* U, void* stream)
{
    KHB_RANGE("khb_ptou");
    KHB_NEED_GEOM(ctx);
    int rc;
    if ((rc = check_fields(ctx, U, "U")) || (rc = check_fields(ctx, P, "P"))) return rc;
    LaunchCommon::ptou(ctx->nv, ctx->d, ctx->g, ctx->ph, *P, *U, S(stream));
    KHB_LAUNCHED(ctx);
    return KHB_OK;
}

int khb_stage(khb_ctx* ctx, int stage, double dt, const khb_fields* P_s, const khb_fields* U_s,
              const khb_fields* U_0, const khb_fields* P_out, const khb_fields* U_out,
              int32_t* pflag, int32_t* fflag, void* stream)
{
    KHB_RANGE("khb_stage");
    KHB_NEED_GEOM(ctx);
    if (ctx->ph.ct_scheme) return fail(KHB_ERR_STATE, "khb_stage: a B_CT block steps with khb_ct_stage/khb_ct_step");
    if (stage != 1 && stage != 2) return fail(KHB_ERR_ARG, "khb_stage: stage must be 1 or 2");
    int rc;
    if ((rc = check_fields(ctx, P_s, "P_s")) || (rc = check_fields(ctx, U_s, "U_s")) ||
        (rc = check_fields(ctx, U_0, "U_0")) || (rc = check_fields(ctx, P_out, "P_out")) ||
        (rc = check_fields(ctx, U_out, "U_out"))) return rc;
    if (!pflag || !fflag) return fail(KHB_ERR_ARG, "khb_stage: NULL flags");
    return do_stage(ctx, stage, dt, *P_s, *U_s, *U_0, *P_out, *U_out, pflag, fflag, S(stream));
}

int khb_zone_pass(khb_ctx* ctx, int stage, double dt, const khb_fields* P_s, const khb_fields* U_s,
                  const khb_fields* U_0, const khb_fields* P_out, const khb_fields* U_out,
                  int32_t* pflag, int32_t* fflag, void* stream)
{
    KHB_RANGE("khb_zone_pass");
    KHB_NEED_GEOM(ctx);
    if (ctx->ph.ct_scheme) return fail(KHB_ERR_STATE, "khb_zone_pass: a B_CT block steps with khb_ct_stage/khb_ct_step");
    if (stage != 1 && stage != 2) return fail(KHB_ERR_ARG, "khb_zone_pass: stage must be 1 or 2");
    int rc;
    if ((rc = check_fields(ctx, P_s, "P_s")) || (rc = check_fields(ctx, U_s, "U_s")) ||
        (rc = check_fields(ctx, U_0, "U_0")) || (rc = check_fields(ctx, P_out, "P_out")) ||
        (rc = check_fields(ctx, U_out, "U_out"))) return rc;
    if (!pflag || !fflag) return fail(KHB_ERR_ARG, "khb_zone_pass: NULL flags");
    return zone_pass(ctx, stage, dt, *P_s, *U_s, *U_0, *P_out, *U_out, pflag, fflag, S(stream));
}

int khb_fix_utop_list(khb_ctx* ctx, const khb_fields* P, const khb_fields* U, const int32_t* pflag, void* stream)
{
    KHB_RANGE("khb_fix_utop_list");
    KHB_NEED_GEOM(ctx);
    int rc;
    if ((rc = check_fields(ctx, U, "U")) || (rc = check_fields(ctx, P, "P"))) return rc;
    if (!pflag) return fail(KHB_ERR_ARG, "khb_fix_utop_list: NULL pflag");
    return launch_fixup(ctx, *P, *U, pflag, S(stream));
}

int khb_step(khb_ctx* ctx, double dt, const khb_fields* P, const khb_fields* U,
             int32_t* pflag, int32_t* fflag, void* stream)
{
    KHB_RANGE("khb_step");
    KHB_NEED_GEOM(ctx);
    if (ctx->ph.ct_scheme) return fail(KHB_ERR_STATE, "khb_step: a B_CT block steps with khb_ct_stage/khb_ct_step");
    int rc;
    if ((rc = check_fields(ctx, P, "P")) || (rc = check_fields(ctx, U, "U"))) return rc;
    if (!pflag || !fflag) return fail(KHB_ERR_ARG, "khb_step: NULL flags");
    khb_fields P1, U1;
    std::memset(&P1, 0, sizeof(P1)); std::memset(&U1, 0, sizeof(U1));
    for (int p = 0; p < ctx->nv; ++p) {
        P1.v[p] = ctx->stageP + (size_t)p*ctx->d.N;
        U1.v[p] = ctx->stageU + (size_t)p*ctx->d.N;
    }
    if ((rc = do_stage(ctx, 1, dt, *P, *U, *U, P1, U1, pflag, fflag, S(stream)))) return rc;
    return do_stage(ctx, 2, dt, P1, U1, *U, *P, *U, pflag, fflag, S(stream));
}

static int check_ct_stage_args(khb_ctx* ctx, const char* who, int stage, const khb_fields* P_s,
                               const khb_fields* U_s, const khb_fields* U_0, const khb_fields* Bf_s,
                               const khb_fields* Bf_0, const khb_fields* P_out, const khb_fields* U_out,
                               const khb_fields* Bf_out, int32_t* pflag, int32_t* fflag)
{
    const std::string w(who);
    if (!ctx->ph.ct_scheme) return fail(KHB_ERR_STATE, w + ": block is not B_CT (cfg.ct_scheme)");
    if (stage != 1 && stage != 2) return fail(KHB_ERR_ARG, w + ": stage must be 1 or 2");
    int rc;
    if ((rc = check_fields(ctx, P_s, "P_s")) || (rc = check_fields(ctx, U_s, "U_s")) ||
        (rc = check_fields(ctx, U_0, "U_0")) || (rc = check_fields(ctx, P_out, "P_out")) ||
        (rc = check_fields(ctx, U_out, "U_out"))) return rc;
    for (const khb_fields* f : {Bf_s, Bf_0, Bf_out})
        if (!f || !f->v[0] || !f->v[1] || !f->v[2]) return fail(KHB_ERR_ARG, w + ": NULL face field");
    if (!pflag || !fflag) return fail(KHB_ERR_ARG, w + ": NULL flags");
    return KHB_OK;
}

int khb_ct_stage(khb_ctx* ctx, int stage, double dt, const khb_fields* P_s, const khb_fields* U_s,
                 const khb_fields* U_0, const khb_fields* Bf_s, const khb_fields* Bf_0, const khb_fields* P_out,
                 const khb_fields* U_out, const khb_fields* Bf_out, int32_t* pflag, int32_t* fflag, void* stream)
{
    KHB_RANGE("khb_ct_stage");
    KHB_NEED_GEOM(ctx);
    int rc;
    if ((rc = check_ct_stage_args(ctx, "khb_ct_stage", stage, P_s, U_s, U_0, Bf_s, Bf_0, P_out, U_out, Bf_out,
                                  pflag, fflag))) return rc;
    return do_ct_stage(ctx, stage, dt, *P_s, *U_s, *U_0, *Bf_s, *Bf_0, *P_out, *U_out, *Bf_out, pflag, fflag, S(stream));
}

int khb_ct_stage_fluxes(khb_ctx* ctx, const khb_fields* P_s, void* stream)
{
    KHB_RANGE("khb_ct_stage_fluxes");
    KHB_NEED_GEOM(ctx);
    if (!ctx->ph.ct_scheme) return fail(KHB_ERR_STATE, "khb_ct_stage_fluxes: block is not B_CT (cfg.ct_scheme)");
    int rc;
    if ((rc = check_fields(ctx, P_s, "P_s"))) return rc;
    return ct_stage_fluxes(ctx, *P_s, S(stream));
}

int khb_ct_stage_update(khb_ctx* ctx, int stage, double dt, const khb_fields* P_s, const khb_fields* U_s,
                        const khb_fields* U_0, const khb_fields* Bf_s, const khb_fields* Bf_0, const khb_fields* P_out,
                        const khb_fields* U_out, const khb_fields* Bf_out, int32_t* pflag, int32_t* fflag,
                        void* stream)
{
    KHB_RANGE("khb_ct_stage_update");
    KHB_NEED_GEOM(ctx);
    int rc;
    if ((rc = check_ct_stage_args(ctx, "khb_ct_stage_update", stage, P_s, U_s, U_0, Bf_s, Bf_0, P_out, U_out,
                                  Bf_out, pflag, fflag))) return rc;
    return ct_stage_update(ctx, stage, dt, *P_s, *U_s, *U_0, *Bf_s, *Bf_0, *P_out, *U_out, *Bf_out, pflag, fflag,
                           S(stream));
}

int khb_ct_stage_update_part(khb_ctx* ctx, int part, int stage, double dt, const khb_fields* P_s,
                             const khb_fields* U_s, const khb_fields* U_0, const khb_fields* Bf_s,
                             const khb_fields* Bf_0, const khb_fields* P_out, const khb_fields* U_out,
                             const khb_fields* Bf_out, int32_t* pflag, int32_t* fflag, void* stream)
{
    KHB_RANGE("khb_ct_stage_update_part");
    KHB_NEED_GEOM(ctx);
    if (part != 1 && part != 2) return fail(KHB_ERR_ARG, "khb_ct_stage_update_part: part is 1 or 2");
    int rc;
    if ((rc = check_ct_stage_args(ctx, "khb_ct_stage_update_part", stage, P_s, U_s, U_0, Bf_s, Bf_0, P_out, U_out,
                                  Bf_out, pflag, fflag))) return rc;
    if (ctx->fp32) return fail(KHB_ERR_UNSUPPORTED, "khb_ct_stage_update_part: FP64 blocks only");
    return ct_stage_update_part(ctx, part, stage, dt, *P_s, *U_s, *U_0, *Bf_s, *Bf_0, *P_out, *U_out, *Bf_out,
                                pflag, fflag, S(stream));
}

int khb_ct_ghost_from_faces(khb_ctx* ctx, const khb_fields* P, const khb_fields* U, const khb_fields* Bf,
                            void* stream)
{
    KHB_RANGE("khb_ct_ghost_from_faces");
    KHB_NEED_GEOM(ctx);
    if (!ctx->ph.ct_scheme) return fail(KHB_ERR_STATE, "khb_ct_ghost_from_faces: block is not B_CT (cfg.ct_scheme)");
    int rc;
    if ((rc = check_fields(ctx, P, "P")) || (rc = check_fields(ctx, U, "U"))) return rc;
    if (!Bf || !Bf->v[0] || !Bf->v[1] || !Bf->v[2]) return fail(KHB_ERR_ARG, "khb_ct_ghost_from_faces: NULL face field");
    const Dims& d = ctx->d;
    cudaStream_t st = S(stream);
    // the X1/X2 ghost zones of the interior k range, then (3D) both X3 ghost planes
    LaunchCommon::ghost_ptou(ctx->nv, d, ctx->g, ctx->ph, *P, *U, st, Bf, 7);
    KHB_LAUNCHED(ctx);
    if (d.ndim > 2) {
        LaunchCommon::ghost_ptou(ctx->nv, d, ctx->g, ctx->ph, *P, *U, st, Bf, 7, 3);
        KHB_LAUNCHED(ctx);
    }
    return KHB_OK;
}

int khb_ct_boundaries(khb_ctx* ctx, const khb_fields* P, const khb_fields* U, const khb_fields* Bf, void* stream)
{
    KHB_RANGE("khb_ct_boundaries");
    KHB_NEED_GEOM(ctx);
    if (!ctx->ph.ct_scheme) return fail(KHB_ERR_STATE, "khb_ct_boundaries: block is not B_CT (cfg.ct_scheme)");
    int rc;
    if ((rc = check_fields(ctx, P, "P")) || (rc = check_fields(ctx, U, "U"))) return rc;
    if (!Bf || !Bf->v[0] || !Bf->v[1] || !Bf->v[2]) return fail(KHB_ERR_ARG, "khb_ct_boundaries: NULL face field");
    return launch_boundaries(ctx, *P, *U, S(stream), Bf);
}

int khb_ct_step(khb_ctx* ctx, double dt, const khb_fields* P, const khb_fields* U, const khb_fields* Bf,
                int32_t* pflag, int32_t* fflag, void* stream)
{
    KHB_RANGE("khb_ct_step");
    KHB_NEED_GEOM(ctx);
    if (!ctx->ph.ct_scheme) return fail(KHB_ERR_STATE, "khb_ct_step: block is not B_CT (cfg.ct_scheme)");
    int rc;
    if ((rc = check_fields(ctx, P, "P")) || (rc = check_fields(ctx, U, "U"))) return rc;
    if (!Bf || !Bf->v[0] || !Bf->v[1] || !Bf->v[2]) return fail(KHB_ERR_ARG, "khb_ct_step: NULL face field");
    if (!pflag || !fflag) return fail(KHB_ERR_ARG, "khb_ct_step: NULL flags");
    khb_fields P1, U1, B1;
    std::memset(&P1, 0, sizeof(P1)); std::memset(&U1, 0, sizeof(U1)); std::memset(&B1, 0, sizeof(B1));
    for (int p = 0; p < ctx->nv; ++p) {
        P1.v[p] = ctx->stageP + (size_t)p*ctx->d.N;
        U1.v[p] = ctx->stageU + (size_t)p*ctx->d.N;
    }
    for (int x = 0; x < 3; ++x) B1.v[x] = ctx->ct_stageBf + (size_t)x*ctx->d.N;
    if ((rc = do_ct_stage(ctx, 1, dt, *P, *U, *U, *Bf, *Bf, P1, U1, B1, pflag, fflag, S(stream)))) return rc;
    return do_ct_stage(ctx, 2, dt, P1, U1, *U, B1, *Bf, *P, *U, *Bf, pflag, fflag, S(stream));
}

int khb_set_timestep(khb_ctx* ctx, double dt, double cfl, double dt_min, double max_dt_increase)
{
    if (!ctx) return fail(KHB_ERR_ARG, "khb_set_timestep: NULL context");
    if (!(dt > 0.) || !(cfl > 0.) || !(max_dt_increase > 0.)) return fail(KHB_ERR_ARG, "khb_set_timestep: bad value");
    if (!ctx->dt_state) KHB_CUDA(cudaMalloc((void**)&ctx->dt_state, 3 * sizeof(double)));
    const double h[3] = {dt, 0., 0.};
    KHB_CUDA(cudaMemcpy(ctx->dt_state, h, sizeof(h), cudaMemcpyHostToDevice));
    KHB_CUDA(cudaDeviceSynchronize());       // the upload is complete before any stream reads it
    ctx->dt_cfl = cfl; ctx->dt_min = dt_min; ctx->dt_max_increase = max_dt_increase;
    return KHB_OK;
}

int khb_get_timestep(khb_ctx* ctx, double* dt_next, double* t, double* dt_last, void* stream)
{
    if (!ctx || !ctx->dt_state) return fail(KHB_ERR_STATE, "khb_get_timestep: no device timestep (khb_set_timestep)");
    double h[3];
    KHB_CUDA(cudaMemcpyAsync(h, ctx->dt_state, sizeof(h), cudaMemcpyDeviceToHost, S(stream)));
    KHB_CUDA(cudaStreamSynchronize(S(stream)));
    if (dt_next) *dt_next = h[0];
    if (t) *t = h[1];
    if (dt_last) *dt_last = h[2];
    return KHB_OK;
}

int khb_step_device_dt(khb_ctx* ctx, const khb_fields* P, const khb_fields* U, int32_t* pflag, int32_t* fflag,
                       void* stream)
{
    KHB_RANGE("khb_step_device_dt");
    KHB_NEED_GEOM(ctx);
    if (ctx->ph.ct_scheme) return fail(KHB_ERR_STATE, "khb_step_device_dt: a B_CT block steps with khb_ct_stage/khb_ct_step");
    if (!ctx->dt_state) return fail(KHB_ERR_STATE, "khb_step_device_dt: no device timestep (khb_set_timestep)");
    int rc;
    if ((rc = check_fields(ctx, P, "P")) || (rc = check_fields(ctx, U, "U"))) return rc;
    if (!pflag || !fflag) return fail(KHB_ERR_ARG, "khb_step_device_dt: NULL flags");
    khb_fields P1, U1;
    std::memset(&P1, 0, sizeof(P1)); std::memset(&U1, 0, sizeof(U1));
    for (int p = 0; p < ctx->nv; ++p) {
        P1.v[p] = ctx->stageP + (size_t)p*ctx->d.N;
        U1.v[p] = ctx->stageU + (size_t)p*ctx->d.N;
    }
    ctx->dt_active = ctx->dt_state;
    rc = do_stage(ctx, 1, 0., *P, *U, *U, P1, U1, pflag, fflag, S(stream));
    if (!rc) rc = do_stage(ctx, 2, 0., P1, U1, *U, *P, *U, pflag, fflag, S(stream));
    ctx->dt_active = nullptr;
    if (rc) return rc;
    LaunchCommon::next_dt(ctx->words, ctx->dt_state, ctx->dt_cfl, ctx->dt_min, ctx->dt_max_increase, S(stream));
    KHB_LAUNCHED(ctx);
    return KHB_OK;
}

int khb_step_graph(khb_ctx* ctx, const khb_fields* P, const khb_fields* U, int32_t* pflag, int32_t* fflag,
                   void* stream)
{
    KHB_RANGE("khb_step_graph");
    KHB_NEED_GEOM(ctx);
    if (ctx->ph.ct_scheme) return fail(KHB_ERR_STATE, "khb_step_graph: a B_CT block steps with khb_ct_stage/khb_ct_step");
    cudaStream_t st = S(stream);
    if (!st) return fail(KHB_ERR_ARG, "khb_step_graph: needs a non-default stream to capture");
    if (!P || !U || !pflag || !fflag) return fail(KHB_ERR_ARG, "khb_step_graph: NULL argument");
    const bool same = ctx->gexec && !std::memcmp(&ctx->graph_P, P, sizeof(khb_fields)) &&
                      !std::memcmp(&ctx->graph_U, U, sizeof(khb_fields)) && ctx->graph_pflag == pflag &&
                      ctx->graph_fflag == fflag;
    if (!same) {
        if (ctx->gexec) { cudaGraphExecDestroy(ctx->gexec); ctx->gexec = nullptr; }
        if (ctx->graph) { cudaGraphDestroy(ctx->graph); ctx->graph = nullptr; }
        const int64_t l0 = ctx->launches;
        KHB_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        int rc = khb_step_device_dt(ctx, P, U, pflag, fflag, stream);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(st, &g);
        ctx->graph_launches = ctx->launches - l0;
        ctx->launches = l0;
        if (rc) { if (g) cudaGraphDestroy(g); return rc; }
        if (e != cudaSuccess) return fail(KHB_ERR_CUDA, std::string("khb_step_graph: capture: ") + cudaGetErrorString(e));
        ctx->graph = g;
        KHB_CUDA(cudaGraphInstantiate(&ctx->gexec, g, 0));
        ctx->graph_P = *P; ctx->graph_U = *U; ctx->graph_pflag = pflag; ctx->graph_fflag = fflag;
    }
    KHB_CUDA(cudaGraphLaunch(ctx->gexec, st));
    ctx->launches += ctx->graph_launches;
    return KHB_OK;
}

int khb_step_host(khb_ctx* ctx, double* const* P_host, const khb_fields* P, const khb_fields* U, int32_t* pflag,
                  int32_t* fflag, void* stream)
{
    KHB_RANGE("khb_step_host");
    KHB_NEED_GEOM(ctx);
    if (ctx->ph.ct_scheme) return fail(KHB_ERR_STATE, "khb_step_host: a B_CT block steps with khb_ct_stage/khb_ct_step");
    int rc;
    if ((rc = check_fields(ctx, P, "P")) || (rc = check_fields(ctx, U, "U"))) return rc;
    if (!P_host) return fail(KHB_ERR_ARG, "khb_step_host: NULL host state");
    for (int p = 0; p < ctx->nv; ++p)
        if (!P_host[p]) return fail(KHB_ERR_ARG, "khb_step_host: NULL host variable");
    cudaStream_t st = S(stream);
    const size_t bytes = sizeof(double) * (size_t)ctx->d.N;
    // the primitives in; the lock-step P -> U at the end of every stage (zone pass, ghost zones, periodic
    // images, fixups) leaves U = U(P) everywhere, so the conserved state is rebuilt, not copied
    for (int p = 0; p < ctx->nv; ++p) KHB_CUDA(cudaMemcpyAsync(P->v[p], P_host[p], bytes, cudaMemcpyHostToDevice, st));
    LaunchCommon::ptou(ctx->nv, ctx->d, ctx->g, ctx->ph, *P, *U, st);
    KHB_LAUNCHED(ctx);
    if ((rc = khb_step_graph(ctx, P, U, pflag, fflag, stream))) return rc;
    for (int p = 0; p < ctx->nv; ++p) KHB_CUDA(cudaMemcpyAsync(P_host[p], P->v[p], bytes, cudaMemcpyDeviceToHost, st));
    return KHB_OK;
}

int khb_step_host_interior(khb_ctx* ctx, double* const* P_host, const khb_fields* P, const khb_fields* U,
                           int32_t* pflag, int32_t* fflag, void* stream)
{
    KHB_RANGE("khb_step_host_interior");
    KHB_NEED_GEOM(ctx);
    if (ctx->ph.ct_scheme) return fail(KHB_ERR_STATE, "khb_step_host_interior: a B_CT block steps with khb_ct_stage/khb_ct_step");
    if (has_exchange_face(ctx->d))
        return fail(KHB_ERR_UNSUPPORTED, "khb_step_host_interior: exchange faces hold the caller's ghost zones; use khb_step_host");
    int rc;
    if ((rc = check_fields(ctx, P, "P")) || (rc = check_fields(ctx, U, "U"))) return rc;
    if (!P_host) return fail(KHB_ERR_ARG, "khb_step_host_interior: NULL host state");
    for (int p = 0; p < ctx->nv; ++p)
        if (!P_host[p]) return fail(KHB_ERR_ARG, "khb_step_host_interior: NULL host variable");
    cudaStream_t st = S(stream);
    const Dims& d = ctx->d;
    const long long nint = (long long)d.nx1 * d.nx2 * d.nx3;
    const size_t bytes = sizeof(double) * (size_t)nint;
    // the stage scratch is free before and after the step: it carries the packed interiors
    double* buf = ctx->stageP;
    for (int p = 0; p < ctx->nv; ++p)
        KHB_CUDA(cudaMemcpyAsync(buf + (size_t)p * nint, P_host[p], bytes, cudaMemcpyHostToDevice, st));
    k_interior_pack<<<blocks_for(nint, 256), 256, 0, st>>>(d, *P, ctx->nv, buf, 1);
    KHB_LAUNCHED(ctx);
    // U = U(P) on the interior (the ghost zones' values are rebuilt next), then the ghost zones
    // exactly as the step's last stage leaves them: boundaries of the interior, U = U(P) there
    LaunchCommon::ptou(ctx->nv, d, ctx->g, ctx->ph, *P, *U, st);
    KHB_LAUNCHED(ctx);
    if ((rc = launch_boundaries(ctx, *P, *U, st))) return rc;
    if ((rc = khb_step_graph(ctx, P, U, pflag, fflag, stream))) return rc;
    k_interior_pack<<<blocks_for(nint, 256), 256, 0, st>>>(d, *P, ctx->nv, buf, 0);
    KHB_LAUNCHED(ctx);
    for (int p = 0; p < ctx->nv; ++p)
        KHB_CUDA(cudaMemcpyAsync(P_host[p], buf + (size_t)p * nint, bytes, cudaMemcpyDeviceToHost, st));
    return KHB_OK;
}

int khb_get_min_ndt(khb_ctx* ctx, double* min_ndt_host, void* stream)
{
    if (!ctx || !min_ndt_host) return fail(KHB_ERR_ARG, "khb_get_min_ndt: NULL argument");
    unsigned long long bits = 0;
    KHB_CUDA(cudaMemcpyAsync(&bits, ctx->words, sizeof(bits), cudaMemcpyDeviceToHost, S(stream)));
    KHB_CUDA(cudaStreamSynchronize(S(stream)));
    std::memcpy(min_ndt_host, &bits, sizeof(double));
    return KHB_OK;
}

int khb_max_divb(khb_ctx* ctx, const khb_fields* U, double* max_divb_host, void* stream)
{
    KHB_RANGE("khb_max_divb");
    KHB_NEED_GEOM(ctx);
    if (!U || !max_divb_host) return fail(KHB_ERR_ARG, "khb_max_divb: NULL argument");
    if (ctx->nv < 8 || ctx->d.ndim < 2) { *max_divb_host = 0.; return KHB_OK; }
    const Dims& d = ctx->d;
    // b_flux_ct.cpp:554-564: skip the X1 corners of physical boundaries without Bflux0 fixes
    const int avoid_in = phys_face(d.bc[0]), avoid_out = phys_face(d.bc[1]);
    const int i_lo = d.is + avoid_in, i_hi = d.ie + !avoid_out;
    KHB_CUDA(cudaMemsetAsync(ctx->words + 1, 0, sizeof(unsigned long long), S(stream)));
    LaunchCommon::divb(d, ctx->ph, *U, i_lo, i_hi, ctx->words + 1, S(stream));
    KHB_LAUNCHED(ctx);
    unsigned long long bits = 0;
    KHB_CUDA(cudaMemcpyAsync(&bits, ctx->words + 1, sizeof(bits), cudaMemcpyDeviceToHost, S(stream)));
    KHB_CUDA(cudaStreamSynchronize(S(stream)));
    std::memcpy(max_divb_host, &bits, sizeof(double));
    return KHB_OK;
}

int khb_set_tuning(khb_ctx* ctx, const char* key, int value)
{
    if (!ctx || !key) return fail(KHB_ERR_ARG, "khb_set_tuning: NULL argument");
    if (std::strcmp(key, "zone_split") == 0) {
        if (value < 0 || value > 2) return fail(KHB_ERR_ARG, "khb_set_tuning: zone_split must be 0, 1 or 2");
        ctx->zone_split = value;
        return KHB_OK;
    }
    return fail(KHB_ERR_ARG, std::string("khb_set_tuning: unknown key ") + key);
}

int64_t khb_launch_count(khb_ctx* ctx) { return ctx ? ctx->launches : 0; }

int khb_bounds_checked(void) { return KHB_BOUNDS_CHECK ? 1 : 0; }

int khb_bounds_status(khb_ctx* ctx, uint64_t* status, void* stream)
{
    if (!ctx || !status) return fail(KHB_ERR_ARG, "khb_bounds_status: NULL argument");
    unsigned long long w = 0;
    KHB_CUDA(cudaMemcpyAsync(&w, ctx->words + 3, sizeof(w), cudaMemcpyDeviceToHost, S(stream)));
    KHB_CUDA(cudaMemsetAsync(ctx->words + 3, 0, sizeof(w), S(stream)));
    KHB_CUDA(cudaStreamSynchronize(S(stream)));
    *status = (uint64_t)w;
    return KHB_OK;
}

// ---------------------------------------------------------------------------- EMHD and implicit solve
static int check_emhd(const khb_emhd_params* e)
{
    if (!e) return fail(KHB_ERR_ARG, "EMHD parameters are NULL");
    if (e->closure < KHB_CLOSURE_CONSTANT || e->closure > KHB_CLOSURE_TORUS) return fail(KHB_ERR_ARG, "unknown EMHD closure");
    return KHB_OK;
}

static int check_fields10(const khb_emhd_params* e, const khb_fields* f, const char* name)
{
    if (!f) return fail(KHB_ERR_ARG, std::string(name) + " is NULL");
    for (int p = 0; p < 8; ++p)
        if (!f->v[p]) return fail(KHB_ERR_ARG, std::string(name) + " has a NULL variable pointer");
    if (e->conduction && !f->v[KHB_Q]) return fail(KHB_ERR_ARG, std::string(name) + ": q slot is NULL with conduction on");
    if (e->viscosity && !f->v[KHB_DP]) return fail(KHB_ERR_ARG, std::string(name) + ": dP slot is NULL with viscosity on");
    return KHB_OK;
}

int khb_set_connection(khb_ctx* ctx, const double* conn)
{
    KHB_NEED_GEOM(ctx);
    if (!conn) return fail(KHB_ERR_ARG, "khb_set_connection: NULL argument");
    const Dims& d = ctx->d;
    const size_t n2n1 = (size_t)d.n2 * d.n1, N = (size_t)d.N;
    std::vector<double> h(64 * n2n1);
    for (size_t x = 0; x < n2n1; ++x)
        for (int m = 0; m < 64; ++m) h[m*n2n1 + x] = conn[x*64 + m];
    if (!ctx->conn_d) {
        KHB_CUDA(cudaMalloc((void**)&ctx->conn_d, h.size() * sizeof(double)));
        KHB_CUDA(cudaMalloc((void**)&ctx->emhd_tmp, 5 * N * sizeof(double)));
        KHB_CUDA(cudaMalloc((void**)&ctx->fix_buf, 7 * N * sizeof(double)));
        KHB_CUDA(cudaMemset(ctx->emhd_tmp, 0, 5 * N * sizeof(double)));
        KHB_CUDA(cudaMemset(ctx->fix_buf, 0, 7 * N * sizeof(double)));
        for (int x = 0; x < 3; ++x) {
            KHB_CUDA(cudaMalloc((void**)&ctx->F10[x], 10 * N * sizeof(double)));
            KHB_CUDA(cudaMemset(ctx->F10[x], 0, 10 * N * sizeof(double)));
        }
        KHB_CUDA(cudaMalloc((void**)&ctx->dudt10, 10 * N * sizeof(double)));
        KHB_CUDA(cudaMemset(ctx->dudt10, 0, 10 * N * sizeof(double)));
    }
    KHB_CUDA(cudaMemcpy(ctx->conn_d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
    KHB_CUDA(cudaDeviceSynchronize());          // complete the upload (see khb_set_geometry)
    return KHB_OK;
}

int khb_emhd_ptou(khb_ctx* ctx, const khb_emhd_params* emhd, const khb_fields* P, const khb_fields* U, void* stream)
{
    KHB_RANGE("khb_emhd_ptou");
    KHB_NEED_GEOM(ctx);
    int rc;
    if ((rc = check_emhd(emhd)) || (rc = check_fields10(emhd, P, "P")) || (rc = check_fields10(emhd, U, "U"))) return rc;
    if (ctx->nv != 8) return fail(KHB_ERR_UNSUPPORTED, "khb_emhd_ptou: the block must carry B (nvar = 8)");
    LaunchEmhd::ptou(ctx->d, ctx->g, ctx->ph.gam, *emhd, *P, *U, S(stream));
    KHB_LAUNCHED(ctx);
    return KHB_OK;
}

int khb_emhd_add_source(khb_ctx* ctx, const khb_emhd_params* emhd, const khb_fields* P, const khb_fields* dUdt,
                        void* stream)
{
    KHB_RANGE("khb_emhd_add_source");
    KHB_NEED_GEOM(ctx);
    int rc;
    if ((rc = check_emhd(emhd)) || (rc = check_fields10(emhd, P, "P")) || (rc = check_fields10(emhd, dUdt, "dUdt")))
        return rc;
    if (!ctx->conn_d) return fail(KHB_ERR_STATE, "khb_emhd_add_source: connection not set (call khb_set_connection)");
    if (ctx->nv != 8) return fail(KHB_ERR_UNSUPPORTED, "khb_emhd_add_source: the block must carry B (nvar = 8)");
    if (!(emhd->conduction || emhd->viscosity)) return KHB_OK;
    LaunchEmhd::add_source(ctx->d, ctx->g, ctx->conn_d, ctx->ph.gam, *emhd, ctx->ph, *P, ctx->emhd_tmp, *dUdt,
                           S(stream));
    ctx->launches += 1;
    KHB_LAUNCHED(ctx);
    return KHB_OK;
}

static int implicit_args(khb_ctx* ctx, const khb_emhd_params* emhd, const khb_implicit_params* imp,
                         const khb_fields* P_full, const khb_fields* U_full, const khb_fields* P_sub,
                         const khb_fields* src, const khb_fields* P_solver, ImpFields& f)
{
    int rc;
    if ((rc = check_emhd(emhd))) return rc;
    if (!imp) return fail(KHB_ERR_ARG, "implicit parameters are NULL");
    if (imp->max_nonlinear_iter < 1 || imp->max_nonlinear_iter > IMP_MAX_ITER)
        return fail(KHB_ERR_ARG, "max_nonlinear_iter must be in [1, 64]");
    if (imp->max_linesearch_iter < 0 || imp->max_linesearch_iter > 1000)
        return fail(KHB_ERR_ARG, "max_linesearch_iter must be in [0, 1000]");
    if (imp->jacobian != KHB_JACOBIAN_FD && imp->jacobian != KHB_JACOBIAN_EXACT)
        return fail(KHB_ERR_ARG, "unknown Jacobian kind");
    if (ctx->nv != 8) return fail(KHB_ERR_UNSUPPORTED, "implicit solve: the block must carry B (nvar = 8)");
    if ((rc = check_fields10(emhd, P_full, "P_full")) || (rc = check_fields10(emhd, U_full, "U_full")) ||
        (rc = check_fields10(emhd, P_sub, "P_sub")) || (rc = check_fields10(emhd, src, "src")) ||
        (rc = check_fields10(emhd, P_solver, "P_solver")))
        return rc;
    f.Pf = *P_full; f.Uf = *U_full; f.Ps = *P_sub; f.S = *src; f.Psol = *P_solver;
    return KHB_OK;
}

int khb_implicit_step(khb_ctx* ctx, const khb_emhd_params* emhd, const khb_implicit_params* imp,
                      const khb_fields* P_full, const khb_fields* U_full, const khb_fields* P_sub,
                      const khb_fields* src, const khb_fields* P_solver, double* solve_norm, double* solve_fail,
                      double dt, void* stream)
{
    KHB_RANGE("khb_implicit_step");
    KHB_NEED_GEOM(ctx);
    ImpFields f;
    int rc;
    if ((rc = implicit_args(ctx, emhd, imp, P_full, U_full, P_sub, src, P_solver, f))) return rc;
    if (!solve_norm || !solve_fail) return fail(KHB_ERR_ARG, "khb_implicit_step: NULL solve_norm/solve_fail");
    f.solve_norm = solve_norm;
    f.solve_fail = solve_fail;
    KHB_CUDA(cudaMemsetAsync(ctx->imp_words, 0, sizeof(unsigned long long) * IMP_WORDS, S(stream)));
    for (int iter = 1; iter <= imp->max_nonlinear_iter; ++iter) {
        LaunchEmhd::implicit_iter(ctx->d, ctx->g, ctx->ph.gam, *emhd, *imp, f, dt, ctx->imp_words, iter, S(stream));
        KHB_LAUNCHED(ctx);
    }
    return KHB_OK;
}

// ---------------------------------------------------------------------------- explicit EMHD step and ImEx stage
namespace {
int emhd_flux_ready(khb_ctx* ctx, const khb_emhd_params* emhd, const char* who)
{
    if (check_emhd(emhd)) return KHB_ERR_ARG;
    if (!ctx->F10[0]) return fail(KHB_ERR_STATE, std::string(who) + ": EMHD scratch not allocated (call khb_set_connection)");
    if (ctx->nv != 8) return fail(KHB_ERR_UNSUPPORTED, std::string(who) + ": the block must carry B (nvar = 8)");
    if (ctx->fp32) return fail(KHB_ERR_UNSUPPORTED, std::string(who) + ": the EMHD path is FP64 only");
    if (ctx->cfg.recon > KHB_RECON_PPM || ctx->ph.weno_lower || ctx->ph.recon_fallback)
        return fail(KHB_ERR_UNSUPPORTED, std::string(who) + ": EMHD fluxes use donor cell, linear MC, WENO5 or PPM");
    return KHB_OK;
}
void emhd_face_range(const Dims& d, int dir, int lo[3], int cnt[3])
{
    const int s[3] = {d.is, d.js, d.ks}, e[3] = {d.ie, d.je, d.ke};
    for (int a = 0; a < 3; ++a) {
        const bool active = (a + 1) <= d.ndim;
        int hi;
        if (a + 1 == dir) { lo[a] = s[a]; hi = e[a] + 1; }
        else if (active) { lo[a] = s[a] - 1; hi = e[a] + 1; }
        else { lo[a] = s[a]; hi = e[a]; }
        cnt[a] = hi - lo[a] + 1;
    }
}
khb_fields fields_of(double* base, long long N)
{
    khb_fields f;
    for (int p = 0; p < KHB_MAX_VARS; ++p) f.v[p] = base + (size_t)p * N;
    return f;
}
} // namespace

int khb_get_flux_emhd(khb_ctx* ctx, const khb_emhd_params* emhd, int dir, const khb_fields* P, void* stream)
{
    KHB_RANGE("khb_get_flux_emhd");
    KHB_NEED_GEOM(ctx);
    int rc;
    if ((rc = emhd_flux_ready(ctx, emhd, "khb_get_flux_emhd")) || (rc = check_fields10(emhd, P, "P"))) return rc;
    if (dir < 1 || dir > ctx->d.ndim) return fail(KHB_ERR_ARG, "khb_get_flux_emhd: bad direction");
    int lo[3], cnt[3];
    emhd_face_range(ctx->d, dir, lo, cnt);
    LaunchEmhd::flux(ctx->cfg.recon, dir, ctx->d, ctx->g, ctx->ph, *emhd, *P, ctx->F10[dir - 1],
                     (double*)ctx->ctop[dir - 1], lo, cnt, S(stream));
    KHB_LAUNCHED(ctx);
    return KHB_OK;
}

int khb_copy_flux_emhd(khb_ctx* ctx, int dir, const khb_fields* F_out, double* ctop_out, void* stream)
{
    if (!ctx || dir < 1 || dir > 3 || !F_out) return fail(KHB_ERR_ARG, "khb_copy_flux_emhd: bad argument");
    if (!ctx->F10[0]) return fail(KHB_ERR_STATE, "khb_copy_flux_emhd: EMHD scratch not allocated");
    const size_t N = (size_t)ctx->d.N;
    for (int p = 0; p < 10; ++p)
        if (F_out->v[p])
            KHB_CUDA(cudaMemcpyAsync(F_out->v[p], ctx->F10[dir - 1] + p * N, N * sizeof(double),
                                     cudaMemcpyDeviceToDevice, S(stream)));
    if (ctop_out)
        KHB_CUDA(cudaMemcpyAsync(ctop_out, ctx->ctop[dir - 1], N * sizeof(double), cudaMemcpyDeviceToDevice, S(stream)));
    return KHB_OK;
}

int khb_imex_stage(khb_ctx* ctx, const khb_emhd_params* emhd, const khb_implicit_params* imp, int stage, double dt,
                   const khb_fields* P_full, const khb_fields* U_full, const khb_fields* P_sub, const khb_fields* U_sub,
                   const khb_fields* P_out, const khb_fields* U_out, double* solve_norm, double* solve_fail,
                   void* stream)
{
    return khb_imex_stage_flags(ctx, emhd, imp, stage, dt, P_full, U_full, P_sub, U_sub, P_out, U_out, solve_norm,
                                solve_fail, nullptr, nullptr, stream);
}

int khb_imex_stage_flags(khb_ctx* ctx, const khb_emhd_params* emhd, const khb_implicit_params* imp, int stage,
                         double dt, const khb_fields* P_full, const khb_fields* U_full, const khb_fields* P_sub,
                         const khb_fields* U_sub, const khb_fields* P_out, const khb_fields* U_out,
                         double* solve_norm, double* solve_fail, int32_t* fflag, int32_t* eflag, void* stream)
{
    KHB_RANGE("khb_imex_stage");
    KHB_NEED_GEOM(ctx);
    if (ctx->ph.ct_scheme) return fail(KHB_ERR_UNSUPPORTED, "khb_imex_stage: EMHD with B_CT is not supported");
    int rc;
    if ((rc = emhd_flux_ready(ctx, emhd, "khb_imex_stage"))) return rc;
    if (stage != 1 && stage != 2) return fail(KHB_ERR_ARG, "khb_imex_stage: stage must be 1 or 2");
    if ((rc = check_fields10(emhd, P_full, "P_full")) || (rc = check_fields10(emhd, U_full, "U_full")) ||
        (rc = check_fields10(emhd, P_sub, "P_sub")) || (rc = check_fields10(emhd, U_sub, "U_sub")) ||
        (rc = check_fields10(emhd, P_out, "P_out")) || (rc = check_fields10(emhd, U_out, "U_out"))) return rc;
    if (P_out->v[0] == P_sub->v[0] || U_out->v[0] == U_sub->v[0])
        return fail(KHB_ERR_ARG, "khb_imex_stage: the output state must not alias the sub-step state");
    if (!solve_norm || !solve_fail) return fail(KHB_ERR_ARG, "khb_imex_stage: NULL solve_norm/solve_fail");
    if (ctx->ph.floors_on && !fflag)
        return fail(KHB_ERR_ARG, "khb_imex_stage: floors on the EMHD state write their flags (khb_imex_stage_flags)");
    if (emhd->stability_limits && !eflag)
        return fail(KHB_ERR_ARG, "khb_imex_stage: the EMHD stability limits write their flags (khb_imex_stage_flags)");
    if (ctx->ph.floors_on && ctx->ph.frame != KHB_FRAME_FLUID && ctx->ph.frame != KHB_FRAME_DRIFT)
        return fail(KHB_ERR_UNSUPPORTED, "khb_imex_stage: floors on the EMHD state in the fluid or drift frame only "
                                         "(the normal frame re-inverts a conserved state the implicit solve does not form)");
    const Dims& d = ctx->d;
    bool physical = false;
    for (int f = 0; f < 2 * d.ndim; ++f) physical |= phys_face(d.bc[f]);
    cudaStream_t st = S(stream);
    const int s = stage - 1;
    // vl2, which the implicit package forces (implicit.cpp:96): gam0 = {0, 0}, gam1 = {1, 1}, beta = {1/2, 1}
    const double g0 = 0.0, g1 = 1.0, beta = (stage == 1) ? 0.5 : 1.0, bdt = beta * dt;
    for (int dir = 1; dir <= d.ndim; ++dir)
        if ((rc = khb_get_flux_emhd(ctx, emhd, dir, P_sub, stream))) return rc;
    // FixFlux on the physical faces (polar B-flux fix, zero polar fluxes of all 10 slots, X1 inflow
    // checks); flux-CT, and the polar zeroing after it, run inside the divergence kernel
    if (physical && (rc = launch_fix_flux_t<double>(ctx, ctx->ph, st, ctx->F10[0], ctx->F10[1], ctx->F10[2], 10)))
        return rc;
    if (stage == 2)
        KHB_CUDA(cudaMemcpyAsync(ctx->words, &ctx->dbl_max_bits, sizeof(unsigned long long), cudaMemcpyHostToDevice, st));
    khb_fields du = fields_of(ctx->dudt10, d.N);
    for (int p = 8; p < 10; ++p)
        if (!((p == 8 && emhd->conduction) || (p == 9 && emhd->viscosity))) du.v[p] = nullptr;
    double* ct[3] = {(double*)ctx->ctop[0], (double*)ctx->ctop[1], (double*)ctx->ctop[2]};
    LaunchEmhd::dudt(d, ctx->g, ctx->ph, *emhd, ctx->F10, ct, *P_sub, du, stage == 2, ctx->words, st);
    KHB_LAUNCHED(ctx);
    LaunchEmhd::add_source(d, ctx->g, ctx->conn_d, ctx->ph.gam, *emhd, ctx->ph, *P_sub, ctx->emhd_tmp, du, st);
    ctx->launches += 1;
    KHB_LAUNCHED(ctx);
    LaunchEmhd::imex_explicit(d, ctx->g, *P_sub, *U_sub, *U_full, du, *P_out, *U_out, g0, g1, bdt, st);
    KHB_LAUNCHED(ctx);
    (void)s;
    if ((rc = khb_implicit_step(ctx, emhd, imp, P_full, U_full, P_sub, &du, P_out, solve_norm, solve_fail, bdt,
                                stream))) return rc;
    // Packages::MeshApplyFloors over the interior (imex_step.cpp:269): the GRMHD floors, then the EMHD
    // package's stability limits
    if (ctx->ph.floors_on) {
        LaunchEmhd::floors(d, ctx->g, ctx->ph, *P_out, fflag, st);
        KHB_LAUNCHED(ctx);
    } else if (fflag) {
        KHB_CUDA(cudaMemsetAsync(fflag, 0, sizeof(int32_t) * (size_t)d.N, st));
    }
    if (emhd->stability_limits) {
        LaunchEmhd::limits(d, ctx->g, ctx->ph.gam, *emhd, *P_out, eflag, st);
        KHB_LAUNCHED(ctx);
    } else if (eflag) {
        KHB_CUDA(cudaMemsetAsync(eflag, 0, sizeof(int32_t) * (size_t)d.N, st));
    }
    if ((rc = khb_fix_solve(ctx, emhd, P_out, U_out, solve_fail, stream))) return rc;
    // ApplyBoundaryConditionsOnCoarseOrFineMD (imex_step.cpp:297-298) on the 10-slot state
    if (physical) {
        if ((rc = launch_boundaries(ctx, *P_out, *U_out, st, nullptr, 10))) return rc;
    } else {
        int pmask = 0;
        if (d.bc[0] == KHB_BC_PERIODIC) pmask |= 1;
        if (d.ndim >= 2 && d.bc[2] == KHB_BC_PERIODIC) pmask |= 2;
        if (d.ndim >= 3 && d.bc[4] == KHB_BC_PERIODIC) pmask |= 4;
        if (pmask) {
            LaunchCommon::periodic(10, d, *P_out, *U_out, pmask, st);
            KHB_LAUNCHED(ctx);
        }
    }
    return khb_emhd_ptou(ctx, emhd, P_out, U_out, stream);
}

int khb_implicit_stats(khb_ctx* ctx, int32_t* iterations, double* max_norms, void* stream)
{
    if (!ctx || !iterations) return fail(KHB_ERR_ARG, "khb_implicit_stats: NULL argument");
    unsigned long long w[IMP_WORDS];
    KHB_CUDA(cudaMemcpyAsync(w, ctx->imp_words, sizeof(w), cudaMemcpyDeviceToHost, S(stream)));
    KHB_CUDA(cudaStreamSynchronize(S(stream)));
    *iterations = (int32_t)w[IMP_ITER_WORD];
    if (max_norms)
        for (int it = 0; it < *iterations; ++it) std::memcpy(max_norms + it, w + it, sizeof(double));
    return KHB_OK;
}

int khb_implicit_jacobian(khb_ctx* ctx, const khb_emhd_params* emhd, const khb_implicit_params* imp,
                          const khb_fields* P_full, const khb_fields* U_full, const khb_fields* P_sub,
                          const khb_fields* src, const khb_fields* P_solver, double dt, double* jacobian,
                          double* residual, void* stream)
{
    KHB_RANGE("khb_implicit_jacobian");
    KHB_NEED_GEOM(ctx);
    ImpFields f;
    int rc;
    if ((rc = implicit_args(ctx, emhd, imp, P_full, U_full, P_sub, src, P_solver, f))) return rc;
    if (!jacobian || !residual) return fail(KHB_ERR_ARG, "khb_implicit_jacobian: NULL output");
    f.solve_norm = nullptr;
    f.solve_fail = nullptr;
    LaunchEmhd::implicit_jacobian(ctx->d, ctx->g, ctx->ph.gam, *emhd, *imp, f, dt, jacobian, residual, S(stream));
    KHB_LAUNCHED(ctx);
    return KHB_OK;
}

int khb_fix_solve(khb_ctx* ctx, const khb_emhd_params* emhd, const khb_fields* P, const khb_fields* U,
                  const double* solve_fail, void* stream)
{
    KHB_RANGE("khb_fix_solve");
    KHB_NEED_GEOM(ctx);
    int rc;
    if ((rc = check_emhd(emhd)) || (rc = check_fields10(emhd, P, "P")) || (rc = check_fields10(emhd, U, "U"))) return rc;
    if (!solve_fail) return fail(KHB_ERR_ARG, "khb_fix_solve: NULL solve_fail");
    if (!ctx->fix_buf) return fail(KHB_ERR_STATE, "khb_fix_solve: EMHD scratch not allocated (call khb_set_connection)");
    if (ctx->nv != 8) return fail(KHB_ERR_UNSUPPORTED, "khb_fix_solve: the block must carry B (nvar = 8)");
    LaunchEmhd::fix_solve(ctx->d, ctx->g, ctx->ph.gam, *emhd, *P, *U, solve_fail, ctx->fix_buf, S(stream));
    ctx->launches += 1;
    KHB_LAUNCHED(ctx);
    return KHB_OK;
}

} // extern "C"

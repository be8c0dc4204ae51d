// khb_batch.cu -- batches of meshblocks: every block of a (static-refined) mesh, of uneven sizes,
// advanced with one launch per kernel per RK stage, the step optionally replayed from a CUDA graph,
// and the tile shape per block size chosen by timing (autotune).
//
// The per-block arithmetic is the single-block path's (the batched kernels call the same device
// functions), so a batch step is bitwise identical to khb_step on each block in turn.
#include "khb_internal.hpp"

#include <algorithm>
#include <array>
#include <cstring>
#include <string>
#include <vector>

using namespace khb;

struct khb_batch {
    std::vector<khb_ctx*> ctx;
    std::vector<khb_fields> P, U;
    std::vector<int32_t*> pflag, fflag;
    int nb = 0, nv = 0, recon = 0, ndim = 0;
    bool fp32 = false;
    // block-size classes and their tile shapes
    std::vector<int> cls;                          // class of each block
    std::vector<std::array<int, 3>> class_size;    // (nx1, nx2, nx3) of each class
    std::vector<int> class_kz;                     // planes per CTA (0 = default)
    int persistent = 0;                            // 1: grid of (SMs x resident CTAs), CTAs loop over tiles
    // launch plan: 0 one launch per kernel per stage (counter reset, faces per direction, ghost-shell
    // copy, update half, cell half, fixups); 1 fused: three launches per stage (all faces with the
    // resets and shell copies, the whole zone pass, fixups), plus one launch for the flux fixes of
    // all blocks with physical faces, one launch per boundary phase for all blocks with physical or
    // periodic faces, and the mesh kernels of SMR meshes
    int plan = 0;
    int nsm = 0;
    // device tables
    void* desc = nullptr;                          // BatchBlock<FT>[nb]
    FixupBlock* fix = nullptr;                     // FixupBlock[nb]
    int** counts = nullptr;                        // fail_count pointer of each block
    int* tiles[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};   // x1-x3 faces, zones, fused-plan faces
    unsigned ntiles[5] = {0, 0, 0, 0, 0};
    unsigned grid[5] = {0, 0, 0, 0, 0};            // 0: one CTA per tile
    unsigned grid_fused_zone = 0;
    int occ[7] = {0, 0, 0, 0, 0, 0, 0};            // resident CTAs per SM: flux x1..x3, update, cell, faces, zone pass
    double* dt_dev = nullptr;
    unsigned long long* word = nullptr;            // minimum zone timestep (bit pattern)
    double dt_host = 0.;                           // source of the timestep upload
    std::vector<int> needs_fix_flux, needs_bounds; // blocks with physical (or periodic) faces
    // the boundary work of those blocks per stage output (0: stage 1's, 1: the state), as tasks of
    // k_bound_tasks grouped by phase: [bound_off[s][p], bound_off[s][p + 1]) in bound_dev[s]
    BoundTask* bound_dev[2] = {nullptr, nullptr};
    // the flux fixes of the blocks in needs_fix_flux, as tasks of k_fix_tasks (FixTask<FT>[n_fix])
    void* fix_dev = nullptr;
    int n_fix = 0, fix_max = 0;
    std::vector<int> bound_off[2];
    std::vector<long long> bound_max[2];
    bool any_exchange = false;                     // some block carries its ghost shell over
    // SMR: ghost-exchange and flux-correction tables (6 ints per entry) of the mesh the blocks form
    int* mesh_ghost = nullptr;
    int* mesh_flux = nullptr;
    long long n_ghost = 0, n_ghost_first = 0, n_flux = 0;
    std::vector<long long> ghost_phase_end;        // ends of the prolongation phases (one per level)
    // exchange of conserved variables with seeds (the kharma driver), else of primitives
    bool sync_cons = false;
    // CUDA graph of one step
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    size_t graph_launches = 0;
    int64_t launches = 0;
};

namespace {

inline cudaStream_t S(void* s) { return (cudaStream_t)s; }

// The mesh's ghost exchange: copies and restrictions, then the prolongations level by level
void enqueue_mesh_ghost(khb_batch* b, int stage, cudaStream_t st)
{
    LaunchCommon::mesh_ghost(b->nv, b->fix, b->mesh_ghost, 0, b->n_ghost_first, stage, st);
    long long begin = b->n_ghost_first;
    for (long long end : b->ghost_phase_end) {
        LaunchCommon::mesh_ghost(b->nv, b->fix, b->mesh_ghost, begin, end, stage, st);
        begin = end;
    }
    b->launches += 1 + (int64_t)b->ghost_phase_end.size();
}

// The kharma driver's exchange in the same phases (conserved variables and inversion seeds), then
// the inversion, floors and U = U(P) of every ghost zone it filled.  Stage s (0, 1): between the
// update and the cell half of the zone pass; s = -1: outside a stage, on the blocks' state.
template <typename FT>
void enqueue_mesh_cons(khb_batch* b, int s, cudaStream_t st)
{
    const int seed_sel = (s < 0) ? 0 : s, u_sel = (s < 0) ? 1 : s;
    LaunchCommon::mesh_ghost_cons(b->nv, b->fix, b->mesh_ghost, 0, b->n_ghost_first, seed_sel, u_sel, st);
    long long begin = b->n_ghost_first;
    for (long long end : b->ghost_phase_end) {
        LaunchCommon::mesh_ghost_cons(b->nv, b->fix, b->mesh_ghost, begin, end, seed_sel, u_sel, st);
        begin = end;
    }
    const bool kast = b->ctx[0]->ph.inverter == KHB_INVERTER_KASTAUN;
    Launch<FT>::mesh_ghost_cell(b->nv, kast, (const BatchBlock<FT>*)b->desc, b->mesh_ghost, b->n_ghost,
                                (s < 0) ? 1 : s, s < 0, st);
    b->launches += 2 + (int64_t)b->ghost_phase_end.size();
}

#define KHB_BCUDA(call)                                                                  \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return set_error(KHB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define KHB_BLAUNCHED(b, n)                                                              \
    do {                                                                                 \
        cudaError_t e_ = cudaGetLastError();                                             \
        if (e_ != cudaSuccess) return set_error(KHB_ERR_CUDA, std::string("batch launch: ") + cudaGetErrorString(e_)); \
        (b)->launches += (n);                                                            \
    } while (0)

void free_tables(khb_batch* b)
{
    cudaDeviceSynchronize();          // no batched kernel may still read the tables
    cudaFree(b->desc); b->desc = nullptr;
    cudaFree(b->fix); b->fix = nullptr;
    cudaFree(b->counts); b->counts = nullptr;
    for (int x = 0; x < 5; ++x) { cudaFree(b->tiles[x]); b->tiles[x] = nullptr; }
    for (int s = 0; s < 2; ++s) {
        cudaFree(b->bound_dev[s]); b->bound_dev[s] = nullptr;
        b->bound_off[s].clear(); b->bound_max[s].clear();
    }
    cudaFree(b->fix_dev); b->fix_dev = nullptr;
    b->n_fix = 0; b->fix_max = 0;
}

void drop_graph(khb_batch* b)
{
    if (b->gexec) cudaGraphExecDestroy(b->gexec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->gexec = nullptr;
    b->graph = nullptr;
}

// Face ranges of one direction as khb_get_flux covers them: [s, e+1] along dir, [s-1, e+1] across
void flux_range(const Dims& d, int dir, int lo[3], int cnt[3])
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

int build_bound_tasks(khb_batch* b);
template <typename FT> int build_fix_tasks(khb_batch* b);

// Descriptors and tile tables for the current tile shapes
template <typename FT>
int build_tables(khb_batch* b)
{
    free_tables(b);
    std::vector<BatchBlock<FT>> desc(b->nb);
    std::vector<FixupBlock> fix(b->nb);
    std::vector<int*> counts(b->nb);
    std::vector<int> tiles[5];
    for (int x = 0; x < b->nb; ++x) {
        khb_ctx* c = b->ctx[x];
        const Dims& d = c->d;
        BatchBlock<FT>& B = desc[x];
        std::memset((void*)&B, 0, sizeof(B));
        B.d = d; B.g = c->g; B.ph = c->ph;
        khb_fields P1, U1;
        std::memset(&P1, 0, sizeof(P1)); std::memset(&U1, 0, sizeof(U1));
        for (int p = 0; p < c->nv; ++p) {
            P1.v[p] = c->stageP + (size_t)p * d.N;
            U1.v[p] = c->stageU + (size_t)p * d.N;
        }
        const khb_fields Pin[2] = {b->P[x], P1}, Uin[2] = {b->U[x], U1};
        const khb_fields Pout[2] = {P1, b->P[x]}, Uout[2] = {U1, b->U[x]};
        for (int s = 0; s < 2; ++s) {
            ZoneArgs<FT>& a = B.za[s];
            a.Ps = Pin[s]; a.Us = Uin[s]; a.U0 = b->U[x]; a.Pout = Pout[s]; a.Uout = Uout[s];
            for (int q = 0; q < 3; ++q) { a.F[q] = (const FT*)c->F[q]; a.ctop[q] = (const FT*)c->ctop[q]; }
            a.pflag = b->pflag[x]; a.fflag = b->fflag[x];
            a.g0 = kRkGam0[s]; a.g1 = kRkGam1[s]; a.bdt = 0.;      // bdt: beta * dt, set on the device
            a.ndt_word = b->word;
            a.fail_count = c->fail_count; a.fail_list = c->fail_list;
            a.mode = 0;
            B.Pin[s] = Pin[s];
            fix[x].Pin[s] = Pin[s]; fix[x].Uin[s] = Uin[s];
            fix[x].P[s] = Pout[s]; fix[x].U[s] = Uout[s];
        }
        for (int q = 0; q < 3; ++q) { B.F[q] = (FT*)c->F[q]; B.ctop[q] = (FT*)c->ctop[q]; }
        const int kz = b->class_kz[b->cls[x]];
        for (int dir = 1; dir <= 3; ++dir) {
            int lo[3], cnt[3];
            flux_range(d, dir, lo, cnt);
            B.fbox[dir - 1] = make_box(lo[0], lo[1], lo[2], cnt[0], cnt[1], cnt[2], (kz && cnt[2] >= kz) ? kz : 0);
        }
        B.zbox = make_box(d.is, d.js, d.ks, d.ie - d.is + 1, d.je - d.js + 1, d.ke - d.ks + 1,
                          (kz && d.ke - d.ks + 1 >= kz) ? kz : 0);
        for (int q = 0; q < 4; ++q) {
            const Box& bx = (q < 3) ? B.fbox[q] : B.zbox;
            if (q < 3 && q + 1 > b->ndim) { B.tile0[q] = 0; continue; }
            B.tile0[q] = (unsigned)tiles[q].size();
            const unsigned n = box_blocks(bx);
            tiles[q].insert(tiles[q].end(), n, x);
        }
        // the fused plan's table: this block's faces of every direction, then its ghost shell in
        // tiles of 128 zones when it has an exchange face (entry = block | kind << 28)
        bool exch = false;
        for (int f = 0; f < 2 * d.ndim; ++f) if (d.bc[f] == KHB_BC_EXCHANGE) exch = true;
        for (int q = 0; q < 4; ++q) {
            B.tile0c[q] = (unsigned)tiles[4].size();
            unsigned n = 0;
            if (q < 3 && q + 1 <= b->ndim) n = box_blocks(B.fbox[q]);
            if (q == 3 && exch) {
                const long long shell = d.N - (long long)(d.ie - d.is + 1) * (d.je - d.js + 1) * (d.ke - d.ks + 1);
                n = (unsigned)((shell + 127) / 128);
            }
            tiles[4].insert(tiles[4].end(), n, x | (q << 28));
        }
        fix[x].d = d; fix[x].g = c->g; fix[x].ph = c->ph;
        fix[x].exch = 0;
        for (int f = 0; f < 2 * d.ndim; ++f) if (d.bc[f] == KHB_BC_EXCHANGE) fix[x].exch = 1;
        if (fix[x].exch) b->any_exchange = true;
        fix[x].pflag = b->pflag[x];
        fix[x].fail_count = c->fail_count; fix[x].fail_list = c->fail_list;
        counts[x] = c->fail_count;
    }
    KHB_BCUDA(cudaMalloc(&b->desc, sizeof(BatchBlock<FT>) * b->nb));
    KHB_BCUDA(cudaMemcpy(b->desc, desc.data(), sizeof(BatchBlock<FT>) * b->nb, cudaMemcpyHostToDevice));
    KHB_BCUDA(cudaMalloc((void**)&b->fix, sizeof(FixupBlock) * b->nb));
    KHB_BCUDA(cudaMemcpy(b->fix, fix.data(), sizeof(FixupBlock) * b->nb, cudaMemcpyHostToDevice));
    KHB_BCUDA(cudaMalloc((void**)&b->counts, sizeof(int*) * b->nb));
    KHB_BCUDA(cudaMemcpy(b->counts, counts.data(), sizeof(int*) * b->nb, cudaMemcpyHostToDevice));
    if (b->nb >= (1 << 28)) return set_error(KHB_ERR_ARG, "khb_batch: too many blocks for the fused plan's table");
    for (int q = 0; q < 5; ++q) {
        b->ntiles[q] = (unsigned)tiles[q].size();
        if (tiles[q].empty()) continue;
        KHB_BCUDA(cudaMalloc((void**)&b->tiles[q], sizeof(int) * tiles[q].size()));
        KHB_BCUDA(cudaMemcpy(b->tiles[q], tiles[q].data(), sizeof(int) * tiles[q].size(), cudaMemcpyHostToDevice));
    }
    int rc_b = build_bound_tasks(b);
    if (rc_b) return rc_b;
    if ((rc_b = build_fix_tasks<FT>(b))) return rc_b;
    // copies from pageable memory may return before they land, and the caller's non-blocking
    // streams do not wait for the legacy stream: the tables must be on the device before any
    // batched kernel reads them
    KHB_BCUDA(cudaDeviceSynchronize());
    // persistent grids: every SM holds as many CTAs as the kernel's registers allow
    for (int q = 0; q < 5; ++q) {
        const int occ = (q < 3) ? b->occ[q] : ((q == 3) ? std::min(b->occ[3], b->occ[4]) : b->occ[5]);
        const unsigned full = (unsigned)(b->nsm * std::max(occ, 1));
        b->grid[q] = b->persistent ? std::min(b->ntiles[q], full) : 0;
    }
    b->grid_fused_zone = b->persistent ? std::min(b->ntiles[3], (unsigned)(b->nsm * std::max(b->occ[6], 1))) : 0;
    drop_graph(b);
    return KHB_OK;
}

int rebuild(khb_batch* b) { return b->fp32 ? build_tables<float>(b) : build_tables<double>(b); }

// The boundaries of blocks with physical or periodic faces: each phase of the per-block boundary
// launches (faces by direction, ghost P->U, periodic images) for all those blocks in one launch
int enqueue_bounds(khb_batch* b, int s, cudaStream_t st)
{
    if (!b->bound_dev[s]) return KHB_OK;
    for (int p = 0; p < BOUND_PHASES; ++p) {
        const int n = b->bound_off[s][p + 1] - b->bound_off[s][p];
        if (!n) continue;
        LaunchCommon::bound_tasks(b->nv, b->bound_dev[s] + b->bound_off[s][p], n, b->bound_max[s][p], st);
        KHB_BLAUNCHED(b, 1);
    }
    return KHB_OK;
}

// The boundary tasks of each stage output, uploaded once with the other tables
int build_bound_tasks(khb_batch* b)
{
    for (int s = 0; s < 2; ++s) {
        std::vector<BoundTask> phases[BOUND_PHASES];
        for (int x : b->needs_bounds) {
            khb_ctx* c = b->ctx[x];
            khb_fields Po, Uo;
            if (s == 0) {
                std::memset(&Po, 0, sizeof(Po)); std::memset(&Uo, 0, sizeof(Uo));
                for (int p = 0; p < c->nv; ++p) {
                    Po.v[p] = c->stageP + (size_t)p * c->d.N;
                    Uo.v[p] = c->stageU + (size_t)p * c->d.N;
                }
            } else {
                Po = b->P[x]; Uo = b->U[x];
            }
            boundary_tasks(c, Po, Uo, phases);
        }
        std::vector<BoundTask> all;
        b->bound_off[s].assign(1, 0);
        b->bound_max[s].clear();
        for (int p = 0; p < BOUND_PHASES; ++p) {
            long long mx = 0;
            for (const BoundTask& t : phases[p]) mx = t.count > mx ? t.count : mx;
            all.insert(all.end(), phases[p].begin(), phases[p].end());
            b->bound_off[s].push_back((int)all.size());
            b->bound_max[s].push_back(mx);
        }
        if (all.empty()) continue;
        KHB_BCUDA(cudaMalloc((void**)&b->bound_dev[s], sizeof(BoundTask) * all.size()));
        KHB_BCUDA(cudaMemcpy(b->bound_dev[s], all.data(), sizeof(BoundTask) * all.size(), cudaMemcpyHostToDevice));
    }
    return KHB_OK;
}

// The flux fixes of all blocks with physical faces that need them, in one launch
template <typename FT>
int enqueue_fix_flux(khb_batch* b, cudaStream_t st)
{
    if (!b->n_fix) return KHB_OK;
    Launch<FT>::fix_tasks(b->nv, (const FixTask<FT>*)b->fix_dev, b->n_fix, b->fix_max, st);
    KHB_BLAUNCHED(b, 1);
    return KHB_OK;
}

// The fixes the per-block path makes (launch_fix_flux: polar x2 faces, then x1 inflow checks), as tasks
template <typename FT>
int build_fix_tasks(khb_batch* b)
{
    std::vector<FixTask<FT>> tasks;
    for (int x : b->needs_fix_flux) {
        khb_ctx* c = b->ctx[x];
        const Dims& d = c->d;
        FixTask<FT> t;
        std::memset((void*)&t, 0, sizeof(t));
        t.d = d; t.ph = c->ph;
        t.F1 = (FT*)c->F[0]; t.F2 = (FT*)c->F[1]; t.F3 = (FT*)c->F[2];
        const int nk = (d.ndim > 2) ? d.ke - d.ks + 3 : 1;
        if (d.ndim >= 2 && (c->ph.zero_polar_flux || (c->nv > 5 && c->ph.fix_polar_flux))) {
            for (int face = 2; face <= 3; ++face) {
                if (!phys_face(d.bc[face])) continue;
                t.x1 = 0; t.inner = face == 2; t.count = (d.ie - d.is + 3) * nk;
                tasks.push_back(t);
            }
        }
        const int nj = (d.ndim > 1) ? d.je - d.js + 3 : 1;
        if (c->ph.check_inflow_in && phys_face(d.bc[0])) { t.x1 = 1; t.inner = 1; t.count = nj * nk; tasks.push_back(t); }
        if (c->ph.check_inflow_out && phys_face(d.bc[1])) { t.x1 = 1; t.inner = 0; t.count = nj * nk; tasks.push_back(t); }
    }
    b->n_fix = (int)tasks.size();
    b->fix_max = 0;
    for (const auto& t : tasks) b->fix_max = t.count > b->fix_max ? t.count : b->fix_max;
    if (tasks.empty()) return KHB_OK;
    KHB_BCUDA(cudaMalloc(&b->fix_dev, sizeof(FixTask<FT>) * tasks.size()));
    KHB_BCUDA(cudaMemcpy(b->fix_dev, tasks.data(), sizeof(FixTask<FT>) * tasks.size(), cudaMemcpyHostToDevice));
    return KHB_OK;
}

// The fused plan: faces of all directions (with the resets and shell copies), the whole zone pass,
// fixups; the same device functions on the same data as the one-kernel-per-launch plan
template <typename FT>
int enqueue_stage_fused(khb_batch* b, int s, cudaStream_t st)
{
    const int stage = s + 1;
    const BatchBlock<FT>* desc = (const BatchBlock<FT>*)b->desc;
    Launch<FT>::batch_flux_all(b->recon, b->nv, desc, b->tiles[4], b->ntiles[4], b->grid[4], stage, b->counts, b->nb,
                               s == 1 ? b->word : nullptr, st);
    KHB_BLAUNCHED(b, 1);
    int rc;
    if ((rc = enqueue_fix_flux<FT>(b, st))) return rc;
    if (b->n_flux) {
        Launch<FT>::mesh_flux(b->nv, desc, b->mesh_flux, b->n_flux, st);
        KHB_BLAUNCHED(b, 1);
    }
    const int fused = M_ZONE_FUSED | ((b->ctx[0]->ph.inverter == KHB_INVERTER_KASTAUN) ? M_KASTAUN : 0);
    Launch<FT>::batch_zone(b->nv, fused, desc, b->tiles[3], b->ntiles[3], b->grid_fused_zone, stage,
                           s == 1 ? M_DT : 0, kRkBeta[s], b->dt_dev, st);
    KHB_BLAUNCHED(b, 1);
    LaunchCommon::batch_fixup(b->nv, b->fix, b->nb, stage, st);
    KHB_BLAUNCHED(b, 1);
    // the mesh's exchange, then the physical faces over the ghost rows it filled (the reference's
    // sync before its domain conditions, kharma_step.cpp:209-249)
    if (b->n_ghost) {
        enqueue_mesh_ghost(b, stage, st);
        KHB_BLAUNCHED(b, 0);
    }
    return enqueue_bounds(b, s, st);
}

template <typename FT>
int enqueue_stage(khb_batch* b, int s, cudaStream_t st)
{
    // the fused plan inverts in the pass that updates: the kharma driver's exchange needs the plain one
    if (b->plan == 1 && !(b->sync_cons && b->n_ghost)) return enqueue_stage_fused<FT>(b, s, st);
    const int stage = s + 1;
    const BatchBlock<FT>* desc = (const BatchBlock<FT>*)b->desc;
    LaunchCommon::batch_reset(b->counts, b->nb, s == 1 ? b->word : nullptr, st);
    KHB_BLAUNCHED(b, 1);
    for (int dir = 1; dir <= b->ndim; ++dir) {
        Launch<FT>::batch_flux(b->recon, b->nv, dir, desc, b->tiles[dir - 1], b->ntiles[dir - 1], b->grid[dir - 1],
                               stage, st);
        KHB_BLAUNCHED(b, 1);
    }
    int rc;
    if ((rc = enqueue_fix_flux<FT>(b, st))) return rc;
    if (b->n_flux) {
        Launch<FT>::mesh_flux(b->nv, desc, b->mesh_flux, b->n_flux, st);
        KHB_BLAUNCHED(b, 1);
    }
    if (b->any_exchange) {
        LaunchCommon::batch_ghost_copy(b->nv, b->fix, b->nb, stage, st);
        KHB_BLAUNCHED(b, 1);
    }
    Launch<FT>::batch_zone(b->nv, M_UPDATE, desc, b->tiles[3], b->ntiles[3], b->grid[3], stage, 0, kRkBeta[s],
                           b->dt_dev, st);
    KHB_BLAUNCHED(b, 1);
    const bool cons = b->sync_cons && b->n_ghost;
    if (cons) {
        // the kharma driver: the updated conserved state and the seeds cross before any inversion
        // (kharma_step.cpp:209-236), and the ghost zones are inverted like the interior
        enqueue_mesh_cons<FT>(b, s, st);
        KHB_BLAUNCHED(b, 0);
    }
    const int cell = M_ZONE_CELL | ((b->ctx[0]->ph.inverter == KHB_INVERTER_KASTAUN) ? M_KASTAUN : 0);
    Launch<FT>::batch_zone(b->nv, cell, desc, b->tiles[3], b->ntiles[3], b->grid[3], stage,
                           s == 1 ? M_DT : 0, kRkBeta[s], b->dt_dev, st);
    KHB_BLAUNCHED(b, 1);
    LaunchCommon::batch_fixup(b->nv, b->fix, b->nb, stage, st);
    KHB_BLAUNCHED(b, 1);
    // the mesh's exchange, then the physical faces over the ghost rows it filled (the reference's
    // sync before its domain conditions, kharma_step.cpp:209-249)
    if (b->n_ghost && !cons) {
        enqueue_mesh_ghost(b, stage, st);
        KHB_BLAUNCHED(b, 0);
    }
    return enqueue_bounds(b, s, st);
}

int enqueue_stage_any(khb_batch* b, int s, cudaStream_t st)
{
    return b->fp32 ? enqueue_stage<float>(b, s, st) : enqueue_stage<double>(b, s, st);
}

int upload_dt(khb_batch* b, double dt, cudaStream_t st)
{
    b->dt_host = dt;
    KHB_BCUDA(cudaMemcpyAsync(b->dt_dev, &b->dt_host, sizeof(double), cudaMemcpyHostToDevice, st));
    return KHB_OK;
}

int query_occupancy(khb_batch* b)
{
    int dev = 0;
    KHB_BCUDA(cudaGetDevice(&dev));
    KHB_BCUDA(cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, dev));
    for (int dir = 1; dir <= 3; ++dir)
        b->occ[dir - 1] = b->fp32 ? Launch<float>::batch_flux(b->recon, b->nv, dir, nullptr, nullptr, 0, 0, 1, 0)
                                  : Launch<double>::batch_flux(b->recon, b->nv, dir, nullptr, nullptr, 0, 0, 1, 0);
    const int modes[2] = {M_UPDATE, M_ZONE_CELL};
    for (int m = 0; m < 2; ++m)
        b->occ[3 + m] = b->fp32 ? Launch<float>::batch_zone(b->nv, modes[m], nullptr, nullptr, 0, 0, 1, 0, 1., nullptr, 0)
                                : Launch<double>::batch_zone(b->nv, modes[m], nullptr, nullptr, 0, 0, 1, 0, 1., nullptr, 0);
    b->occ[5] = b->fp32 ? Launch<float>::batch_flux_all(b->recon, b->nv, nullptr, nullptr, 0, 0, 1, nullptr, 0, nullptr, 0)
                        : Launch<double>::batch_flux_all(b->recon, b->nv, nullptr, nullptr, 0, 0, 1, nullptr, 0, nullptr, 0);
    b->occ[6] = b->fp32 ? Launch<float>::batch_zone(b->nv, M_ZONE_FUSED, nullptr, nullptr, 0, 0, 1, 0, 1., nullptr, 0)
                        : Launch<double>::batch_zone(b->nv, M_ZONE_FUSED, nullptr, nullptr, 0, 0, 1, 0, 1., nullptr, 0);
    KHB_BCUDA(cudaGetLastError());
    return KHB_OK;
}

// Time reps runs of stage 1 (it writes only the stage scratch, the flags and the failed-zone
// lists, never the state) and return the median in ms
int time_stage1(khb_batch* b, int reps, cudaStream_t st, float* ms)
{
    cudaEvent_t e0, e1;
    KHB_BCUDA(cudaEventCreate(&e0));
    KHB_BCUDA(cudaEventCreate(&e1));
    std::vector<float> t;
    int rc = KHB_OK;
    for (int r = 0; r <= reps && rc == KHB_OK; ++r) {
        cudaEventRecord(e0, st);
        rc = enqueue_stage_any(b, 0, st);
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess) rc = set_error(KHB_ERR_CUDA, "khb_batch_autotune: stage failed");
        float x = 0.f;
        cudaEventElapsedTime(&x, e0, e1);
        if (r > 0) t.push_back(x);            // the first run warms up
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    std::sort(t.begin(), t.end());
    *ms = t[t.size() / 2];
    return KHB_OK;
}

} // namespace

extern "C" {

int khb_batch_create(khb_ctx* const* blocks, int nblocks, const khb_fields* P, const khb_fields* U,
                     int32_t* const* pflag, int32_t* const* fflag, khb_batch** out)
{
    if (!blocks || nblocks < 1 || !P || !U || !pflag || !fflag || !out)
        return set_error(KHB_ERR_ARG, "khb_batch_create: NULL argument or no blocks");
    *out = nullptr;
    khb_batch* b = new khb_batch();
    b->nb = nblocks;
    for (int x = 0; x < nblocks; ++x) {
        khb_ctx* c = blocks[x];
        if (!c || !c->geom_set) { delete b; return set_error(KHB_ERR_STATE, "khb_batch_create: block without geometry"); }
        if (c->ph.fofc) { delete b; return set_error(KHB_ERR_UNSUPPORTED, "khb_batch_create: fofc blocks are stepped with khb_step"); }
        if (c->ph.ct_scheme) { delete b; return set_error(KHB_ERR_UNSUPPORTED, "khb_batch_create: B_CT blocks are stepped with khb_ct_step"); }
        if (c->cfg.recon > KHB_RECON_PPM || c->ph.weno_lower || c->ph.recon_fallback) {
            delete b;
            return set_error(KHB_ERR_UNSUPPORTED, "khb_batch_create: batches use donor cell, linear MC, WENO5 or PPM "
                                                  "without lowering or fallback");
        }
        if (x == 0) {
            b->nv = c->nv; b->recon = c->cfg.recon; b->fp32 = c->fp32; b->ndim = c->d.ndim;
        } else if (c->nv != b->nv || c->cfg.recon != b->recon || c->fp32 != b->fp32 || c->d.ndim != b->ndim ||
                   c->cfg.riemann != blocks[0]->cfg.riemann || c->ph.inverter != blocks[0]->ph.inverter) {
            delete b;
            return set_error(KHB_ERR_ARG, "khb_batch_create: blocks differ in nvar, dimension, reconstruction, "
                                          "Riemann solver, inverter or precision");
        }
        for (int p = 0; p < c->nv; ++p)
            if (!P[x].v[p] || !U[x].v[p]) { delete b; return set_error(KHB_ERR_ARG, "khb_batch_create: NULL field"); }
        if (!pflag[x] || !fflag[x]) { delete b; return set_error(KHB_ERR_ARG, "khb_batch_create: NULL flags"); }
        b->ctx.push_back(c);
        b->P.push_back(P[x]); b->U.push_back(U[x]);
        b->pflag.push_back(pflag[x]); b->fflag.push_back(fflag[x]);
        // size class
        const std::array<int, 3> sz = {c->d.nx1, c->d.nx2, c->d.nx3};
        int k = -1;
        for (size_t q = 0; q < b->class_size.size(); ++q) if (b->class_size[q] == sz) k = (int)q;
        if (k < 0) { k = (int)b->class_size.size(); b->class_size.push_back(sz); b->class_kz.push_back(0); }
        b->cls.push_back(k);
        // per-block launches that stay outside the batched kernels
        bool fixes = false, bounds = false;
        for (int f = 0; f < 2 * c->d.ndim; ++f) {
            if (phys_face(c->d.bc[f])) bounds = true;
            if (c->d.bc[f] == KHB_BC_PERIODIC) bounds = true;
        }
        if (c->d.ndim >= 2 && (c->ph.zero_polar_flux || (c->nv > 5 && c->ph.fix_polar_flux)) &&
            (phys_face(c->d.bc[2]) || phys_face(c->d.bc[3]))) fixes = true;
        if ((c->ph.check_inflow_in && phys_face(c->d.bc[0])) || (c->ph.check_inflow_out && phys_face(c->d.bc[1])))
            fixes = true;
        if (fixes) b->needs_fix_flux.push_back(x);
        if (bounds) b->needs_bounds.push_back(x);
    }
    int rc = KHB_OK;
    if (cudaMalloc((void**)&b->dt_dev, sizeof(double)) != cudaSuccess ||
        cudaMalloc((void**)&b->word, sizeof(unsigned long long)) != cudaSuccess) {
        rc = set_error(KHB_ERR_CUDA, "khb_batch_create: allocation failed");
    }
    if (!rc) rc = query_occupancy(b);
    if (!rc) rc = rebuild(b);
    if (rc) { cudaFree(b->dt_dev); cudaFree(b->word); free_tables(b); delete b; return rc; }
    *out = b;
    return KHB_OK;
}

int khb_batch_destroy(khb_batch* b)
{
    if (!b) return KHB_OK;
    drop_graph(b);
    free_tables(b);
    cudaFree(b->mesh_ghost);
    cudaFree(b->mesh_flux);
    cudaFree(b->dt_dev);
    cudaFree(b->word);
    delete b;
    return KHB_OK;
}

int khb_batch_set_mesh(khb_batch* b, const int32_t* ghost, int64_t n_ghost, int64_t n_ghost_first,
                       const int32_t* flux, int64_t n_flux)
{
    if (!b) return set_error(KHB_ERR_ARG, "khb_batch_set_mesh: NULL batch");
    if (n_ghost < 0 || n_flux < 0 || n_ghost_first < 0 || n_ghost_first > n_ghost ||
        (n_ghost && !ghost) || (n_flux && !flux))
        return set_error(KHB_ERR_ARG, "khb_batch_set_mesh: bad table sizes");
    if (b->nv != 5) return set_error(KHB_ERR_UNSUPPORTED, "khb_batch_set_mesh: SMR meshes of hydro blocks (nvar 5) only");
    // every index is checked here, so the kernels read and write inside the blocks' arrays
    for (int64_t e = 0; e < n_ghost; ++e) {
        const int32_t* t = ghost + 6 * e;
        if (t[0] < 0 || t[0] >= b->nb || t[3] < 0 || t[3] >= b->nb || t[2] < 0 || t[2] > 2)
            return set_error(KHB_ERR_ARG, "khb_batch_set_mesh: ghost entry with a bad block or op");
        const Dims& dd = b->ctx[t[0]]->d;
        const Dims& ds = b->ctx[t[3]]->d;
        if (t[1] < 0 || t[1] >= dd.N) return set_error(KHB_ERR_ARG, "khb_batch_set_mesh: ghost entry outside its block");
        // the source stencil: the zone, +1 per active direction (restrict), +-1 (prolong)
        long long lo = t[4], hi = t[4];
        const long long st[3] = {1, ds.sj, ds.sk};
        for (int d = 0; d < ds.ndim; ++d) {
            if (t[2] == 1) hi += st[d];
            if (t[2] == 2) { lo -= st[d]; hi += st[d]; }
        }
        if (lo < 0 || hi >= ds.N) return set_error(KHB_ERR_ARG, "khb_batch_set_mesh: ghost source outside its block");
        if ((e < n_ghost_first) != (t[2] != 2))
            return set_error(KHB_ERR_ARG, "khb_batch_set_mesh: prolongations must follow copies and restrictions");
        if (t[2] == 2) {
            const int phase = t[5] >> 8;
            if (phase < 0 || (e > n_ghost_first && phase < (ghost[6 * (e - 1) + 5] >> 8)))
                return set_error(KHB_ERR_ARG, "khb_batch_set_mesh: prolongations must come in phase order");
        }
    }
    std::vector<long long> phase_end;
    for (int64_t e = n_ghost_first; e < n_ghost; ++e)
        if (e + 1 == n_ghost || (ghost[6 * (e + 1) + 5] >> 8) != (ghost[6 * e + 5] >> 8)) phase_end.push_back(e + 1);
    for (int64_t e = 0; e < n_flux; ++e) {
        const int32_t* t = flux + 6 * e;
        if (t[0] < 0 || t[0] >= b->nb || t[3] < 0 || t[3] >= b->nb || t[1] < 1 || t[1] > b->ndim)
            return set_error(KHB_ERR_ARG, "khb_batch_set_mesh: flux entry with a bad block or direction");
        const Dims& dc = b->ctx[t[0]]->d;
        const Dims& df = b->ctx[t[3]]->d;
        const long long t1 = (t[1] == 1) ? df.sj : 1, t2 = (t[1] == 3) ? df.sj : df.sk;
        const long long hi = t[4] + t1 + ((df.ndim > 2) ? t2 : 0);
        if (t[2] < 0 || t[2] >= dc.N || t[4] < 0 || hi >= df.N)
            return set_error(KHB_ERR_ARG, "khb_batch_set_mesh: flux entry outside its blocks");
    }
    drop_graph(b);
    cudaFree(b->mesh_ghost); cudaFree(b->mesh_flux);
    b->mesh_ghost = nullptr; b->mesh_flux = nullptr;
    b->n_ghost = b->n_ghost_first = b->n_flux = 0;
    b->ghost_phase_end.clear();
    if (n_ghost) {
        KHB_BCUDA(cudaMalloc((void**)&b->mesh_ghost, sizeof(int32_t) * 6 * (size_t)n_ghost));
        KHB_BCUDA(cudaMemcpy(b->mesh_ghost, ghost, sizeof(int32_t) * 6 * (size_t)n_ghost, cudaMemcpyHostToDevice));
    }
    if (n_flux) {
        KHB_BCUDA(cudaMalloc((void**)&b->mesh_flux, sizeof(int32_t) * 6 * (size_t)n_flux));
        KHB_BCUDA(cudaMemcpy(b->mesh_flux, flux, sizeof(int32_t) * 6 * (size_t)n_flux, cudaMemcpyHostToDevice));
    }
    KHB_BCUDA(cudaDeviceSynchronize());
    b->n_ghost = n_ghost; b->n_ghost_first = n_ghost_first; b->n_flux = n_flux;
    b->ghost_phase_end = phase_end;
    return KHB_OK;
}

int khb_batch_mesh_exchange(khb_batch* b, void* stream)
{
    KHB_RANGE("khb_batch_mesh_exchange");
    if (!b) return set_error(KHB_ERR_ARG, "khb_batch_mesh_exchange: NULL batch");
    if (b->n_ghost) {
        if (b->sync_cons) {
            if (b->fp32) enqueue_mesh_cons<float>(b, -1, S(stream));
            else enqueue_mesh_cons<double>(b, -1, S(stream));
        } else {
            enqueue_mesh_ghost(b, 2, S(stream));
        }
        KHB_BCUDA(cudaGetLastError());
        int rc;
        if ((rc = enqueue_bounds(b, 1, S(stream)))) return rc;
    }
    return KHB_OK;
}

int khb_batch_set_mesh_sync(khb_batch* b, int mode)
{
    if (!b) return set_error(KHB_ERR_ARG, "khb_batch_set_mesh_sync: NULL batch");
    if (mode != KHB_SYNC_PRIMS && mode != KHB_SYNC_CONSERVED)
        return set_error(KHB_ERR_ARG, "khb_batch_set_mesh_sync: mode is KHB_SYNC_PRIMS or KHB_SYNC_CONSERVED");
    if (b->sync_cons != (mode == KHB_SYNC_CONSERVED)) drop_graph(b);      // a captured step runs the other exchange
    b->sync_cons = mode == KHB_SYNC_CONSERVED;
    return KHB_OK;
}

int khb_batch_step(khb_batch* b, double dt, void* stream)
{
    KHB_RANGE("khb_batch_step");
    if (!b) return set_error(KHB_ERR_ARG, "khb_batch_step: NULL batch");
    int rc;
    if ((rc = upload_dt(b, dt, S(stream)))) return rc;
    if ((rc = enqueue_stage_any(b, 0, S(stream)))) return rc;
    return enqueue_stage_any(b, 1, S(stream));
}

int khb_batch_step_graph(khb_batch* b, double dt, void* stream)
{
    KHB_RANGE("khb_batch_step_graph");
    if (!b) return set_error(KHB_ERR_ARG, "khb_batch_step_graph: NULL batch");
    cudaStream_t st = S(stream);
    if (!st) return set_error(KHB_ERR_ARG, "khb_batch_step_graph: needs a non-default stream to capture");
    if (!b->gexec) {
        const int64_t l0 = b->launches;
        KHB_BCUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_stage_any(b, 0, st);
        if (!rc) rc = enqueue_stage_any(b, 1, st);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(st, &g);
        b->launches = l0;
        if (rc) { if (g) cudaGraphDestroy(g); return rc; }
        if (e != cudaSuccess) return set_error(KHB_ERR_CUDA, std::string("khb_batch_step_graph: capture: ") + cudaGetErrorString(e));
        b->graph = g;
        size_t n = 0;
        KHB_BCUDA(cudaGraphGetNodes(g, nullptr, &n));
        b->graph_launches = n;
        KHB_BCUDA(cudaGraphInstantiate(&b->gexec, g, 0));
    }
    int rc;
    if ((rc = upload_dt(b, dt, st))) return rc;
    KHB_BCUDA(cudaGraphLaunch(b->gexec, st));
    b->launches += (int64_t)b->graph_launches;
    return KHB_OK;
}

int khb_batch_get_min_ndt(khb_batch* b, double* min_ndt_host, void* stream)
{
    if (!b || !min_ndt_host) return set_error(KHB_ERR_ARG, "khb_batch_get_min_ndt: NULL argument");
    unsigned long long bits = 0;
    KHB_BCUDA(cudaMemcpyAsync(&bits, b->word, sizeof(bits), cudaMemcpyDeviceToHost, S(stream)));
    KHB_BCUDA(cudaStreamSynchronize(S(stream)));
    std::memcpy(min_ndt_host, &bits, sizeof(double));
    return KHB_OK;
}

int khb_batch_classes(khb_batch* b, int32_t* nclasses, int32_t* sizes, int32_t* kz, int max)
{
    if (!b || !nclasses) return set_error(KHB_ERR_ARG, "khb_batch_classes: NULL argument");
    *nclasses = (int32_t)b->class_size.size();
    for (int q = 0; q < *nclasses && q < max; ++q) {
        if (sizes) for (int a = 0; a < 3; ++a) sizes[3 * q + a] = b->class_size[q][a];
        if (kz) kz[q] = b->class_kz[q];
    }
    return KHB_OK;
}

int khb_batch_set_tuning(khb_batch* b, int size_class, int kz, int persistent)
{
    if (!b) return set_error(KHB_ERR_ARG, "khb_batch_set_tuning: NULL batch");
    if (size_class >= (int)b->class_size.size()) return set_error(KHB_ERR_ARG, "khb_batch_set_tuning: no such class");
    if (kz != 0 && kz != 1 && kz != 2 && kz != 4) return set_error(KHB_ERR_ARG, "khb_batch_set_tuning: kz must be 0, 1, 2 or 4");
    if (size_class >= 0) b->class_kz[size_class] = kz;
    b->persistent = persistent ? 1 : 0;
    return rebuild(b);
}

int khb_batch_autotune(khb_batch* b, int reps, int32_t* kz_out, int32_t* persistent_out, void* stream)
{
    KHB_RANGE("khb_batch_autotune");
    if (!b || reps < 1) return set_error(KHB_ERR_ARG, "khb_batch_autotune: bad argument");
    cudaStream_t st = S(stream);
    int rc;
    if ((rc = upload_dt(b, 0., st))) return rc;       // stage 1 reads dt; its value does not change the timing
    const int64_t l0 = b->launches;
    // tile shape per size class, by coordinate descent over the classes
    for (size_t q = 0; q < b->class_size.size(); ++q) {
        int best = b->class_kz[q];
        float best_ms = 1e30f;
        for (int kz : {1, 2, 4}) {
            if (kz > 1 && b->class_size[q][2] < kz) continue;
            b->class_kz[q] = kz;
            if ((rc = rebuild(b))) return rc;
            float ms = 0.f;
            if ((rc = time_stage1(b, reps, st, &ms))) return rc;
            if (ms < best_ms) { best_ms = ms; best = kz; }
        }
        b->class_kz[q] = best;
    }
    // then the launch mode
    int best_p = 0;
    float best_ms = 1e30f;
    for (int p : {0, 1}) {
        b->persistent = p;
        if ((rc = rebuild(b))) return rc;
        float ms = 0.f;
        if ((rc = time_stage1(b, reps, st, &ms))) return rc;
        if (ms < best_ms) { best_ms = ms; best_p = p; }
    }
    b->persistent = best_p;
    if ((rc = rebuild(b))) return rc;
    // then the launch plan (the tables serve both)
    int best_plan = 0;
    best_ms = 1e30f;
    for (int plan : {0, 1}) {
        b->plan = plan;
        float ms = 0.f;
        if ((rc = time_stage1(b, reps, st, &ms))) return rc;
        if (ms < best_ms) { best_ms = ms; best_plan = plan; }
    }
    b->plan = best_plan;
    drop_graph(b);
    b->launches = l0;
    if (kz_out) for (size_t q = 0; q < b->class_size.size(); ++q) kz_out[q] = b->class_kz[q];
    if (persistent_out) *persistent_out = b->persistent;
    return KHB_OK;
}

int khb_batch_set_plan(khb_batch* b, int plan)
{
    if (!b) return set_error(KHB_ERR_ARG, "khb_batch_set_plan: NULL batch");
    if (plan != 0 && plan != 1) return set_error(KHB_ERR_ARG, "khb_batch_set_plan: plan must be 0 or 1");
    b->plan = plan;
    drop_graph(b);
    return KHB_OK;
}

int khb_batch_get_plan(khb_batch* b, int32_t* plan)
{
    if (!b || !plan) return set_error(KHB_ERR_ARG, "khb_batch_get_plan: NULL argument");
    *plan = b->plan;
    return KHB_OK;
}

int64_t khb_batch_launch_count(khb_batch* b) { return b ? b->launches : 0; }

} // extern "C"

// khb_internal.hpp -- the context object and host helpers shared by the host units of libkhb
// (khb_api.cu, khb_batch.cu).  Not part of the C ABI.
#pragma once

#include "khb_types.cuh"

#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

// A named NVTX range around one C-ABI call, the counterpart of the reference's Flag/EndFlag timer
// regions (types.hpp:286-293): it shows each call on a profiler's timeline and costs a test of an
// unset pointer when no profiler is attached (header-only NVTX v3, no library to link)
struct KhbRange {
    explicit KhbRange(const char* name) { nvtxRangePushA(name); }
    ~KhbRange() { nvtxRangePop(); }
    KhbRange(const KhbRange&) = delete;
    KhbRange& operator=(const KhbRange&) = delete;
};
#define KHB_RANGE(name) KhbRange khb_range_scope_(name)

struct khb_ctx {
    khb_config cfg;
    khb::Dims d;
    khb::Phys ph;
    khb::DevGeom g;
    int nv;
    bool fp32;
    void* F[3];            // raw face fluxes, [nv][N] of FT
    void* ctop[3];         // max(cmax, cmin) per face, [N] of FT
    void* emf;             // corner EMFs for khb_flux_ct, [3][N] of FT
    double* stageP;        // intermediate RK stage
    double* stageU;
    unsigned long long* words;   // [0] min zone dt bits, [1] max divB bits
    int* fail_count;
    int* fail_list;
    double* geo_d;
    float* geo_f;
    bool geom_set;
    int64_t launches;
    unsigned long long dbl_max_bits;   // host source of the reduction reset (outlives async copies)
    int zone_split;        // zone pass as 1 kernel (0), 2 (1: update; inversion+floors+P->U) or
                           // 3 (2: update; inversion; floors+P->U)
    // EMHD / implicit solve
    double* conn_d;        // connection Gamma^lam_{mu nu}, [64][n2][n1] with index lam*16 + mu*4 + nu
    double* emhd_tmp;      // EMHD::AddSource temporaries u_mu, Theta: [5][N]
    double* fix_buf;       // FixSolve replacement values: [7][N]
    unsigned long long* imp_words;   // implicit-solve reductions, IMP_WORDS entries
    double* F10[3];        // EMHD face fluxes, [10][N] per direction
    double* dudt10;        // EMHD dU/dt of an ImEx stage, [10][N]
    int32_t* fofc_flag;    // first-order flux correction flags, [N] (when fofc is on)
    // device-resident timestep: state [dt, t, dt_last] and the schedule parameters
    double* dt_state;
    const double* dt_active;          // set while a step reads its dt from dt_state
    double dt_cfl, dt_min, dt_max_increase;
    // CUDA graph of one step with the device timestep, for the state it was captured with
    cudaGraph_t graph;
    cudaGraphExec_t gexec;
    khb_fields graph_P, graph_U;
    int32_t* graph_pflag;
    int32_t* graph_fflag;
    int64_t graph_launches;
    // adjoint scratch (khb_adjoint_step): face-flux adjoints [3][nv][N], the updated-state adjoint
    // [nv][N] and the intermediate stage's adjoints [2][nv][N]; flags of the recomputed stage [2][N]
    double* adj_buf;
    int32_t* adj_flags;
    double* adj_red;       // partial sums of khb_flux_dot
    // adjoint through the floors: the fluid primitives each recomputed stage inverted, before the
    // floors changed them ([2 stages][5][N]), the recomputed second stage ([2][nv][N]: P, U) and its
    // flags ([2][N]: pflag, fflag); prefloor_dst, set only while the adjoint recomputes a stage, makes
    // the zone pass run split and copy its inverted primitives there before the floors
    double* adj_pf;
    double* adj_s2;
    int32_t* adj_flags2;
    double* prefloor_dst;
    // B_CT: zone-centred EMFs [3][N] of FT, the intermediate stage's face field [3][N], and the face
    // field a zone pass in progress reads (set only inside khb_ct_stage)
    void* ct_emfc;
    double* ct_stageBf;
    const double* ct_bf[3];
    bool ct_active;
};


namespace khb {

// Parthenon "rk2" low-storage weights: gam0 = {0, 1/2}, gam1 = {1, 1/2}, beta = {1, 1/2}
constexpr double kRkGam0[2] = {0.0, 0.5}, kRkGam1[2] = {1.0, 0.5}, kRkBeta[2] = {1.0, 0.5};

// Record an error message for khb_last_error and return code
int set_error(int code, const std::string& msg);
// Flux fixes and ghost zones of one block, as khb_stage issues them
int ctx_fix_flux(khb_ctx* ctx, cudaStream_t st);
int ctx_boundaries(khb_ctx* ctx, const khb_fields& P, const khb_fields& U, cudaStream_t st);
// ctx_boundaries as tasks of k_bound_tasks, by phase (phases: BOUND_PHASES vectors)
void boundary_tasks(khb_ctx* ctx, const khb_fields& P, const khb_fields& U, std::vector<BoundTask>* phases);
// B_CT stage pieces (khb_ct.cu): edge EMFs from the stage's face fluxes and primitives, and the face
// update Bf_out = gam0 Bf_s + gam1 Bf_0 + beta dt dBf/dt
int ct_emf(khb_ctx* ctx, const khb_fields& Ps, cudaStream_t st);
int ct_face_boundaries(khb_ctx* ctx, const khb_fields& Bf, cudaStream_t st);
int ct_face_update(khb_ctx* ctx, int stage, double dt, const khb_fields& Bs, const khb_fields& B0,
                   const khb_fields& Bout, cudaStream_t st);

} // namespace khb

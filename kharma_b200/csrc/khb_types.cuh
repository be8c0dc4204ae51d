// khb_types.cuh -- plain structs shared by the host side (khb_api.cu) and the kernels, and the
// launcher interface the precision-specific translation units implement.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/khb.h"

namespace khb {

// Floors::Prescription (floors.hpp:100-117); same layout as khb_floors
struct Prescription {
    double rho_min_const, u_min_const;
    double rho_min_geom, u_min_geom, r_char;
    double bsq_over_rho_max, bsq_over_u_max, u_over_rho_max;
    double ktot_max, gamma_max;
    int32_t use_r_char, temp_adjust_u, adjust_k, radius_dependent_floors;
    double floors_switch_r;
};

struct Dims {
    int n1, n2, n3, ndim;
    int is, ie, js, je, ks, ke;
    int nx1, nx2, nx3;
    long long N;
    long long sj, sk;
    int bc[6];
    // status word of the bounds-checked build (KHB_BOUNDS_CHECK): the first out-of-range index a
    // checked access met, with its site; unused otherwise
    unsigned long long* chk;
};

// Sites of the bounds-checked accesses (the top 16 bits of the status word)
enum { CHK_FLUX_STENCIL = 1, CHK_FLUX_STORE = 2, CHK_ZONE_FLUX = 3, CHK_ZONE_CT = 4, CHK_FIXUP = 5,
       CHK_BC = 6, CHK_PERIODIC = 7, CHK_GEOM = 8 };

// Index check of the bounds-checked build (-DKHB_BOUNDS_CHECK=1, the stand-in for a memory checker):
// an index outside [0, n) is recorded in the status word (site << 48 | low 48 bits of the index, the
// first one wins) and replaced by 0, so the access stays inside its array and nothing traps.  In the
// regular build it is the identity.
#ifndef KHB_BOUNDS_CHECK
#define KHB_BOUNDS_CHECK 0
#endif
__host__ __device__ __forceinline__ long long kchk(const Dims& d, long long x, long long n, int site)
{
#if KHB_BOUNDS_CHECK && defined(__CUDA_ARCH__)
    if (x < 0 || x >= n) {
        if (d.chk) atomicCAS(d.chk, 0ull, ((unsigned long long)site << 48) | ((unsigned long long)x & 0xffffffffffffull));
        return 0;
    }
#else
    (void)d; (void)n; (void)site;
#endif
    return x;
}

struct DevGeom {
    int G1, G2, n1;
    long long gs;                          // component stride of the location tables, G1*G2
    const double* gcov[4];                 // face1, face2, face3, centre: [16][G2][G1]
    const double* gcon[4];
    const double* gdet[4];                 // [G2][G1]
    const float* gcov_f[3];                // FP32 copies of the face tables
    const float* gcon_f[3];
    const float* gdet_f[3];
    const double* gdet_conn;               // [64][n2][n1], index (nu*4+lam)*4+mu as gdet_conn(nu,lam,mu)
    const double* rcen;                    // [n2][n1]
    const double* floor_rho;               // geometric density floor per zone centre, [n2][n1]
    const double* floor_u;                 // geometric internal-energy floor, [n2][n1]
};

struct Phys {
    double gam;
    int riemann, recon_floors, spherical, cart_minkowski;
    int floors_on, frame, iter_max, fix_avg, fix_atmo;
    double err_tol;
    double dx1, dx2, dx3;
    int zero_polar_flux, fix_polar_flux, check_inflow_in, check_inflow_out;
    int inverter;                          // KHB_INVERTER_*
    int fofc, fofc_polar_cells;            // first-order flux correction
    double fofc_r_mark;                    // r_horizon + fofc/eh_buffer (spherical coordinates)
    int ct_scheme;                         // KHB_CT_* (B_CT face-centred field when nonzero)
    int recon_extra;                       // EX_* scheme of the RECON_EXTRA flux kernels
    int weno_lower;                        // WENO5 lowered to MC: 1 near X1 block edges, 2 near the poles
    int recon_fallback;                    // faces whose reconstructed states hit the floors take PPM
    Prescription fl;
    Prescription fl_inner;                 // r < fl.floors_switch_r when fl.radius_dependent_floors
    double frame_switch_r, frame_switch_beta;
    int fofc_glf, fofc_source;             // fofc/use_glf, fofc/use_source_term
};

enum { M_UPDATE = 1, M_UTOP = 2, M_FLOORS = 4, M_PTOU = 8, M_DT = 16, M_FAILLIST = 32 };
// The whole zone pass in one kernel, or its two halves (update; inversion + floors + P->U)
enum { M_ZONE_CELL = M_UTOP | M_FLOORS | M_PTOU | M_FAILLIST, M_ZONE_FUSED = M_UPDATE | M_ZONE_CELL };
// ... or in three (update; inversion; floors + P->U)
enum { M_ZONE_FLOORS = M_FLOORS | M_PTOU | M_FAILLIST };
// Inversion by the Kastaun scheme instead of 1D_W (a compile-time variant of the kernels with M_UTOP)
enum { M_KASTAUN = 64 };
// B_CT: the zone B comes from the face field (ZoneArgs::Bf) instead of the flux-CT divergence; run
// through the run-time-mode kernel (MODE = 0)
enum { M_BCT = 128 };
// Ghost zones of a B_CT mesh block (compile-time only): without M_UPDATE, U_B is rebuilt from the
// faces before the inversion, and the last ghost layer of a direction, whose upper face the arrays
// do not hold, takes B from its lower face
enum { M_GHOSTB = 256 };

struct Box {
    int lo_i, lo_j, lo_k, cnt_i, cnt_j, cnt_k;
    unsigned np;      // cnt_i * cnt_j
    unsigned nbp;     // blocks across the plane
    int kz;           // k planes per block (1, 2 or 4)
    int pshift;       // log2(128 / kz): plane positions per block = 1 << pshift
};
inline Box make_box(int lo_i, int lo_j, int lo_k, int cnt_i, int cnt_j, int cnt_k, int kz = 0)
{
    Box b;
    b.lo_i = lo_i; b.lo_j = lo_j; b.lo_k = lo_k; b.cnt_i = cnt_i; b.cnt_j = cnt_j; b.cnt_k = cnt_k;
    b.np = (unsigned)cnt_i * (unsigned)cnt_j;
    if (kz <= 0) kz = (cnt_k >= 4) ? 4 : 1;
    b.kz = kz;
    b.pshift = (kz == 4) ? 5 : ((kz == 2) ? 6 : 7);
    const unsigned per = 1u << b.pshift;
    b.nbp = (b.np + per - 1) / per;
    return b;
}
inline unsigned box_blocks(const Box& b) { return b.nbp * (unsigned)((b.cnt_k + b.kz - 1) / b.kz); }
template <typename FT>
struct ZoneArgs {
    khb_fields Ps, Us, U0, Pout, Uout;
    const FT* F[3];
    const FT* ctop[3];
    int32_t* pflag;
    int32_t* fflag;
    double g0, g1, bdt;
    const double* dt_dev;      // when set, bdt = beta * dt_dev[0] (device-resident timestep)
    double beta;
    unsigned long long* ndt_word;
    int* fail_count;
    int* fail_list;
    int mode;
    const double* Bf[3];       // B_CT: the stage output's face field (M_BCT), else unused
};


// One meshblock of a batch as the batched kernels see it: built once by khb_batch_create in device
// memory and staged in shared memory by each CTA.  za[s] are the zone-pass arguments of stage s + 1
// (bdt and the timestep flag are set in the kernel from the device timestep); Pin[s] is the flux
// input of that stage.  tile0[x]: the first tile of this block in the flux x1..x3 (x = 0..2) and
// zone (x = 3) launches.
template <typename FT>
struct BatchBlock {
    Dims d;
    DevGeom g;
    Phys ph;
    ZoneArgs<FT> za[2];
    khb_fields Pin[2];
    FT* F[3];
    FT* ctop[3];
    Box fbox[3];
    Box zbox;
    unsigned tile0[4];
    unsigned tile0c[4];        // first tile of each kind in the fused plan's combined table (x1-x3 faces, shell)
};

// One launch of launch_boundaries (a block's physical face, its ghost P->U pass or its periodic
// images) as a task of k_bound_tasks, which runs a phase's tasks of many blocks in one launch
enum { BOUND_BC = 0, BOUND_GHOST_PTOU = 1, BOUND_PERIODIC = 2 };
enum { BOUND_PHASES = 8 };         // X1 faces, X2 faces, corner fix, ghost P->U, its X3 planes, X3 faces,
                                   // P->U of the X3 ghost planes, periodic images
struct BoundTask {
    Dims d;
    DevGeom g;
    Phys ph;
    khb_fields P, U, Bf;           // Bf: all NULL (no face field)
    int kind;
    int face, lo_a, cnt_a, lo_k, cnt_k;     // BOUND_BC
    int kplanes, pfaces;                    // BOUND_GHOST_PTOU
    int pmask;                              // BOUND_PERIODIC
    long long count;                        // zones (threads) of the task
};

// One block's flux fix (a polar x2 face or an x1 inflow check) as a task of k_fix_tasks
template <typename FT>
struct FixTask {
    Dims d;
    Phys ph;
    FT* F1;
    FT* F2;
    FT* F3;
    int x1;                        // 1: the x1 inflow fix, 0: the polar x2 fix
    int inner;
    int count;                     // zones (threads) of the fix
};

// What the batched fixup reads of each block (independent of the flux precision)
struct FixupBlock {
    Dims d;
    DevGeom g;
    Phys ph;
    khb_fields Pin[2], Uin[2]; // stage inputs of stage 1 and 2
    khb_fields P[2], U[2];     // stage outputs of stage 1 and 2
    int exch;                  // the block has an exchange face: its ghost shell carries over
    int32_t* pflag;
    int* fail_count;
    int* fail_list;
};

// Launchers.  Launch<double> is compiled without FMA contraction (the FP64 path keeps the
// reference's rounding); Launch<float> (the FP32-flux form) is compiled with contraction.
template <typename FT>
struct Launch {
    static void flux(int recon, int nv, int dir, const Dims& d, const DevGeom& g, const Phys& ph,
                     const khb_fields& P, FT* F, FT* ctop, const int lo[3], const int cnt[3], cudaStream_t st);
    static void fix_flux_x2(int nv, const Dims& d, const Phys& ph, FT* F1, FT* F2, FT* F3, int inner, cudaStream_t st);
    static void fix_flux_x1(const Dims& d, FT* F1, int inner, cudaStream_t st);
    // the flux fixes of many blocks in one launch (max_count: the largest task's zone count)
    static void fix_tasks(int nv, const FixTask<FT>* tasks, int ntasks, int max_count, cudaStream_t st);
    static void zone(int nv, const Dims& d, const DevGeom& g, const Phys& ph, const ZoneArgs<FT>& a, cudaStream_t st);
    static void flux_ct(const Dims& d, FT* F1, FT* F2, FT* F3, FT* emf, cudaStream_t st);
    static void copy_flux(long long N, int nv, const FT* F, const FT* ctop, const khb_fields& out, double* ctop_out,
                          cudaStream_t st);
    // First-order flux correction of one stage: guess update from the raw fluxes, inversion and floor
    // test, flags (polar rows, periodic images), donor-cell LLF on the faces bordering a flagged zone
    static void fofc(int nv, const Dims& d, const DevGeom& g, const Phys& ph, const khb_fields& Ps,
                     const khb_fields& Us, const khb_fields& U0, FT* const F[3], FT* const ctop[3], double g0,
                     double g1, double bdt, const double* dt_dev, double beta, int32_t* flag, cudaStream_t st);
    // Batched launches over every block of a batch: tiles[t] is the block of tile t; grid = 0 runs
    // one CTA per tile, otherwise grid CTAs loop over the tiles.  Return the CTAs per SM the kernel
    // can keep resident (for sizing a persistent grid) when called with ntiles = 0.
    static int batch_flux(int recon, int nv, int dir, const BatchBlock<FT>* blocks, const int* tiles, unsigned ntiles,
                          unsigned grid, int stage, cudaStream_t st);
    static int batch_zone(int nv, int mode, const BatchBlock<FT>* blocks, const int* tiles, unsigned ntiles,
                          unsigned grid, int stage, int dtm, double beta, const double* dt, cudaStream_t st);
    // The fused plan's first launch of a stage: every block's faces along all directions and the
    // ghost-shell copies of blocks with exchange faces from one table (entry = block | kind << 28,
    // kind 0-2 faces along x1-x3, 3 the shell), after CTA 0 has reset the failed-zone counters
    // (counts[0..nblocks)) and, when word is given, the timestep minimum
    static int batch_flux_all(int recon, int nv, const BatchBlock<FT>* blocks, const int* tiles, unsigned ntiles,
                              unsigned grid, int stage, int* const* counts, int nblocks, unsigned long long* word,
                              cudaStream_t st);
    // SMR flux correction over the entries of a mesh's flux table (6 ints each)
    static void mesh_flux(int nv, const BatchBlock<FT>* blocks, const int* table, long long n, cudaStream_t st);
    static void mesh_ghost_cell(int nv, bool kastaun, const BatchBlock<FT>* blocks, const int* table, long long n,
                                int s, int standalone, cudaStream_t st);
};

// Zone-local FP64 work shared by both forms (compiled with the FP64 unit)
struct LaunchCommon {
    static void fixup(int nv, const Dims& d, const DevGeom& g, const Phys& ph, const khb_fields& P, const khb_fields& U,
                      const int32_t* pflag, const int* fail_count, const int* fail_list, cudaStream_t st);
    static void bc(int nv, const Dims& d, const DevGeom& g, const Phys& ph, const khb_fields& P, const khb_fields& U,
                   int face, int lo_a, int cnt_a, int lo_k, int cnt_k, cudaStream_t st);
    // kplanes: the ghost planes of physical X3 faces (bit 0: below ks, bit 1: above ke) instead of
    // the X1/X2 ghost zones of the interior planes.  pfaces (nonzero): only the zones past the faces
    // whose bits are set (bit f: face f = inner/outer X1, X2, X3), the boundary domains of a block
    // whose other faces are exchanged
    static void ghost_ptou(int nv, const Dims& d, const DevGeom& g, const Phys& ph, const khb_fields& P,
                           const khb_fields& U, cudaStream_t st, const khb_fields* Bf = nullptr, int ct_mask = 0,
                           int kplanes = 0, int pfaces = 0);
    static void periodic(int nv, const Dims& d, const khb_fields& P, const khb_fields& U, int pmask, cudaStream_t st);
    // ntasks tasks of one boundary phase in one launch; max_count: the largest task's zone count
    static void bound_tasks(int nv, const BoundTask* tasks, int ntasks, long long max_count, cudaStream_t st);
    static void ghost_copy(int nv, const Dims& d, const khb_fields& Pin, const khb_fields& Uin, const khb_fields& Pout,
                           const khb_fields& Uout, cudaStream_t st);
    static void batch_ghost_copy(int nv, const FixupBlock* blocks, int nblocks, int stage, cudaStream_t st);
    static void ptou(int nv, const Dims& d, const DevGeom& g, const Phys& ph, const khb_fields& P, const khb_fields& U,
                     cudaStream_t st);
    static void divb(const Dims& d, const Phys& ph, const khb_fields& U, int i_lo, int i_hi,
                     unsigned long long* word, cudaStream_t st);
    // Batched fixups (one CTA row per block) and the per-stage reset of the failed-zone counters
    // (and, when word != NULL, of the timestep minimum)
    static void batch_fixup(int nv, const FixupBlock* blocks, int nblocks, int stage, cudaStream_t st);
    // SMR ghost zones of stage `stage`'s outputs from entries [begin, end) of a mesh's ghost table
    static void mesh_ghost(int nv, const FixupBlock* blocks, const int* table, long long begin, long long end,
                           int stage, cudaStream_t st);
    // The same entries on conserved variables (U[u_sel]) and inversion seeds (Pin[seed_sel]), the
    // kharma driver's exchange; Launch<FT>::mesh_ghost_cell then inverts those ghost zones
    static void mesh_ghost_cons(int nv, const FixupBlock* blocks, const int* table, long long begin, long long end,
                                int seed_sel, int u_sel, cudaStream_t st);
    static void batch_reset(int* const* counts, int nblocks, unsigned long long* word, cudaStream_t st);
    // Per-stage reset of one block's failed-zone counter (and of the timestep minimum when word)
    static void stage_reset(int* count, unsigned long long* word, cudaStream_t st);
    // Device-resident timestep (grmhd.cpp:252-343, kharma_driver.cpp:439-460): state[0] = dt,
    // state[1] = time, state[2] = the dt of the last step; advanced from the minimum zone timestep
    static void next_dt(const unsigned long long* ndt_word, double* state, double cfl, double dt_min,
                        double max_dt_increase, cudaStream_t st);
};

// EMHD and implicit-solve parameters are passed to the kernels as the C-ABI structs themselves
typedef khb_emhd_params EmhdArgs;
typedef khb_implicit_params ImplicitArgs;

// Device fields of one implicit solve (all [10 slots][N] like khb_fields)
struct ImpFields {
    khb_fields Pf, Uf, Ps, S, Psol;
    double* solve_norm;
    double* solve_fail;
};

// Reduction words of the implicit solve: [it-1] maximum solve_norm of iteration it (bit pattern),
// [IMP_ITER_WORD] iterations taken
enum { IMP_MAX_ITER = 64, IMP_ITER_WORD = 64, IMP_WORDS = 65 };

struct LaunchEmhd {
    // explicit EMHD step: face fluxes of the 10-slot state ([10][N] per direction), dU/dt with the
    // EMHD geometric source (and the zone timestep minimum when dtm), the ImEx explicit update
    static void flux(int recon, int dir, const Dims& d, const DevGeom& g, const Phys& ph, const EmhdArgs& E,
                     const khb_fields& P, double* F, double* ctop, const int lo[3], const int cnt[3], cudaStream_t st);
    static void dudt(const Dims& d, const DevGeom& g, const Phys& ph, const EmhdArgs& E, double* const F[3],
                     double* const ctop[3], const khb_fields& Ps, const khb_fields& dUdt, int dtm,
                     unsigned long long* word, cudaStream_t st);
    static void imex_explicit(const Dims& d, const DevGeom& g, const khb_fields& Psub, const khb_fields& Usub,
                              const khb_fields& Ufull, const khb_fields& dUdt, const khb_fields& Pout,
                              const khb_fields& Uout, double g0, double g1, double bdt, cudaStream_t st);
    static void ptou(const Dims& d, const DevGeom& g, double gam, const EmhdArgs& E, const khb_fields& P,
                     const khb_fields& U, cudaStream_t st);
    static void add_source(const Dims& d, const DevGeom& g, const double* conn, double gam, const EmhdArgs& E,
                           const Phys& ph, const khb_fields& P, double* tmp, const khb_fields& dUdt, cudaStream_t st);
    static void implicit_iter(const Dims& d, const DevGeom& g, double gam, const EmhdArgs& E, const ImplicitArgs& ip,
                              const ImpFields& f, double dt, unsigned long long* words, int iter, cudaStream_t st);
    static void implicit_jacobian(const Dims& d, const DevGeom& g, double gam, const EmhdArgs& E,
                                  const ImplicitArgs& ip, const ImpFields& f, double dt, double* jac, double* res,
                                  cudaStream_t st);
    // ImEx stage: floors (fluid/drift frame) and stability limits over the interior, flag bits out
    static void floors(const Dims& d, const DevGeom& g, const Phys& ph, const khb_fields& P, int32_t* fflag,
                       cudaStream_t st);
    static void limits(const Dims& d, const DevGeom& g, double gam, const EmhdArgs& E, const khb_fields& P,
                       int32_t* eflag, cudaStream_t st);
    static void fix_solve(const Dims& d, const DevGeom& g, double gam, const EmhdArgs& E, const khb_fields& P,
                          const khb_fields& U, const double* solve_fail, double* scratch, cudaStream_t st);
};

inline unsigned blocks_for(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

// A face of the global domain with a physical boundary condition (outflow or reflecting), as
// opposed to a periodic face or an exchange face filled by the caller from a neighbouring block
__host__ __device__ inline bool phys_face(int bc)
{
    return bc == KHB_BC_OUTFLOW || bc == KHB_BC_REFLECTING || bc == KHB_BC_TRANSMITTING;
}

// Validate a khb_config and derive the block index ranges and physics parameters (no allocation).
// Returns KHB_OK or a KHB_ERR_* code with a message in *why.
int derive_block(const khb_config* cfg, Dims& d, Phys& ph, const char** why);

} // namespace khb

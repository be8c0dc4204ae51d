/*
 * khb.h -- C ABI of libkhb, the B200 (sm_100a) implementation of KHARMA's per-step GRMHD path.
 *
 * Each entry point replaces one Kokkos loop (or a fixed sequence of them) inside a KHARMA
 * package callback; the reference function it stands in for is cited beside it.  Paths are
 * relative to the KHARMA source tree (AFD-Illinois/kharma).
 *
 * Conventions
 *  - Every function returns 0 on success and a negative KHB_ERR_* code on failure; it never
 *    aborts and never traps on the device.  khb_last_error() returns a message for the
 *    calling thread.
 *  - All work is asynchronous on the caller's cudaStream_t (passed as void*; NULL = legacy
 *    default stream).  No call synchronizes except the two that return a value to the host,
 *    khb_get_min_ndt and khb_max_divb, which say so.
 *  - The caller owns the state: primitive and conserved fields are device arrays of doubles,
 *    one array per variable (as Parthenon allocates them), each [n3][n2][n1] with i fastest,
 *    covering the whole block including ghosts.  n1 = nx1 + 2 ng, and n2 (n3) = nx2 + 2 ng
 *    (nx3 + 2 ng) when that direction is active, else 1.  Variable order is
 *    rho, u, u1, u2, u3, B1, B2, B3 (primitives) and rho u^t, T^t_t + rho u^t, T^t_1..3,
 *    B^1..3 sqrt(-g) (conserved), matching KHARMA's VarMap for a GRMHD+flux-CT pack.  The EMHD
 *    entry points also read q~, dP~ (primitives) and q~ u^t sqrt(-g), dP~ u^t sqrt(-g) (conserved)
 *    from slots 8 and 9.
 *  - The context owns only scratch: face fluxes, signal speeds, the intermediate RK stage,
 *    reduction words and the geometry tables copied in by khb_set_geometry().
 *  - Per-zone flags keep the reference encodings: pflag is Inverter::Status
 *    (inverter/invert_template.hpp:53), fflag holds Floors::FFlag bits (floors/floors.hpp:52-70).
 *    They are int32 device arrays over the block.
 *  - A context is not thread-safe; use one per host thread or serialize externally.
 */
#ifndef KHB_H
#define KHB_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KHB_MAX_VARS 10

/* Slots of khb_fields: rho, u, u1-u3, B1-B3 in 0-7; the EMHD variables q~ and dP~ (the "tilde"
 * primitives of emhd/emhd.hpp:313-332 and their conserved forms) in 8 and 9 when EMHD is on. */
enum { KHB_RHO = 0, KHB_UU = 1, KHB_U1 = 2, KHB_B1 = 5, KHB_Q = 8, KHB_DP = 9 };

enum { KHB_OK = 0, KHB_ERR_ARG = -1, KHB_ERR_CUDA = -2, KHB_ERR_STATE = -3, KHB_ERR_UNSUPPORTED = -4 };

/* Reconstruction schemes (flux/reconstruction.hpp:49, flux.cpp:75-122; donor_cell_c gives the same
 * states as donor_cell).  linear_vl is Parthenon's simplified van Leer PLM on a uniform grid. */
enum { KHB_RECON_DONOR_CELL = 0, KHB_RECON_LINEAR_MC = 1, KHB_RECON_WENO5 = 2, KHB_RECON_PPM = 3,
       KHB_RECON_LINEAR_VL = 4, KHB_RECON_WENO5_LINEAR = 5, KHB_RECON_PPMX = 6, KHB_RECON_MP5 = 7 };
/* WENO5 lowered to linear MC (flux/low_order_edges, flux/low_order_poles; reconstruction.hpp:694-771) */
enum { KHB_RECON_LOWER_NONE = 0, KHB_RECON_LOWER_EDGES = 1, KHB_RECON_LOWER_POLES = 2 };
/* Riemann solvers (flux/flux.hpp:110-121) */
enum { KHB_FLUX_LLF = 0, KHB_FLUX_HLLE = 1 };
/* Boundary types per face (boundaries/boundaries.cpp:57-368).  KHB_BC_EXCHANGE (any face of an
 * active direction) marks a face whose ghost zones the caller fills from the neighbouring block
 * (Parthenon's boundary communication): khb_boundaries and the flux fixes leave it alone, and
 * khb_fix_utop reads the neighbour values there. */
enum { KHB_BC_PERIODIC = 0, KHB_BC_OUTFLOW = 1, KHB_BC_REFLECTING = 2, KHB_BC_EXCHANGE = 3,
       /* transmitting polar faces (one_block_transmit.cpp:43-137): X2 faces of a 3D block covering all
        * of x3 (periodic, even nx3) in coordinates symmetric about the pole; a ghost zone takes the
        * mirrored zone half-way round in x3 with u^2, u^3, B^2, B^3 inverted */
       KHB_BC_TRANSMITTING = 4 };
/* Floor injection frames (floors/floors.hpp:93, floors.cpp:66-91): the mixed frames take the normal
 * frame inside frame_switch_r and the fluid frame outside it, or the drift frame where
 * min(rho, u)/b^2 < frame_switch_beta and the normal frame elsewhere (floors_impl.hpp:84-106) */
enum { KHB_FRAME_FLUID = 0, KHB_FRAME_NORMAL = 1, KHB_FRAME_DRIFT = 2, KHB_FRAME_MIXED_FLUID_NORMAL = 3,
       KHB_FRAME_MIXED_NORMAL_DRIFT = 4 };
/* Arithmetic of reconstruction, Riemann fluxes and EMF averaging */
enum { KHB_PREC_FP64 = 0, KHB_PREC_FP32_FLUX = 1 };
/* Primitive recovery (inverter/type, inverter.cpp:54-64): 1D_W of Noble et al. (2006) or the
 * robust Kastaun et al. (2021) scheme with the inverter floors inside its residual */
enum { KHB_INVERTER_ONEDW = 0, KHB_INVERTER_KASTAUN = 1 };
/* Driver step semantics (driver/simple_step.cpp, driver/kharma_step.cpp) */
enum { KHB_DRIVER_SIMPLE = 0, KHB_DRIVER_KHARMA = 1 };

/* Floors::Prescription (floors/floors.hpp:100-117) */
typedef struct {
    double rho_min_const, u_min_const;
    double rho_min_geom, u_min_geom, r_char;
    double bsq_over_rho_max, bsq_over_u_max, u_over_rho_max;
    double ktot_max, gamma_max;
    int32_t use_r_char, temp_adjust_u, adjust_k, radius_dependent_floors;
    double floors_switch_r;
} khb_floors;

/* Block and package parameters, filled by the calling packages from their Params. */
typedef struct {
    int32_t nx1, nx2, nx3, ng;        /* interior zones per direction, ghost zones */
    double dx1, dx2, dx3;             /* native-coordinate zone widths (Dxc) */
    double gam;                       /* GRMHD/gamma */
    int32_t nvar;                     /* 5 (GRHD) or 8 (GRMHD with cell-centred B and flux-CT) */
    int32_t recon, riemann, precision;
    int32_t bc[6];                    /* inner_x1, outer_x1, inner_x2, outer_x2, inner_x3, outer_x3 */
    int32_t check_inflow_inner_x1, check_inflow_outer_x1;   /* boundaries/check_inflow_* */
    int32_t zero_polar_flux;          /* boundaries/zero_polar_flux */
    int32_t fix_polar_flux;           /* b_field/fix_polar_flux */
    int32_t fix_corner_inner;         /* boundaries/fix_corner_inner */
    int32_t spherical;                /* coordinates are spherical (floors use r) */
    int32_t cart_minkowski;           /* Cartesian Minkowski: geometric source is skipped (flux.cpp:407) */
    int32_t floors_on, floor_frame, recon_floors;
    int32_t iter_max; double err_tol; /* inverter/iter_max, inverter/err_tol (1D_W: 8, 1e-8;
                                         Kastaun: 25, 1e-12) */
    int32_t fix_average_neighbors, fix_atmosphere;
    khb_floors floors;                /* floors; also the inverter floors of the Kastaun scheme */
    int32_t inverter;                 /* KHB_INVERTER_* */
    /* first-order flux correction (fofc/on, fofc/polar_cells, fofc/eh_buffer; flux.cpp:175-221) and
     * the event-horizon radius of the coordinates (0 without one, coordinate_embedding.hpp:247-258) */
    int32_t fofc, fofc_polar_cells;
    double fofc_eh_buffer, r_horizon;
    /* magnetic field transport: KHB_CT_NONE is B_FluxCT (cell-centred B, flux-CT); the others are
     * B_CT (face-centred B, edge EMFs, b_field/ct_scheme, b_ct.cpp:65-67) and need the khb_ct_* calls */
    int32_t ct_scheme;
    /* KHB_RECON_LOWER_* (weno5 only), and flux/reconstruction_fallback: faces whose reconstructed
     * states hit the geometric floors take the PPM states (weno5, weno5_linear, linear_vl, ppmx, mp5;
     * needs floors) */
    int32_t recon_lower, recon_fallback;
    /* floors_inner (floors.hpp:155-167): the prescription for r < floors.floors_switch_r when
     * floors.radius_dependent_floors is set (for the floors, ceilings and the Kastaun inverter's
     * floors); the switch points of the mixed injection frames */
    khb_floors floors_inner;
    double frame_switch_r, frame_switch_beta;
    /* fofc/use_glf (replaced faces take the speed-of-light Lax-Friedrichs speeds, fofc.cpp:200-205) and
     * fofc/use_source_term (the guess update also takes the geometric source, kharma_driver.cpp:308-312) */
    int32_t fofc_use_glf, fofc_use_source_term;
} khb_config;

/* B_CT EMF schemes (b_ct.cpp:65): Balsara & Spicer 1999 flux averaging, Gardiner & Stone 2005
 * with the zone-centred EMF (E^0), and with upwinded E^c corrections (also "sg07") */
enum { KHB_CT_NONE = 0, KHB_CT_BS99 = 1, KHB_CT_GS05_0 = 2, KHB_CT_GS05_C = 3 };

/* Coordinate system for khb_build_geometry (coordinates/coordinate_systems.hpp) */
enum { KHB_BASE_CART_MINKOWSKI = 0, KHB_BASE_SPH_MINKOWSKI = 1, KHB_BASE_SPH_KS = 2, KHB_BASE_SPH_BL = 3 };
enum { KHB_TRANSFORM_NULL = 0, KHB_TRANSFORM_EKS = 1, KHB_TRANSFORM_MKS = 2, KHB_TRANSFORM_FMKS = 3 };
typedef struct {
    int32_t base, transform;
    double a, hslope, mks_smooth, poly_xt, poly_alpha, startx1;
} khb_coords;

typedef struct khb_ctx khb_ctx;

/* EMHD closures (emhd/emhd.hpp:58, selected by emhd/closure_type, emhd.cpp:62-102) */
enum { KHB_CLOSURE_CONSTANT = 0, KHB_CLOSURE_SOUNDSPEED = 1, KHB_CLOSURE_KAPPA_ETA = 2, KHB_CLOSURE_TORUS = 3 };
/* Jacobian of the implicit residual: the reference's forward differences (implicit.hpp:208-255)
 * or the exact Jacobian by a hand-written tangent (no counterpart in the reference) */
enum { KHB_JACOBIAN_FD = 0, KHB_JACOBIAN_EXACT = 1 };
/* Per-zone solver status (implicit/implicit.hpp:63-69), stored as doubles like solve_fail */
enum { KHB_SOLVE_CONVERGED = 0, KHB_SOLVE_FAIL = 1, KHB_SOLVE_BEYOND_TOL = 2, KHB_SOLVE_BACKTRACK = 3 };

/* EMHD::EMHD_parameters (emhd/emhd.hpp:60-84) with the package switches emhd/conduction and
 * emhd/viscosity (emhd.cpp:60-72); q~ is evolved iff conduction, dP~ iff viscosity.
 * stability_limits: emhd/stability_limits (emhd.cpp:118-125), the heat-flux and pressure-anisotropy
 * limits an ImEx stage applies after the implicit solve. */
typedef struct {
    int32_t closure, higher_order_terms, feedback, conduction, viscosity, stability_limits;
    double tau, conduction_alpha, viscosity_alpha, kappa, eta;
} khb_emhd_params;

/* Implicit package parameters (implicit/implicit.cpp:99-119); max_nonlinear_iter <= 64 */
typedef struct {
    int32_t min_nonlinear_iter, max_nonlinear_iter, use_qr, linesearch, max_linesearch_iter, jacobian;
    double jacobian_delta, rootfind_tol, linesearch_eps, linesearch_lambda;
} khb_implicit_params;

/* One device pointer per variable (Parthenon allocates each variable separately). */
typedef struct { double* v[KHB_MAX_VARS]; } khb_fields;

const char* khb_last_error(void);
int khb_version(void);

/* Create/destroy a context for one meshblock shape and option set.  Allocates the scratch listed
 * above on the current device. */
int khb_create(const khb_config* cfg, khb_ctx** out);
int khb_destroy(khb_ctx* ctx);

/* Host-side GRCoordinates cache construction (coordinates/gr_coordinates.cpp:96-248,
 * connection_average_points = 1).  Fills caller host arrays in GRCoordinates layout:
 *   gcov, gcon  [7][n2+1][n1+1][4][4]   gdet [7][n2+1][n1+1]
 *   gdet_conn   [n2][n1][4][4][4]       r_center [n2][n1] (embedding r, or |x| if Cartesian)
 * x1min..x3min are the native coordinates of the first interior face. */
int khb_build_geometry(const khb_coords* coords, const khb_config* cfg,
                       double x1min, double x2min, double x3min,
                       double* gcov, double* gcon, double* gdet, double* gdet_conn, double* r_center);

/* Copy a block's geometry (host arrays in the layout above, e.g. GRCoordinates::gcov_direct)
 * to the device, in the layout the kernels read. */
int khb_set_geometry(khb_ctx* ctx, const double* gcov, const double* gcon, const double* gdet,
                     const double* gdet_conn, const double* r_center);

/* ---------------------------------------------------------------------------------------------
 * Package-level entry points (each replaces the Kokkos loops of one reference function)
 * ------------------------------------------------------------------------------------------- */

/* Flux::GetFlux<recon, dir> (flux/get_flux.hpp:60-373): reconstruct P at the dir-faces, compute
 * conserved states and fluxes (prim_to_flux, flux_functions.hpp:116-178), signal speeds (vchar,
 * :368-439) and the LLF/HLLE flux into the context's flux scratch for that direction.  Faces
 * cover [s, e+1] along dir and [s-1, e+1] across it. */
int khb_get_flux(khb_ctx* ctx, int dir, const khb_fields* P, void* stream);

/* khb_get_flux over the faces whose x3 index lies in [k_lo, k_hi] only (each face's flux is
 * independent of the others: the union of calls over disjoint ranges equals khb_get_flux).  A slab
 * of an x3 decomposition computes the faces that read no x3 ghost plane while its halo exchange is in
 * flight, then the rest (the interior compute the halo exchange overlaps, kharma_driver.cpp:151). */
int khb_get_flux_planes(khb_ctx* ctx, int dir, const khb_fields* P, int k_lo, int k_hi, void* stream);

/* First-order flux correction of one stage (KHARMADriver::AddFOFC, kharma_driver.cpp:292-337;
 * Flux::MarkFOFC and Flux::FOFC, fofc.cpp:45-226), between khb_get_flux and khb_fix_flux: a guess of
 * the stage's conserved state from the raw face fluxes (interior plus the zones whose flags the
 * corrected faces read), its inversion (started from P_s) and floor test; zones that would hit
 * floors, lie within fofc_eh_buffer of the horizon or in the polar rows are flagged (periodic ghost
 * zones take their images' flags); every face bordering a flagged zone gets the donor-cell LLF flux
 * of all variables and its signal speed.  khb_stage and khb_step call it when cfg.fofc is set. */
int khb_fofc(khb_ctx* ctx, int stage, double dt, const khb_fields* P_s, const khb_fields* U_s,
             const khb_fields* U_0, void* stream);

/* B_FluxCT::FixFlux polar corrections (b_flux_ct.cpp:264-303, 372-470) and
 * KBoundaries::FixFlux (boundaries.cpp:611-690) applied to the raw face fluxes in scratch. */
int khb_fix_flux(khb_ctx* ctx, void* stream);

/* B_FluxCT::FluxCT (b_flux_ct.cpp:307-370): rewrite the B fluxes in scratch from corner EMFs.
 * khb_update() applies the same averaging on the fly, so calling this is only needed when the
 * caller reads the fluxes back (khb_copy_flux). */
int khb_flux_ct(khb_ctx* ctx, void* stream);

/* Copy one direction's face fluxes (nvar arrays shaped like the block) and max(cmax, cmin)
 * (one array) from scratch to caller device memory, as doubles. */
int khb_copy_flux(khb_ctx* ctx, int dir, const khb_fields* F_out, double* ctop_out, void* stream);

/* KHARMADriver::FluxDivergence (kharma_driver.hpp:208-231) with flux-CT B fluxes, plus
 * Flux::AddGeoSource (flux.cpp:395-444), plus AddStateUpdate's two WeightedSumData calls
 * (kharma_driver.cpp:339-387):  U_out = gam0 U_s + gam1 U_0 + beta_dt (-div F + S(P_s)),
 * over the interior.  U_out may alias U_0 or U_s. */
int khb_update(khb_ctx* ctx, const khb_fields* P_s, const khb_fields* U_s, const khb_fields* U_0,
               double gam0, double gam1, double beta_dt, const khb_fields* U_out, void* stream);

/* Inverter::BlockUtoP with the 1D_W inverter (inverter.cpp:131-182, onedw.hpp:89-233) and
 * B_FluxCT::BlockUtoP (b_flux_ct.cpp:196-217) over the interior.  P holds the guess on entry. */
int khb_utop(khb_ctx* ctx, const khb_fields* U, const khb_fields* P, int32_t* pflag, int32_t* fflag,
             void* stream);

/* Floors::ApplyGRMHDFloors (floors.cpp:262-270, floors_impl.hpp:45-128) over the interior,
 * including ceilings and the P->U of floored zones. */
int khb_apply_floors(khb_ctx* ctx, const khb_fields* P, const khb_fields* U, int32_t* pflag,
                     int32_t* fflag, void* stream);

/* Inverter::MeshFixUtoP (fixup.cpp:47-156) over the interior, periodic neighbours wrapped. */
int khb_fix_utop(khb_ctx* ctx, const khb_fields* P, const khb_fields* U, const int32_t* pflag,
                 void* stream);

/* Physical and periodic boundary conditions for P (fluid primitives) and the conserved field,
 * then B_P = B_U/gdet and U = U(P) in every ghost zone (boundaries.cpp:369-589 with Parthenon's
 * outflow/reflecting functions, and Flux::MeshPtoU on the ghosts).  A block with exchange faces: the
 * conditions over the whole transverse range, after the caller's exchange, and B_P, U only past its
 * physical faces. */
int khb_boundaries(khb_ctx* ctx, const khb_fields* P, const khb_fields* U, void* stream);

/* Flux::MeshPtoU (flux.cpp:276-322) over the whole block. */
int khb_ptou(khb_ctx* ctx, const khb_fields* P, const khb_fields* U, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Fused step (the driver's per-stage task list, kharma_step.cpp:77-319 / simple_step.cpp:39-168)
 * ------------------------------------------------------------------------------------------- */

/* One RK2 stage (stage = 1 or 2) with Parthenon's rk2 weights: fluxes in all active directions,
 * flux fixes, then ONE fused zone pass doing flux-CT, divergence, geometric source, the RK
 * combination, 1D_W inversion, floors and the lock-step P->U; then fixups of failed zones and
 * ghost zones.  A block with exchange faces first carries the ghost shell of P_s/U_s over to
 * P_out/U_out (the reference's P_s -> P_{s+1} guess copy, kharma_driver.cpp:380-384), as it stands
 * until the caller's exchange replaces it.  P_s/U_s are the stage input, U_0 the step-start conserved state, P_out/U_out the
 * result.  P_out may alias P_s only if the caller does not need P_s afterwards AND stage == 2
 * is not reading it (use distinct buffers).  On the last stage the minimum zone timestep is
 * accumulated on the device (read with khb_get_min_ndt). */
int khb_stage(khb_ctx* ctx, int stage, double dt, const khb_fields* P_s, const khb_fields* U_s,
              const khb_fields* U_0, const khb_fields* P_out, const khb_fields* U_out,
              int32_t* pflag, int32_t* fflag, void* stream);

/* The fused zone pass of one stage alone: flux-CT, divergence, geometric source, RK combination,
 * 1D_W inversion, floors and P->U over the interior (and, on stage 2, the CFL reduction), reading
 * the face fluxes left in scratch by khb_get_flux/khb_fix_flux.  khb_stage = khb_get_flux (each
 * direction) + khb_fix_flux + khb_zone_pass + khb_fix_utop_list + khb_boundaries. */
int khb_zone_pass(khb_ctx* ctx, int stage, double dt, const khb_fields* P_s, const khb_fields* U_s,
                  const khb_fields* U_0, const khb_fields* P_out, const khb_fields* U_out,
                  int32_t* pflag, int32_t* fflag, void* stream);

/* Inverter::MeshFixUtoP over the zones the last khb_zone_pass flagged (no scan of pflag). */
int khb_fix_utop_list(khb_ctx* ctx, const khb_fields* P, const khb_fields* U, const int32_t* pflag,
                      void* stream);

/* Full RK2 step in place on (P, U) using the context's scratch for the intermediate stage.
 * Equivalent to two khb_stage calls.  Launches only; no host synchronisation. */
int khb_step(khb_ctx* ctx, double dt, const khb_fields* P, const khb_fields* U,
             int32_t* pflag, int32_t* fflag, void* stream);

/* Minimum zone timestep (before cfl and clipping) of the last stage-2 zone pass, as
 * GRMHD::EstimateTimestep computes it (grmhd.cpp:294-330).  Synchronizes the stream. */
int khb_get_min_ndt(khb_ctx* ctx, double* min_ndt_host, void* stream);

/* Device-resident timestep control: GRMHD::EstimateTimestep and KHARMADriver::SetGlobalTimeStep
 * (grmhd.cpp:252-343, kharma_driver.cpp:439-460) evaluated on the device after each step, so a
 * step needs no host synchronisation.  khb_set_timestep gives the first dt and the schedule
 * (GRMHD/cfl, parthenon/time/dt_min, max_dt_increase); khb_get_timestep reads back the next dt, the
 * accumulated time and the dt of the last step (synchronizes). */
int khb_set_timestep(khb_ctx* ctx, double dt, double cfl, double dt_min, double max_dt_increase);
int khb_get_timestep(khb_ctx* ctx, double* dt_next, double* t, double* dt_last, void* stream);

/* khb_step with the device timestep, followed by the next timestep on the device.  Launches only. */
int khb_step_device_dt(khb_ctx* ctx, const khb_fields* P, const khb_fields* U, int32_t* pflag, int32_t* fflag,
                       void* stream);

/* The same step replayed from a CUDA graph, captured on the first call with a given state (P, U,
 * flags) on a non-default stream and replayed while the state pointers stay the same. */
int khb_step_graph(khb_ctx* ctx, const khb_fields* P, const khb_fields* U, int32_t* pflag, int32_t* fflag,
                   void* stream);

/* ---------------------------------------------------------------------------------------------
 * Discrete adjoint of the step (no reference counterpart: KHARMA has no adjoint; the step it
 * differentiates is khb_step, i.e. kharma_step.cpp:77-319 with the flux, flux-CT, update and
 * inversion kernels above)
 * ------------------------------------------------------------------------------------------- */

/* Adjoint of one khb_step (P_n, U_n) -> (P_np1, U_np1) at the given dt.  On entry (Pbar, Ubar)
 * hold the adjoint of the step's output; on return, the adjoint of its input (P_n, U_n), so that
 * calls for steps N-1, ..., 0 in turn carry an adjoint back through a run.  rho_flux1_weight (NULL:
 * none) adds the objective sum over stages of weight_scale * sum_faces weight[f] * F1[rho][f] of
 * the raw x1 face fluxes ([N] doubles, indexed like the zone arrays; with weight_scale = dt/2 and
 * weights of dx2 dx3 on one x1 face layer, the RK2-consistent mass through that layer in the step).
 * Both stages are recomputed from (P_n, U_n) (the intermediate one into the context's stage
 * scratch); the inversion is differentiated by the implicit-function theorem at the converged
 * state; the floors (fluid or drift frame, floors_functions.hpp:50-252) through the Jacobian of the
 * floor map at the inverted primitives before the floors, which the recompute keeps; a zone whose
 * inversion failed through its fixup (fixup.cpp:47-156: the weighted neighbour average, its
 * geometric floors and the zone's own B); periodic
 * ghost-zone adjoints are folded into their images, exchange ghost zones are constants, and the
 * ghost fills of outflow/reflecting X1/X2 faces (inflow checks, the corner fix, the ghost B of MHD
 * blocks) and the flux fixes (the X1 mass-flux clip, zero polar fluxes, B_FluxCT's polar B-flux fix,
 * boundaries.cpp:369-690, b_flux_ct.cpp:372-418) are transposed.  Supported: LLF fluxes with linear MC
 * or donor-cell reconstruction, periodic, exchange, outflow or reflecting faces, floors off or in the
 * fluid or drift frame with the 1D_W inverter, recon floors and FOFC off (KHB_ERR_UNSUPPORTED
 * otherwise).  Ghost zones of Pbar/Ubar are zero on return.  Scratch (8 nv N doubles, 4 N flags;
 * with floors 10 N doubles more) is allocated on the first call. */
int khb_adjoint_step(khb_ctx* ctx, double dt, const khb_fields* P_n, const khb_fields* U_n,
                     const khb_fields* P_np1, const khb_fields* Pbar, const khb_fields* Ubar,
                     const double* rho_flux1_weight, double weight_scale, void* stream);

/* *out += scale * sum_f weight[f] * F_dir[var][f] over the raw face fluxes left in the context's
 * scratch by the last khb_stage / khb_get_flux (the objective whose adjoint khb_adjoint_step seeds
 * for var = rho, dir = 1).  weight: [N] device doubles indexed like the zone arrays; out: one device
 * double.  Summed in a fixed order (reproducible).  Launches only. */
int khb_flux_dot(khb_ctx* ctx, int dir, int var, const double* weight, double scale, double* out, void* stream);

/* Pbar += (dU/dP)^T Ubar at every zone of P (the adjoint of Flux::p_to_u, flux_functions.hpp:343-352,
 * e.g. of the conserved initial state formed from primitive initial data). */
int khb_adjoint_ptou(khb_ctx* ctx, const khb_fields* P, const khb_fields* Ubar, const khb_fields* Pbar,
                     void* stream);

/* ---------------------------------------------------------------------------------------------
 * B_CT: face-centred magnetic field (cfg.ct_scheme != KHB_CT_NONE; 2D and 3D blocks; X1/X2 faces
 * periodic, exchange, outflow, reflecting or transmitting, X3 faces periodic or exchange; 4 ghost zones with
 * physical faces).  Face fields are passed as khb_fields with v[0..2] = the conserved sqrt(-g) B^1,
 * B^2, B^3 on x1, x2, x3 faces, each [n3][n2][n1] like the zone arrays, face i being the left face
 * of zone i (faces of the interior, [is, ie+1] along their own direction, are the state; the cell
 * B slots of P and U are derived from them).
 * ------------------------------------------------------------------------------------------- */

/* One RK2 stage with B_CT (kharma_step.cpp:163-214 with use_b_ct): fluxes, FixFlux, then
 * B_CT::CalculateEMF (b_ct.cpp:262-410: zone-centred EMF, edge EMFs by the configured scheme),
 * B_CT::AddSource (b_ct.cpp:412-470: face changes from the EMF circulation) and the face update
 * Bf_out = gam0 Bf_s + gam1 Bf_0 + beta dt dBf/dt (kharma_driver.cpp:339-387, WeightedSumDataFace),
 * then the zone pass with the zone B taken from the updated faces (B_CT::BlockUtoP,
 * b_ct.cpp:160-188) instead of the flux-CT divergence, fixups and ghost zones as khb_stage.  A block
 * with exchange faces (a block of a mesh) gets no ghost zones here: the caller exchanges, then calls
 * khb_ct_ghost_from_faces and, for physical faces, khb_ct_boundaries (the reference's sync, MeshUtoP
 * over the entire block, then its domain conditions: kharma_step.cpp:209-249). */
int khb_ct_stage(khb_ctx* ctx, int stage, double dt, const khb_fields* P_s, const khb_fields* U_s,
                 const khb_fields* U_0, const khb_fields* Bf_s, const khb_fields* Bf_0, const khb_fields* P_out,
                 const khb_fields* U_out, const khb_fields* Bf_out, int32_t* pflag, int32_t* fflag, void* stream);

/* Ghost zones of a B_CT block (KBoundaries::ApplyBoundary with B_CT, boundaries.cpp:369-500): with
 * physical faces, the face field's ghost layers first — reflecting faces: tangential components
 * mirrored, the normal one zero on the domain face and reflected beyond it (reflect_face_vector);
 * outflow faces: tangential components copied, the normal one rebuilt outward for zero divergence
 * (clean_face_B, b_ct_boundaries.cpp:190-262); transmitting X2 faces: the mirror rows half-way
 * round in x3 (one_block_transmit.cpp:60-143) — then the zone boundaries as khb_boundaries, with the
 * ghost zones' B from their faces (B_CT::BlockUtoP over the boundary domain).  Without physical
 * faces it is khb_boundaries.  On a block with exchange faces the conditions run over the whole
 * transverse range (the ghost rows the exchange filled included) and B and U = U(P) are rebuilt past
 * the physical faces only.  During each stage reflecting faces zero the EMFs on their domain-face
 * edges (zero_EMF, b_ct_boundaries.cpp:40-62) and transmitting ones average them (average_EMF,
 * b_ct_boundaries.cpp:64-186). */
int khb_ct_boundaries(khb_ctx* ctx, const khb_fields* P, const khb_fields* U, const khb_fields* Bf, void* stream);

/* khb_ct_stage in two halves, for a mesh whose blocks exchange corrections between them
 * (kharma_step.cpp:163-214: the flux and EMF corrections of a multilevel mesh run between
 * CalculateEMF and the update): khb_ct_stage_fluxes forms the face fluxes, their fixes and the edge
 * EMFs in context scratch; khb_ct_stage_update the face update, the zone pass, fixups and ghost
 * zones from them.  Same arguments and checks as khb_ct_stage. */
int khb_ct_stage_fluxes(khb_ctx* ctx, const khb_fields* P_s, void* stream);
int khb_ct_stage_update(khb_ctx* ctx, int stage, double dt, const khb_fields* P_s, const khb_fields* U_s,
                        const khb_fields* U_0, const khb_fields* Bf_s, const khb_fields* Bf_0, const khb_fields* P_out,
                        const khb_fields* U_out, const khb_fields* Bf_out, int32_t* pflag, int32_t* fflag,
                        void* stream);

/* B_CT::BlockUtoP over every ghost zone (b_ct.cpp:160-188 on the boundary domain): B^i as the average
 * of the zone's two faces (the last ghost layer of a direction, whose upper face the arrays do not
 * hold, from its lower face) and U = U(P); for blocks whose face field's ghost layers the caller
 * filled (an SMR mesh's exchange). */
int khb_ct_ghost_from_faces(khb_ctx* ctx, const khb_fields* P, const khb_fields* U, const khb_fields* Bf,
                            void* stream);

/* ---------------------------------------------------------------------------------------------
 * SMR meshes of B_CT blocks (KHARMA's default field transport on multilevel meshes,
 * kharma.cpp:376-395): tables from kharma_b200/ctmesh.py.  Blocks: FP64, any coordinates (the
 * operators act on the native grid; faces, fluxes and EMFs carry sqrt(-g)), one shape, 2D or 3D; every face an exchange face or an outflow/reflecting domain face, which the
 * block applies with khb_ct_boundaries after the exchange (no table entry reaches past it).  Per stage: khb_ct_stage_fluxes on every
 * block, khb_ctmesh_correct (the fluid fluxes of coarse faces on a fine-coarse boundary become the
 * mean of the fine fluxes, and coarse edge EMFs that coincide with fine edges the mean of the fine
 * EMFs along them: Parthenon's flux correction, kharma_step.cpp:183-194), khb_ct_stage_update on
 * every block, then khb_ctmesh_exchange on the stage output (ghost-zone fluid primitives by copy,
 * restriction or minmod prolongation; ghost faces by copy, area-average restriction (RestrictAverage),
 * minmod prolongation onto faces shared with coarse faces (ProlongateSharedMinMod) and Olivares'
 * divergence-preserving prolongation inside coarse zones (ProlongateInternalOlivares,
 * b_ct_functions.hpp:151-200)) and khb_ct_ghost_from_faces on every block.  Tables: ghost zones
 * (int32 x 6, the hydro mesh's format) with the end of each phase (copies and restrictions, then
 * one phase per destination level); ghost faces (int32 x 8) with phase ends; fluxes and EMFs
 * (int32 x 6).  P and Bf of khb_ctmesh_exchange are arrays of nblocks fields; the first exchange of a
 * state (its set of P and Bf pointers) uploads that state's descriptors and waits for the copy, later
 * ones, and every khb_ctmesh_correct, only launch kernels.
 * --------------------------------------------------------------------------------------------- */
typedef struct khb_ctmesh khb_ctmesh;
int khb_ctmesh_create(khb_ctx* const* ctxs, int nblocks, const int32_t* cell, int64_t n_cell,
                      const int64_t* cell_ends, int n_cell_phases, const int32_t* face, int64_t n_face,
                      const int64_t* face_ends, int n_face_phases, const int32_t* flux, int64_t n_flux,
                      const int32_t* emf, int64_t n_emf, khb_ctmesh** out);
int khb_ctmesh_destroy(khb_ctmesh* mesh);
int khb_ctmesh_correct(khb_ctmesh* mesh, void* stream);
int khb_ctmesh_exchange(khb_ctmesh* mesh, const khb_fields* P, const khb_fields* Bf, void* stream);

/* The kharma driver's stage on a B_CT mesh (sync_prims false, kharma_driver.cpp:109-118;
 * kharma_step.cpp:209-249): khb_ct_stage_fluxes and khb_ctmesh_correct as above, then
 * khb_ct_stage_update_part(part 1) on every block (face update, ghost-shell copy, the update half of
 * the zone pass: U_out holds the updated conserved state), khb_ctmesh_exchange_cons (ghost-zone fluid
 * U and seed primitives P_s by the cell entries — GRMHD sync_utop_seed, grmhd.cpp:159-165 — ghost
 * faces by the face entries, then every entry's ghost zone inverted from its seed with B and U_B from
 * its faces, floored and given U = U(P), as MeshUtoP and MeshApplyFloors over the entire block do),
 * khb_ct_stage_update_part(part 2) on every block (the cell half over the interior and the fixups),
 * and khb_ct_boundaries on blocks with physical faces.  The seeds of the ghost zones are written into
 * P_s (whose ghost zones the stage's fluxes have already read).  Arrays per block as
 * khb_ctmesh_exchange; descriptors cached per pointer set in the same way. */
int khb_ct_stage_update_part(khb_ctx* ctx, int part, int stage, double dt, const khb_fields* P_s,
                             const khb_fields* U_s, const khb_fields* U_0, const khb_fields* Bf_s,
                             const khb_fields* Bf_0, const khb_fields* P_out, const khb_fields* U_out,
                             const khb_fields* Bf_out, int32_t* pflag, int32_t* fflag, void* stream);
int khb_ctmesh_exchange_cons(khb_ctmesh* mesh, const khb_fields* P_s, const khb_fields* U, const khb_fields* P_out,
                             const khb_fields* Bf, int32_t* const* pflag, int32_t* const* fflag, void* stream);

/* Full RK2 step with B_CT in place on (P, U, Bf), the intermediate stage in context scratch. */
int khb_ct_step(khb_ctx* ctx, double dt, const khb_fields* P, const khb_fields* U, const khb_fields* Bf,
                int32_t* pflag, int32_t* fflag, void* stream);

/* B_CT::BlockUtoP (b_ct.cpp:160-188) over the interior: zone B^i (P slots 5-7) as the average of the
 * two faces' B^i, zone sqrt(-g) B^i (U slots 5-7) from it.  Ghost zones: khb_ct_boundaries. */
int khb_ct_utop(khb_ctx* ctx, const khb_fields* Bf, const khb_fields* P, const khb_fields* U, void* stream);

/* B_CT::DangerousPtoU (b_ct.cpp:190-253): interior faces from the zone B of P (average of the two
 * zones times sqrt(-g) at the face), e.g. to start from cell-centred initial data. */
int khb_ct_faces_from_prims(khb_ctx* ctx, const khb_fields* P, const khb_fields* Bf, void* stream);

/* B_CT::BlockMaxDivB (b_ct.cpp:499-520, face_div b_ct_functions.hpp:47-56): max over the interior of
 * |sum_d (Bf_d(+) - Bf_d(-)) / dx_d|.  Synchronizes the stream. */
int khb_ct_max_divb(khb_ctx* ctx, const khb_fields* Bf, double* max_divb_host, void* stream);

/* One step of a host-resident state (nv host arrays of the primitives, entire block, pinned for
 * asynchronous copies), through the device state (P, U): the primitives are copied in, U = U(P) is
 * rebuilt on the device (the lock-step P -> U of every stage leaves U = U(P) at the end of a step, so
 * this is the state's own U, bit for bit), the step runs as khb_step_graph (device timestep; set it
 * with khb_set_timestep; non-default stream), and the primitives are copied back into P_host.
 * Launches and copies only; the caller synchronizes before reading P_host. */
int khb_step_host(khb_ctx* ctx, double* const* P_host, const khb_fields* P, const khb_fields* U, int32_t* pflag,
                  int32_t* fflag, void* stream);

/* khb_step_host for a host state holding the interior zones only (nv host arrays [nx3][nx2][nx1],
 * pinned): the ghost zones of a block whose faces are all physical or periodic are functions of its
 * interior, so they are rebuilt on the device (U = U(P) on the interior, then the block's boundaries,
 * as the step's last stage leaves them, bit for bit) instead of crossing the bus; 0.82x the bytes of
 * khb_step_host at 128^3.  The interiors travel packed through the context's stage scratch.  Blocks
 * with exchange faces (whose ghost zones are the caller's) are rejected. */
int khb_step_host_interior(khb_ctx* ctx, double* const* P_host, const khb_fields* P, const khb_fields* U,
                           int32_t* pflag, int32_t* fflag, void* stream);

/* B_FluxCT::MaxDivB (b_flux_ct.cpp:566-607): max |corner divB| of the conserved field.
 * Synchronizes the stream. */
int khb_max_divb(khb_ctx* ctx, const khb_fields* U, double* max_divb_host, void* stream);

/* No counterpart in the reference.  For callers that cannot allocate device memory (a framework
 * that hands out device memory only from its own pre-reserved pool, or a diagnostic hook holding
 * only the field pointers and no context, since creating a context allocates its scratch): the
 * same maximum as khb_max_divb, computed without a context and without any allocation (0 for
 * blocks without B, nvar < 8, and for 1D blocks, as khb_max_divb returns).  The per-block partial
 * maxima live in a file-scope __device__ array of 16384 doubles (128 KiB, held by every GPU that
 * loads the library until exit), so blocks with more than 256 * 16384 corners are rejected with
 * KHB_ERR_ARG.  The result is written asynchronously to *max_divb_out (device memory); the host
 * does not wait for the stream.  The first call on a device looks the array's address up
 * (cudaGetSymbolAddress) with that device current and keeps it for the life of the process: make
 * that first call before any stream capture begins, and do not call this again on a device after
 * cudaDeviceReset (the kept address belongs to the destroyed context).  Calls that overlap on the
 * GPU share the array and race; serialize them.  Errors: khb_noalloc_last_error(). */
int khb_max_divb_noalloc(const khb_config* cfg, const khb_fields* U, double* max_divb_out, void* stream);
const char* khb_noalloc_last_error(void);

/* ---------------------------------------------------------------------------------------------
 * Batches of meshblocks (no single counterpart in the reference: Parthenon's MeshData packs run the
 * same task list over all blocks of a partition, kharma_step.cpp:77-319, with uniform block
 * sizes).  Every block of a mesh, of uneven sizes, goes through one launch per kernel per RK stage;
 * the step can be replayed from a CUDA graph; the tile shape per block size is chosen by timing.
 * ------------------------------------------------------------------------------------------- */
typedef struct khb_batch khb_batch;

/* Group nblocks contexts (each created and given its geometry as for a single block; sizes may
 * differ, while nvar, dimension, reconstruction, Riemann solver and precision must agree) with the
 * state each block is stepped on: P[b], U[b] (its fields), pflag[b], fflag[b] (its flags).  The
 * contexts and arrays must outlive the batch.  Ghost zones of exchange faces are the caller's;
 * physical and periodic faces are filled per block as khb_boundaries does. */
int khb_batch_create(khb_ctx* const* blocks, int nblocks, const khb_fields* P, const khb_fields* U,
                     int32_t* const* pflag, int32_t* const* fflag, khb_batch** out);
int khb_batch_destroy(khb_batch* batch);

/* One RK2 step of every block in place: the arithmetic of khb_step on each block (bitwise), with
 * each kernel launched once per stage for all blocks.  No host synchronisation. */
int khb_batch_step(khb_batch* batch, double dt, void* stream);

/* The same step replayed from a CUDA graph captured on the first call on a non-default stream
 * (captured again after khb_batch_set_tuning or khb_batch_autotune).  dt is read from device memory
 * by the kernels, so one graph serves every timestep. */
int khb_batch_step_graph(khb_batch* batch, double dt, void* stream);

/* Minimum zone timestep over all blocks from the last step, as khb_get_min_ndt.  Synchronizes. */
int khb_batch_get_min_ndt(khb_batch* batch, double* min_ndt_host, void* stream);

/* Block-size classes (distinct nx1, nx2, nx3) in order of first appearance: sizes[3 c + a] and
 * the planes per CTA kz[c] of each (0 = the default shape); up to max classes are written. */
int khb_batch_classes(khb_batch* batch, int32_t* nclasses, int32_t* sizes, int32_t* kz, int max);

/* Tile shape of one class (kz = 1, 2 or 4 k planes per 128-thread CTA, 0 = default; size_class < 0
 * leaves the classes alone) and the launch mode: persistent = 1 sizes each grid to the SMs times
 * the CTAs each can hold, and the CTAs loop over the tiles; 0 launches one CTA per tile. */
int khb_batch_set_tuning(khb_batch* batch, int size_class, int kz, int persistent);

/* Autotuner: for each class in turn, time reps runs of a stage-1 pass with each tile shape and
 * keep the fastest; then the same for the launch mode and the launch plan.  Stage 1 writes only the
 * contexts' stage scratch, the flags and the failed-zone lists, so the state is unchanged.  Writes
 * the chosen kz per class and the launch mode (the plan: khb_batch_get_plan).  Synchronizes. */
int khb_batch_autotune(khb_batch* batch, int reps, int32_t* kz_out, int32_t* persistent_out, void* stream);

/* Launch plan of a stage (results bitwise the same): 0 (the default) launches each kernel once per
 * stage for all blocks (counter reset, faces per direction, ghost-shell copy, update half, cell
 * half, fixups: 8 launches per stage for blocks with exchange faces); 1 fuses them into three (all
 * faces of all directions with the resets and ghost-shell copies, the whole zone pass, fixups).
 * Blocks with physical faces add one launch for all their flux fixes and one launch per boundary
 * phase for all of them (faces by direction, corner fix, ghost P->U, X3 planes, periodic images),
 * SMR meshes the flux correction and ghost exchange, in either plan.  A captured graph is captured
 * again. */
int khb_batch_set_plan(khb_batch* batch, int plan);
int khb_batch_get_plan(khb_batch* batch, int32_t* plan);

/* Device kernel launches issued for this batch so far (a graph replay counts its nodes). */
int64_t khb_batch_launch_count(khb_batch* batch);

/* Static mesh refinement over the blocks of a batch (Parthenon's boundary communication and flux
 * correction for a refined mesh, kharma_step.cpp:157-214, with its cell-centred refinement operators):
 * the blocks form one mesh whose ghost zones are filled from their neighbours after every stage and
 * whose coarse faces on fine-coarse boundaries take the average of the fine fluxes before the update.
 * ghost: n_ghost entries of 6 int32 {dst block, dst zone, op, src block, src zone, aux}, op 0 copy,
 * 1 restriction (average of the 2^ndim fine zones from src zone upwards), 2 prolongation (src coarse
 * zone plus minmod-limited slopes times +-1/4; aux bit d: + side along direction d+1, aux bits 8 and
 * up: the prolongation phase, the destination level less one); the first n_ghost_first entries are
 * the copies and restrictions, the rest the prolongations in phase order, each phase launched after
 * the previous one (a level's prolongations read coarse ghost zones the coarser level's filled).  The primitives
 * are filled, then U = U(P) in those zones.  flux: n_flux entries {coarse block, direction, coarse
 * face, fine block, fine face of lowest index, 0}.  Hydro blocks (nvar 5) with exchange faces; a
 * block on an outflow or reflecting domain face applies it after each exchange, over the ghost rows
 * the exchange filled (no entry reaches past it).  Every index is checked against the blocks' sizes.
 * Synchronizes the device. */
int khb_batch_set_mesh(khb_batch* batch, const int32_t* ghost, int64_t n_ghost, int64_t n_ghost_first,
                       const int32_t* flux, int64_t n_flux);

/* Fill every block's ghost zones of the state (P, U) from the mesh (e.g. after initial data), then
 * the physical domain faces of the blocks on them.  With KHB_SYNC_CONSERVED: U and P (the seeds) by
 * the entries, then the inversion, floors and U = U(P) in those ghost zones. */
int khb_batch_mesh_exchange(khb_batch* batch, void* stream);

/* What a mesh's exchange moves (kharma_driver.cpp:109-118: sync_prims = driver_type != kharma).
 * KHB_SYNC_PRIMS (the simple and ImEx drivers, the default): after each stage, the primitives by
 * the entries, then U = U(P) there.  KHB_SYNC_CONSERVED (the kharma driver): between the update and
 * the inversion of each stage, the updated conserved variables and, as the inversion's seeds, the
 * stage's input primitives (GRMHD sync_utop_seed, grmhd.cpp:159-165), both by the entries; then the
 * ghost zones are inverted, floored and given U = U(P) as the interior is (MeshUtoP and
 * MeshApplyFloors over the entire block, kharma_step.cpp:233-236).  The conserved exchange runs the
 * plain launch plan (the fused one inverts in the pass that updates). */
enum { KHB_SYNC_PRIMS = 0, KHB_SYNC_CONSERVED = 1 };
int khb_batch_set_mesh_sync(khb_batch* batch, int mode);

/* ---------------------------------------------------------------------------------------------
 * Extended MHD and the implicit solve (emhd/, implicit/)
 * ------------------------------------------------------------------------------------------- */

/* Host construction of the connection coefficients Gamma^a_bc at zone centres
 * (gr_coordinates.cpp:156-161, conn_direct): conn [n2][n1][4][4][4], same arguments as
 * khb_build_geometry. */
int khb_build_connection(const khb_coords* coords, const khb_config* cfg, double x1min, double x2min,
                         double x3min, double* conn);

/* Copy the connection (host, layout above) to the device and allocate the EMHD scratch of this
 * context (5 + 7 doubles per zone).  Required before khb_emhd_add_source and khb_fix_solve. */
int khb_set_connection(khb_ctx* ctx, const double* conn);

/* Flux::MeshPtoU with the EMHD stress tensor (flux_functions.hpp:80-107, 180-232) and
 * EMHD::BlockPtoU (emhd.cpp:251-281) over the whole block: all 8 + (q, dP) conserved variables. */
int khb_emhd_ptou(khb_ctx* ctx, const khb_emhd_params* emhd, const khb_fields* P, const khb_fields* U,
                  void* stream);

/* EMHD::AddSource (emhd.cpp:288-397): adds the explicit conduction and viscosity sources
 * (gradients of u_mu and Theta by MC slopes, emhd_utils.hpp:55-79) to slots 8/9 of dUdt over the
 * interior.  P needs one valid ghost layer in each active direction. */
int khb_emhd_add_source(khb_ctx* ctx, const khb_emhd_params* emhd, const khb_fields* P, const khb_fields* dUdt,
                        void* stream);

/* Implicit::Step (implicit.cpp:159-571) over the interior: up to max_nonlinear_iter Newton
 * iterations of the per-zone implicit residual (implicit.hpp:139-200) with a forward-difference
 * (reference) or exact Jacobian, QR with column pivoting (or the LU path), backtracking and line
 * search.  P_full/U_full: state at the start of the step; P_sub: at the start of this sub-step;
 * src: flux divergence plus explicit sources (dU/dt); P_solver: initial guess on entry, result on
 * return (implicit variables only; its B is used as given).  solve_norm and solve_fail are the
 * reference's per-zone fields (doubles over the block), read and written; a zone that enters with
 * solve_fail == KHB_SOLVE_FAIL is skipped.  The iteration stops, as in the reference, after
 * min_nonlinear_iter iterations once the maximum solve_norm is below rootfind_tol; that test runs on
 * the device, so nothing is synchronized. */
int khb_implicit_step(khb_ctx* ctx, const khb_emhd_params* emhd, const khb_implicit_params* imp,
                      const khb_fields* P_full, const khb_fields* U_full, const khb_fields* P_sub,
                      const khb_fields* src, const khb_fields* P_solver, double* solve_norm, double* solve_fail,
                      double dt, void* stream);

/* Flux::GetFlux with the EMHD variables (get_flux.hpp:60-373; prim_to_flux with the EMHD stress
 * tensor, flux_functions.hpp:80-107 and 180-232; vchar with the EMHD-augmented sound speed,
 * flux_functions.hpp:380-403): face fluxes of all 10 slots along dir into the context's EMHD flux
 * scratch (allocated by khb_set_connection).  FP64 contexts with B only. */
int khb_get_flux_emhd(khb_ctx* ctx, const khb_emhd_params* emhd, int dir, const khb_fields* P, void* stream);

/* Copy one direction's EMHD face fluxes (10 slots, as doubles) and max(cmax, cmin) out of scratch. */
int khb_copy_flux_emhd(khb_ctx* ctx, int dir, const khb_fields* F_out, double* ctop_out, void* stream);

/* One ImEx stage (driver/imex_step.cpp:58-356) of the vl2 integrator the implicit package forces
 * (implicit.cpp:96; stage 1: beta 1/2, stage 2: beta 1, both from the step-start state):
 * EMHD fluxes, flux-CT, the flux fixes of physical faces (boundaries.cpp:611-690: X1 inflow checks,
 * zero polar fluxes of all 10 slots), divergence, the geometric source with the EMHD tensor and
 * EMHD::AddSource into dU/dt; the explicit update of B and B_P = B_U/gdet; the implicit guess copied
 * from the sub-step state; Implicit::Step with beta dt (fluid and EMHD variables); the floors
 * (imex_step.cpp:269; fluid or drift frame) and the EMHD stability limits (emhd_limits.hpp:55-130)
 * over the interior; FixSolve; the ghost zones of the 10-slot state (periodic images and the
 * outflow/reflecting faces, q~ and dP~ copied as the density); P -> U with the EMHD tensor over the
 * whole block.  P_out/U_out must not alias P_sub/U_sub; exchange faces carry the sub-step ghost zones
 * over.  Floors or stability limits need the flag arrays: use khb_imex_stage_flags (KHB_ERR_ARG
 * here).  The last stage accumulates the zone timestep minimum (khb_get_min_ndt). */
int khb_imex_stage(khb_ctx* ctx, const khb_emhd_params* emhd, const khb_implicit_params* imp, int stage, double dt,
                   const khb_fields* P_full, const khb_fields* U_full, const khb_fields* P_sub, const khb_fields* U_sub,
                   const khb_fields* P_out, const khb_fields* U_out, double* solve_norm, double* solve_fail,
                   void* stream);

/* khb_imex_stage with the stage's flag fields ([N] int32 each, device): fflag the floor bits
 * (KHB_FFLAG_*) and eflag the EMHD limit bits (1 heat flux, 2 pressure anisotropy above, 4 below;
 * emhd_limits.hpp:38-40) of the interior zones, written every call (zeros where the floors or the
 * limits are off; either may be NULL while its step is off).  The normal-observer and mixed floor
 * frames are rejected (KHB_ERR_UNSUPPORTED) on the EMHD state. */
int khb_imex_stage_flags(khb_ctx* ctx, const khb_emhd_params* emhd, const khb_implicit_params* imp, int stage,
                         double dt, const khb_fields* P_full, const khb_fields* U_full, const khb_fields* P_sub,
                         const khb_fields* U_sub, const khb_fields* P_out, const khb_fields* U_out,
                         double* solve_norm, double* solve_fail, int32_t* fflag, int32_t* eflag, void* stream);

/* Iterations taken by the last khb_implicit_step and the maximum solve_norm of each (max_norms
 * has room for max_nonlinear_iter values).  Synchronizes the stream. */
int khb_implicit_stats(khb_ctx* ctx, int32_t* iterations, double* max_norms, void* stream);

/* Residual and Jacobian at P_solver without updating it (the split implicit_jacobian kernel,
 * implicit.cpp:286-320, which stores Implicit.jacobian and Implicit.residual): jacobian is
 * [nf*nf][n3][n2][n1] row-major per zone, residual [nf][n3][n2][n1], nf = 5 + conduction + viscosity. */
int khb_implicit_jacobian(khb_ctx* ctx, const khb_emhd_params* emhd, const khb_implicit_params* imp,
                          const khb_fields* P_full, const khb_fields* U_full, const khb_fields* P_sub,
                          const khb_fields* src, const khb_fields* P_solver, double dt, double* jacobian,
                          double* residual, void* stream);

/* Implicit::FixSolve (fix_solve.cpp:44-130) over the whole block: zones with solve_fail ==
 * KHB_SOLVE_FAIL get the distance-weighted average of their non-failed neighbours' implicit
 * primitives (all neighbours if none is good), read from the state before this call, and U = U(P). */
int khb_fix_solve(khb_ctx* ctx, const khb_emhd_params* emhd, const khb_fields* P, const khb_fields* U,
                  const double* solve_fail, void* stream);

/* Launch-shape choices that do not change results (bitwise): "zone_split" = 0 runs the zone pass
 * as one kernel, 1 (the default) as two (update; inversion + floors + P->U), 2 as three (update;
 * inversion; floors + P->U). */
int khb_set_tuning(khb_ctx* ctx, const char* key, int value);

/* Number of device kernel launches issued through this context so far (for accounting). */
int64_t khb_launch_count(khb_ctx* ctx);

/* No counterpart in the reference.  The bounds-checked build of this library (kharma_b200/lib/
 * libkhb_checked.so, compiled with KHB_BOUNDS_CHECK=1): the stencil loads and stores of the face
 * kernels, the zone pass's flux and corner-EMF loads, the fixups' neighbours, the boundary and
 * periodic-image copies and the geometry indices are checked against their arrays; an index outside
 * is replaced by 0 (so the access stays inside the array and nothing traps) and the first one is
 * recorded in the context's status word as site << 48 | its low 48 bits (sites: 1 face stencil, 2
 * face store, 3 zone-pass flux, 4 corner EMF, 5 fixup neighbour, 6 boundary copy, 7 periodic image,
 * 8 geometry).  khb_bounds_checked: 1 in that build, 0 in the regular one (whose checks compile away
 * and whose status stays 0).  khb_bounds_status reads the word and clears it; synchronizes. */
int khb_bounds_checked(void);
int khb_bounds_status(khb_ctx* ctx, uint64_t* status, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* KHB_H */

"""ctypes binding of the CPU oracle (oracle/_build/liborc.so).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the CPU-baseline leg of
bench.py as the checker.  Builds the library with `make -C oracle` on first use.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liborc.so")


class Prescription(C.Structure):
    _fields_ = [
        ("rho_min_const", C.c_double), ("u_min_const", C.c_double),
        ("rho_min_geom", C.c_double), ("u_min_geom", C.c_double), ("r_char", C.c_double),
        ("bsq_over_rho_max", C.c_double), ("bsq_over_u_max", C.c_double), ("u_over_rho_max", C.c_double),
        ("ktot_max", C.c_double), ("gamma_max", C.c_double),
        ("use_r_char", C.c_int32), ("temp_adjust_u", C.c_int32), ("adjust_k", C.c_int32),
        ("radius_dependent_floors", C.c_int32),
        ("floors_switch_r", C.c_double),
    ]


class CoordSpec(C.Structure):
    _fields_ = [("base", C.c_int32), ("transform", C.c_int32),
                ("a", C.c_double), ("hslope", C.c_double), ("mks_smooth", C.c_double),
                ("poly_xt", C.c_double), ("poly_alpha", C.c_double), ("startx1", C.c_double)]


class Config(C.Structure):
    _fields_ = [
        ("nx1", C.c_int32), ("nx2", C.c_int32), ("nx3", C.c_int32), ("ng", C.c_int32),
        ("x1min", C.c_double), ("x2min", C.c_double), ("x3min", C.c_double),
        ("dx1", C.c_double), ("dx2", C.c_double), ("dx3", C.c_double),
        ("gam", C.c_double),
        ("recon", C.c_int32), ("riemann", C.c_int32),
        ("nvar", C.c_int32),
        ("driver", C.c_int32),
        ("bc", C.c_int32 * 6),
        ("check_inflow_inner_x1", C.c_int32), ("check_inflow_outer_x1", C.c_int32),
        ("zero_polar_flux", C.c_int32), ("fix_polar_flux", C.c_int32), ("fix_corner_inner", C.c_int32),
        ("floors_on", C.c_int32), ("floor_frame", C.c_int32), ("recon_floors", C.c_int32),
        ("iter_max", C.c_int32), ("err_tol", C.c_double),
        ("fix_average_neighbors", C.c_int32), ("fix_atmosphere", C.c_int32),
        ("cfl", C.c_double), ("dt_min", C.c_double), ("max_dt_increase", C.c_double),
        ("floors", Prescription),
        ("inverter", C.c_int32),
        ("fofc", C.c_int32), ("fofc_polar_cells", C.c_int32),
        ("fofc_eh_buffer", C.c_double), ("r_horizon", C.c_double),
        ("ct_scheme", C.c_int32),
        ("recon_lower", C.c_int32), ("recon_fallback", C.c_int32),
        ("floors_inner", Prescription),
        ("frame_switch_r", C.c_double), ("frame_switch_beta", C.c_double),
        ("fofc_use_glf", C.c_int32), ("fofc_use_source_term", C.c_int32),
    ]


RECON = {"donor_cell": 0, "donor_cell_c": 0, "linear_mc": 1, "weno5": 2, "ppm": 3, "linear_vl": 4, "weno5_linear": 5,
         "ppmx": 6, "mp5": 7}
BC = {"periodic": 0, "outflow": 1, "reflecting": 2, "exchange": 3, "transmitting": 4, "dirichlet": 3, "bondi": 3}
FRAME = {"fluid": 0, "normal": 1, "drift": 2, "mixed": 3, "mixed_fluid_normal": 3, "mixed_normal_drift": 4}
BASE = {"cartesian_minkowski": 0, "spherical_minkowski": 1, "spherical_ks": 2, "spherical_bl": 3}
TRANSFORM = {"null": 0, "eks": 1, "mks": 2, "fmks": 3}

_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    src = os.path.join(HERE, "khb_oracle.cpp")
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.run(["make", "-C", HERE], check=True, capture_output=True)
    lib = C.CDLL(LIB)
    P = C.c_void_p
    lib.orc_create.restype = P
    lib.orc_create.argtypes = [C.POINTER(Config), C.POINTER(CoordSpec)]
    lib.orc_destroy.argtypes = [P]
    lib.orc_set_threads.restype = C.c_int
    lib.orc_set_threads.argtypes = [C.c_int]
    lib.orc_get_dims.argtypes = [P, P]
    lib.orc_get_geometry.argtypes = [P, P, P, P, P, P]
    lib.orc_set_geometry.argtypes = [P, P, P, P, P, P]
    lib.orc_get_flux.argtypes = [P, C.c_int, P, P, P, P]
    lib.orc_fix_flux.argtypes = [P, P, P, P]
    lib.orc_utop.argtypes = [P, P, P, P, P]
    lib.orc_floors.argtypes = [P, P, P, P, P]
    lib.orc_fix_utop.argtypes = [P, P, P, P]
    lib.orc_ptou.argtypes = [P, P, P]
    lib.orc_boundaries.argtypes = [P, P, P]
    lib.orc_step.argtypes = [P, P, P, P, P, C.c_double, P, P]
    lib.orc_ct_step.argtypes = [P, P, P, P, P, P, C.c_double, P, P]
    lib.orc_ct_utop.argtypes = [P, P, P, P]
    lib.orc_ct_faces_from_prims.argtypes = [P, P, P]
    lib.orc_ct_boundaries.argtypes = [P, P, P, P]
    lib.orc_ct_max_divb.restype = C.c_double
    lib.orc_ct_max_divb.argtypes = [P, P]
    lib.orc_max_divb.restype = C.c_double
    lib.orc_max_divb.argtypes = [P, P, C.c_int, C.c_int]
    lib.orc_utop_cell.restype = C.c_int
    lib.orc_utop_cell.argtypes = [P, C.c_int, C.c_int, P, P]
    lib.orc_get_connection.argtypes = [P, P]
    lib.orc_emhd_ptou.argtypes = [P, P, P, P]
    lib.orc_emhd_add_source.argtypes = [P, P, P, P]
    lib.orc_implicit_jacobian.argtypes = [P, P, P, P, P, P, P, P, C.c_double, P, P]
    lib.orc_implicit_residual.argtypes = [P, P, P, P, P, P, P, C.c_double, P]
    lib.orc_dense_solve.argtypes = [C.c_int, C.c_int, P, P]
    lib.orc_implicit_step.restype = C.c_int
    lib.orc_implicit_step.argtypes = [P, P, P, P, P, P, P, P, P, P, C.c_double, P]
    lib.orc_fix_solve.argtypes = [P, P, P, P, P]
    lib.orc_get_flux_emhd.argtypes = [P, P, C.c_int, P, P, P, P]
    lib.orc_imex_stage.restype = C.c_int
    lib.orc_imex_stage.argtypes = [P, P, P, C.c_int, C.c_double, P, P, P, P, P, P, P, P, P]
    lib.orc_imex_stage_flags.restype = C.c_int
    lib.orc_imex_stage_flags.argtypes = [P, P, P, C.c_int, C.c_double, P, P, P, P, P, P, P, P, P, P, P]
    _lib = lib
    return lib


def set_threads(n):
    """OpenMP threads of the oracle's parallel loops from now on; returns the previous maximum."""
    return int(load().orc_set_threads(int(n)))


def _ptr(a):
    assert a.flags["C_CONTIGUOUS"] and a.dtype == np.float64
    return a.ctypes.data_as(C.c_void_p)


def config_from_spec(spec):
    c = Config()
    c.nx1, c.nx2, c.nx3, c.ng = spec.nx1, spec.nx2, spec.nx3, spec.ng
    c.x1min, c.x2min, c.x3min = spec.x1min, spec.x2min, spec.x3min
    c.dx1, c.dx2, c.dx3 = spec.dx
    c.gam = spec.gam
    c.recon = RECON[spec.recon]
    c.riemann = 1 if spec.riemann == "hlle" else 0
    c.nvar = spec.nvar
    c.driver = 0 if spec.driver == "simple" else 1
    for x in range(6):
        c.bc[x] = BC[spec.bc[x]]
    c.check_inflow_inner_x1 = int(spec.check_inflow_inner_x1)
    c.check_inflow_outer_x1 = int(spec.check_inflow_outer_x1)
    c.zero_polar_flux = int(spec.zero_polar_flux)
    c.fix_polar_flux = int(spec.fix_polar_flux)
    c.fix_corner_inner = int(spec.fix_corner_inner)
    c.floors_on = int(spec.floors_on)
    c.floor_frame = FRAME[spec.floor_frame]
    c.recon_floors = int(spec.recon_floors and spec.floors_on)
    c.iter_max, c.err_tol = spec.iter_max, spec.err_tol
    c.fix_average_neighbors = int(spec.fix_average_neighbors)
    c.fix_atmosphere = int(spec.fix_atmosphere)
    c.cfl, c.dt_min, c.max_dt_increase = spec.cfl, spec.dt_min, spec.max_dt_increase
    c.inverter = 1 if spec.inverter == "kastaun" else 0
    c.fofc, c.fofc_polar_cells, c.fofc_eh_buffer = int(spec.fofc), spec.fofc_polar_cells, spec.fofc_eh_buffer
    c.r_horizon = spec.r_horizon
    c.ct_scheme = {"none": 0, "bs99": 1, "gs05_0": 2, "gs05_c": 3, "sg07": 3}[spec.b_ct]
    c.recon_lower = 1 if spec.low_order_edges else (2 if spec.low_order_poles else 0)
    c.recon_fallback = int(spec.recon_fallback and spec.floors_on)
    inner = spec.floors_inner if spec.floors_inner is not None else spec.floors
    for name, _ in Prescription._fields_:
        setattr(c.floors, name, type(getattr(c.floors, name))(getattr(spec.floors, name)))
        setattr(c.floors_inner, name, type(getattr(c.floors_inner, name))(getattr(inner, name)))
    c.frame_switch_r, c.frame_switch_beta = spec.frame_switch_r, spec.frame_switch_beta
    c.fofc_use_glf, c.fofc_use_source_term = int(spec.fofc_use_glf), int(spec.fofc_use_source_term)
    return c


def coords_from_spec(spec):
    s = CoordSpec()
    s.base, s.transform = BASE[spec.base], TRANSFORM[spec.transform]
    s.a, s.hslope, s.mks_smooth = spec.a, spec.hslope, spec.mks_smooth
    s.poly_xt, s.poly_alpha, s.startx1 = spec.poly_xt, spec.poly_alpha, spec.startx1
    return s


class Oracle:
    """One block in the CPU restatement.  Arrays are numpy float64 (nvar, n3, n2, n1)."""

    def __init__(self, spec):
        self.lib = load()
        self.spec = spec
        self._cfg = config_from_spec(spec)
        self._cs = coords_from_spec(spec)
        self.h = self.lib.orc_create(C.byref(self._cfg), C.byref(self._cs))
        self.shape = spec.shape
        n3, n2, n1 = self.shape
        self.N = n1 * n2 * n3

    def __del__(self):
        try:
            if self.h:
                self.lib.orc_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def geometry(self):
        n3, n2, n1 = self.shape
        G1, G2 = n1 + 1, n2 + 1
        g = {"gcov": np.zeros((7, G2, G1, 4, 4)), "gcon": np.zeros((7, G2, G1, 4, 4)),
             "gdet": np.zeros((7, G2, G1)), "gdet_conn": np.zeros((n2, n1, 4, 4, 4)),
             "r_center": np.zeros((n2, n1))}
        self.lib.orc_get_geometry(self.h, _ptr(g["gcov"]), _ptr(g["gcon"]), _ptr(g["gdet"]),
                                  _ptr(g["gdet_conn"]), _ptr(g["r_center"]))
        return g

    def set_geometry(self, g):
        arrs = [np.ascontiguousarray(g[k], dtype=np.float64) for k in ("gcov", "gcon", "gdet", "gdet_conn", "r_center")]
        self.lib.orc_set_geometry(self.h, *[_ptr(a) for a in arrs])
        self._keep = arrs

    def zeros(self):
        return np.zeros((self.spec.nvar,) + self.shape)

    def ptou(self, P):
        U = self.zeros()
        self.lib.orc_ptou(self.h, _ptr(P), _ptr(U))
        return U

    def boundaries(self, P, U):
        self.lib.orc_boundaries(self.h, _ptr(P), _ptr(U))

    def init_state(self, P):
        """Same initialisation sequence as kharma_b200.block.Block.set_prims."""
        P = np.ascontiguousarray(P, dtype=np.float64).copy()
        U = self.ptou(P)
        self.boundaries(P, U)
        self.lib.orc_ptou(self.h, _ptr(P), _ptr(U))
        return P, U

    def get_flux(self, dir, P):
        F = self.zeros()
        cmax = np.zeros(self.shape)
        cmin = np.zeros(self.shape)
        self.lib.orc_get_flux(self.h, dir, _ptr(P), _ptr(F), _ptr(cmax), _ptr(cmin))
        return F, cmax, cmin

    def fix_flux(self, F1, F2, F3):
        self.lib.orc_fix_flux(self.h, _ptr(F1), _ptr(F2), _ptr(F3))

    def utop(self, U, P):
        pflag = np.zeros(self.shape)
        fflag = np.zeros(self.shape)
        self.lib.orc_utop(self.h, _ptr(U), _ptr(P), _ptr(pflag), _ptr(fflag))
        return pflag, fflag

    def floors(self, P, U, pflag, fflag):
        self.lib.orc_floors(self.h, _ptr(P), _ptr(U), _ptr(pflag), _ptr(fflag))

    def fix_utop(self, P, U, pflag):
        """FixUtoP in place as a stage runs it (periodic images of P and pflag filled first)."""
        self.lib.orc_fix_utop(self.h, _ptr(P), _ptr(U), _ptr(pflag))

    def step(self, P, U, dt):
        """One RK2 step in place; returns (pflag, fflag, dt_next, min_ndt)."""
        pflag = np.zeros(self.shape)
        fflag = np.zeros(self.shape)
        dtn = C.c_double()
        mn = C.c_double()
        self.lib.orc_step(self.h, _ptr(P), _ptr(U), _ptr(pflag), _ptr(fflag), dt, C.byref(dtn), C.byref(mn))
        return pflag, fflag, dtn.value, mn.value

    # ---------------------------------------------------------------- B_CT (face fields (3, n3, n2, n1))
    def ct_init_state(self, P, Bf=None):
        """Same sequence as kharma_b200.block.Block.set_prims for a B_CT block: ghost zones, faces
        from the zone B unless given, the zone B from the faces, ghost zones again, U = U(P)."""
        P = np.ascontiguousarray(P, dtype=np.float64).copy()
        U = self.ptou(P)
        self.boundaries(P, U)
        if Bf is None:
            Bf = np.zeros((3,) + self.shape)
            self.lib.orc_ct_faces_from_prims(self.h, _ptr(P), _ptr(Bf))
        else:
            Bf = np.ascontiguousarray(Bf, dtype=np.float64).copy()
        self.lib.orc_ct_utop(self.h, _ptr(Bf), _ptr(P), _ptr(U))
        self.lib.orc_ct_boundaries(self.h, _ptr(P), _ptr(U), _ptr(Bf))
        self.lib.orc_ptou(self.h, _ptr(P), _ptr(U))
        return P, U, Bf

    def ct_step(self, P, U, Bf, dt):
        """One RK2 step with B_CT in place; returns (pflag, fflag, dt_next, min_ndt)."""
        pflag = np.zeros(self.shape)
        fflag = np.zeros(self.shape)
        dtn = C.c_double()
        mn = C.c_double()
        self.lib.orc_ct_step(self.h, _ptr(P), _ptr(U), _ptr(Bf), _ptr(pflag), _ptr(fflag), dt, C.byref(dtn), C.byref(mn))
        return pflag, fflag, dtn.value, mn.value

    def ct_max_divb(self, Bf):
        return self.lib.orc_ct_max_divb(self.h, _ptr(Bf))

    def max_divb(self, U, avoid_inner=False, avoid_outer=False):
        return self.lib.orc_max_divb(self.h, _ptr(U), int(avoid_inner), int(avoid_outer))

    # ---------------------------------------------------------------- EMHD and the implicit solve
    # Field arrays here are (10, n3, n2, n1): rho, u, u1..u3, B1..B3, q~, dP~.
    def connection(self):
        n3, n2, n1 = self.shape
        conn = np.zeros((n2, n1, 4, 4, 4))
        self.lib.orc_get_connection(self.h, _ptr(conn))
        return conn

    def zeros10(self):
        return np.zeros((10,) + self.shape)

    def emhd_ptou(self, emhd, P):
        U = self.zeros10()
        self.lib.orc_emhd_ptou(self.h, C.byref(emhd_params(emhd)), _ptr(P), _ptr(U))
        return U

    def emhd_add_source(self, emhd, P, dUdt):
        self.lib.orc_emhd_add_source(self.h, C.byref(emhd_params(emhd)), _ptr(P), _ptr(dUdt))

    def implicit_jacobian(self, emhd, imp, Pf, Uf, Ps, S, Psol, dt):
        nf = 5 + int(emhd.conduction) + int(emhd.viscosity)
        J = np.zeros((nf * nf,) + self.shape)
        res = np.zeros((nf,) + self.shape)
        self.lib.orc_implicit_jacobian(self.h, C.byref(emhd_params(emhd)), C.byref(implicit_params(imp)),
                                       _ptr(Pf), _ptr(Uf), _ptr(Ps), _ptr(S), _ptr(Psol), dt, _ptr(J), _ptr(res))
        return J, res

    def implicit_residual(self, emhd, Pf, Uf, Ps, S, Ptest, dt):
        nf = 5 + int(emhd.conduction) + int(emhd.viscosity)
        res = np.zeros((nf,) + self.shape)
        self.lib.orc_implicit_residual(self.h, C.byref(emhd_params(emhd)), _ptr(Pf), _ptr(Uf), _ptr(Ps), _ptr(S),
                                       _ptr(Ptest), dt, _ptr(res))
        return res

    def implicit_step(self, emhd, imp, Pf, Uf, Ps, S, Psol, solve_norm, solve_fail, dt):
        """Implicit::Step in place on Psol, solve_norm, solve_fail; returns (iterations, max norms)."""
        mx = np.zeros(imp.max_nonlinear_iter)
        it = self.lib.orc_implicit_step(self.h, C.byref(emhd_params(emhd)), C.byref(implicit_params(imp)),
                                        _ptr(Pf), _ptr(Uf), _ptr(Ps), _ptr(S), _ptr(Psol), _ptr(solve_norm),
                                        _ptr(solve_fail), dt, _ptr(mx))
        return it, mx[:it]

    def fix_solve(self, emhd, P, U, solve_fail):
        self.lib.orc_fix_solve(self.h, C.byref(emhd_params(emhd)), _ptr(P), _ptr(U), _ptr(solve_fail))

    def get_flux_emhd(self, emhd, dir, P):
        """EMHD face fluxes of the 10-slot state along dir: (F [10, ...], cmax, cmin)."""
        F = self.zeros10()
        cmax = np.zeros(self.shape)
        cmin = np.zeros(self.shape)
        self.lib.orc_get_flux_emhd(self.h, C.byref(emhd_params(emhd)), dir, _ptr(P), _ptr(F), _ptr(cmax), _ptr(cmin))
        return F, cmax, cmin

    def imex_stage(self, emhd, imp, stage, dt, Pfull, Ufull, Psub, Usub, solve_norm, solve_fail):
        """One ImEx stage (vl2 weights); returns (Pout, Uout, newton iterations, min zone dt)."""
        Pout, Uout = self.zeros10(), self.zeros10()
        mn = C.c_double()
        it = self.lib.orc_imex_stage(self.h, C.byref(emhd_params(emhd)), C.byref(implicit_params(imp)), stage, dt,
                                     _ptr(Pfull), _ptr(Ufull), _ptr(Psub), _ptr(Usub), _ptr(Pout), _ptr(Uout),
                                     _ptr(solve_norm), _ptr(solve_fail), C.byref(mn))
        return Pout, Uout, it, mn.value

    def imex_stage_flags(self, emhd, imp, stage, dt, Pfull, Ufull, Psub, Usub, solve_norm, solve_fail):
        """imex_stage with the interior floor and EMHD-limit flags: (Pout, Uout, iterations, min zone dt,
        fflag, eflag)."""
        Pout, Uout = self.zeros10(), self.zeros10()
        fflag, eflag = np.zeros(self.shape), np.zeros(self.shape)
        mn = C.c_double()
        it = self.lib.orc_imex_stage_flags(self.h, C.byref(emhd_params(emhd)), C.byref(implicit_params(imp)), stage,
                                           dt, _ptr(Pfull), _ptr(Ufull), _ptr(Psub), _ptr(Usub), _ptr(Pout),
                                           _ptr(Uout), _ptr(solve_norm), _ptr(solve_fail), C.byref(mn),
                                           _ptr(fflag), _ptr(eflag))
        return Pout, Uout, it, mn.value, fflag, eflag


class EmhdParams(C.Structure):
    _fields_ = [("type", C.c_int32), ("higher_order_terms", C.c_int32), ("feedback", C.c_int32),
                ("conduction", C.c_int32), ("viscosity", C.c_int32), ("stability_limits", C.c_int32),
                ("tau", C.c_double), ("conduction_alpha", C.c_double), ("viscosity_alpha", C.c_double),
                ("kappa", C.c_double), ("eta", C.c_double)]


class ImplicitParams(C.Structure):
    _fields_ = [("min_nonlinear_iter", C.c_int32), ("max_nonlinear_iter", C.c_int32), ("use_qr", C.c_int32),
                ("linesearch", C.c_int32), ("max_linesearch_iter", C.c_int32), ("jacobian", C.c_int32),
                ("jacobian_delta", C.c_double), ("rootfind_tol", C.c_double),
                ("linesearch_eps", C.c_double), ("linesearch_lambda", C.c_double)]


CLOSURE = {"constant": 0, "soundspeed": 1, "sound_speed": 1, "kappa_eta": 2, "torus": 3}


def emhd_params(e):
    s = EmhdParams()
    s.type = CLOSURE[e.closure_type]
    s.higher_order_terms, s.feedback = int(e.higher_order_terms), int(e.feedback)
    s.conduction, s.viscosity = int(e.conduction), int(e.viscosity)
    s.stability_limits = int(getattr(e, "stability_limits", False))
    s.tau, s.conduction_alpha, s.viscosity_alpha = e.tau, e.conduction_alpha, e.viscosity_alpha
    s.kappa, s.eta = e.kappa, e.eta
    return s


def implicit_params(p):
    s = ImplicitParams()
    s.min_nonlinear_iter, s.max_nonlinear_iter = p.min_nonlinear_iter, p.max_nonlinear_iter
    s.use_qr, s.linesearch, s.max_linesearch_iter = int(p.use_qr), int(p.linesearch), p.max_linesearch_iter
    s.jacobian = 1 if p.jacobian == "exact" else 0
    s.jacobian_delta, s.rootfind_tol = p.jacobian_delta, p.rootfind_tol
    s.linesearch_eps, s.linesearch_lambda = p.linesearch_eps, p.linesearch_lambda
    return s


def dense_solve(A, b, use_qr=True):
    """The reference's per-zone dense solve (QR with column pivoting, or its LU path) on one system."""
    A = np.ascontiguousarray(A, dtype=np.float64).copy()
    b = np.ascontiguousarray(b, dtype=np.float64).copy()
    load().orc_dense_solve(A.shape[0], int(use_qr), _ptr(A), _ptr(b))
    return b

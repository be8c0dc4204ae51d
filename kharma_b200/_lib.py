"""ctypes binding of libkhb (include/khb.h).

The shared library is built in-tree (kharma_b200/lib/libkhb.so) by kharma_b200.build.  There is
no fallback: if the library is missing, or a call fails, an exception is raised.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# KHB_LIB_PATH selects another build of the same library (e.g. a variant under test)
LIB_PATH = os.environ.get("KHB_LIB_PATH", os.path.join(_HERE, "lib", "libkhb.so"))

MAX_VARS = 10
Q, DP = 8, 9           # khb_fields slots of the EMHD variables

# enums (include/khb.h)
RECON = {"donor_cell": 0, "donor_cell_c": 0, "linear_mc": 1, "weno5": 2, "ppm": 3, "linear_vl": 4, "weno5_linear": 5,
         "ppmx": 6, "mp5": 7}
FLUX = {"llf": 0, "hlle": 1}
# "dirichlet" and "bondi" faces hold the ghost values the caller set (boundaries/dirichlet.cpp restores
# the values saved at initialisation; the bondi faces, the analytic solution): the exchange face's
# carry-over of the ghost shell gives the same ghost zones
BC = {"periodic": 0, "outflow": 1, "reflecting": 2, "exchange": 3, "transmitting": 4, "dirichlet": 3, "bondi": 3}
FRAME = {"fluid": 0, "normal": 1, "drift": 2, "mixed": 3, "mixed_fluid_normal": 3, "mixed_normal_drift": 4}
PREC = {"fp64": 0, "fp32_flux": 1}
INVERTER = {"onedw": 0, "kastaun": 1}
CT_SCHEME = {"none": 0, "bs99": 1, "gs05_0": 2, "gs05_c": 3, "sg07": 3}
BASE = {"cartesian_minkowski": 0, "spherical_minkowski": 1, "spherical_ks": 2, "spherical_bl": 3}
TRANSFORM = {"null": 0, "eks": 1, "mks": 2, "fmks": 3}
CLOSURE = {"constant": 0, "soundspeed": 1, "sound_speed": 1, "kappa_eta": 2, "torus": 3}
JACOBIAN = {"fd": 0, "exact": 1}
SOLVE = {"converged": 0, "fail": 1, "beyond_tol": 2, "backtrack": 3}


class KhbFloors(C.Structure):
    _fields_ = [
        ("rho_min_const", C.c_double), ("u_min_const", C.c_double),
        ("rho_min_geom", C.c_double), ("u_min_geom", C.c_double), ("r_char", C.c_double),
        ("bsq_over_rho_max", C.c_double), ("bsq_over_u_max", C.c_double), ("u_over_rho_max", C.c_double),
        ("ktot_max", C.c_double), ("gamma_max", C.c_double),
        ("use_r_char", C.c_int32), ("temp_adjust_u", C.c_int32), ("adjust_k", C.c_int32),
        ("radius_dependent_floors", C.c_int32),
        ("floors_switch_r", C.c_double),
    ]


class KhbConfig(C.Structure):
    _fields_ = [
        ("nx1", C.c_int32), ("nx2", C.c_int32), ("nx3", C.c_int32), ("ng", C.c_int32),
        ("dx1", C.c_double), ("dx2", C.c_double), ("dx3", C.c_double),
        ("gam", C.c_double),
        ("nvar", C.c_int32),
        ("recon", C.c_int32), ("riemann", C.c_int32), ("precision", C.c_int32),
        ("bc", C.c_int32 * 6),
        ("check_inflow_inner_x1", C.c_int32), ("check_inflow_outer_x1", C.c_int32),
        ("zero_polar_flux", C.c_int32),
        ("fix_polar_flux", C.c_int32),
        ("fix_corner_inner", C.c_int32),
        ("spherical", C.c_int32),
        ("cart_minkowski", C.c_int32),
        ("floors_on", C.c_int32), ("floor_frame", C.c_int32), ("recon_floors", C.c_int32),
        ("iter_max", C.c_int32), ("err_tol", C.c_double),
        ("fix_average_neighbors", C.c_int32), ("fix_atmosphere", C.c_int32),
        ("floors", KhbFloors),
        ("inverter", C.c_int32),
        ("fofc", C.c_int32), ("fofc_polar_cells", C.c_int32),
        ("fofc_eh_buffer", C.c_double), ("r_horizon", C.c_double),
        ("ct_scheme", C.c_int32),
        ("recon_lower", C.c_int32), ("recon_fallback", C.c_int32),
        ("floors_inner", KhbFloors),
        ("frame_switch_r", C.c_double), ("frame_switch_beta", C.c_double),
        ("fofc_use_glf", C.c_int32), ("fofc_use_source_term", C.c_int32),
    ]


class KhbCoords(C.Structure):
    _fields_ = [
        ("base", C.c_int32), ("transform", C.c_int32),
        ("a", C.c_double), ("hslope", C.c_double), ("mks_smooth", C.c_double),
        ("poly_xt", C.c_double), ("poly_alpha", C.c_double), ("startx1", C.c_double),
    ]


class KhbFields(C.Structure):
    _fields_ = [("v", C.c_void_p * MAX_VARS)]


class KhbEmhdParams(C.Structure):
    _fields_ = [("closure", C.c_int32), ("higher_order_terms", C.c_int32), ("feedback", C.c_int32),
                ("conduction", C.c_int32), ("viscosity", C.c_int32), ("stability_limits", C.c_int32),
                ("tau", C.c_double), ("conduction_alpha", C.c_double), ("viscosity_alpha", C.c_double),
                ("kappa", C.c_double), ("eta", C.c_double)]


class KhbImplicitParams(C.Structure):
    _fields_ = [("min_nonlinear_iter", C.c_int32), ("max_nonlinear_iter", C.c_int32), ("use_qr", C.c_int32),
                ("linesearch", C.c_int32), ("max_linesearch_iter", C.c_int32), ("jacobian", C.c_int32),
                ("jacobian_delta", C.c_double), ("rootfind_tol", C.c_double),
                ("linesearch_eps", C.c_double), ("linesearch_lambda", C.c_double)]


# Every entry point declared in include/khb.h, with its ctypes signature
_P = C.c_void_p
_D = C.c_double
_I = C.c_int
SIGNATURES = {
    "khb_last_error": (C.c_char_p, []),
    "khb_version": (_I, []),
    "khb_create": (_I, [C.POINTER(KhbConfig), C.POINTER(_P)]),
    "khb_destroy": (_I, [_P]),
    "khb_build_geometry": (_I, [C.POINTER(KhbCoords), C.POINTER(KhbConfig), _D, _D, _D, _P, _P, _P, _P, _P]),
    "khb_set_geometry": (_I, [_P, _P, _P, _P, _P, _P]),
    "khb_get_flux": (_I, [_P, _I, C.POINTER(KhbFields), _P]),
    "khb_fix_flux": (_I, [_P, _P]),
    "khb_fofc": (_I, [_P, _I, _D, C.POINTER(KhbFields), C.POINTER(KhbFields), C.POINTER(KhbFields), _P]),
    "khb_flux_ct": (_I, [_P, _P]),
    "khb_copy_flux": (_I, [_P, _I, C.POINTER(KhbFields), _P, _P]),
    "khb_update": (_I, [_P, C.POINTER(KhbFields), C.POINTER(KhbFields), C.POINTER(KhbFields), _D, _D, _D,
                        C.POINTER(KhbFields), _P]),
    "khb_utop": (_I, [_P, C.POINTER(KhbFields), C.POINTER(KhbFields), _P, _P, _P]),
    "khb_apply_floors": (_I, [_P, C.POINTER(KhbFields), C.POINTER(KhbFields), _P, _P, _P]),
    "khb_fix_utop": (_I, [_P, C.POINTER(KhbFields), C.POINTER(KhbFields), _P, _P]),
    "khb_boundaries": (_I, [_P, C.POINTER(KhbFields), C.POINTER(KhbFields), _P]),
    "khb_ptou": (_I, [_P, C.POINTER(KhbFields), C.POINTER(KhbFields), _P]),
    "khb_stage": (_I, [_P, _I, _D, C.POINTER(KhbFields), C.POINTER(KhbFields), C.POINTER(KhbFields),
                       C.POINTER(KhbFields), C.POINTER(KhbFields), _P, _P, _P]),
    "khb_zone_pass": (_I, [_P, _I, _D, C.POINTER(KhbFields), C.POINTER(KhbFields), C.POINTER(KhbFields),
                           C.POINTER(KhbFields), C.POINTER(KhbFields), _P, _P, _P]),
    "khb_fix_utop_list": (_I, [_P, C.POINTER(KhbFields), C.POINTER(KhbFields), _P, _P]),
    "khb_step": (_I, [_P, _D, C.POINTER(KhbFields), C.POINTER(KhbFields), _P, _P, _P]),
    "khb_get_min_ndt": (_I, [_P, C.POINTER(_D), _P]),
    "khb_set_timestep": (_I, [_P, _D, _D, _D, _D]),
    "khb_get_timestep": (_I, [_P, C.POINTER(_D), C.POINTER(_D), C.POINTER(_D), _P]),
    "khb_step_device_dt": (_I, [_P, C.POINTER(KhbFields), C.POINTER(KhbFields), _P, _P, _P]),
    "khb_step_graph": (_I, [_P, C.POINTER(KhbFields), C.POINTER(KhbFields), _P, _P, _P]),
    "khb_step_host": (_I, [_P, C.POINTER(_P), C.POINTER(KhbFields), C.POINTER(KhbFields), _P, _P, _P]),
    "khb_step_host_interior": (_I, [_P, C.POINTER(_P), C.POINTER(KhbFields), C.POINTER(KhbFields), _P, _P, _P]),
    "khb_adjoint_step": (_I, [_P, _D, C.POINTER(KhbFields), C.POINTER(KhbFields), C.POINTER(KhbFields),
                              C.POINTER(KhbFields), C.POINTER(KhbFields), _P, _D, _P]),
    "khb_adjoint_ptou": (_I, [_P, C.POINTER(KhbFields), C.POINTER(KhbFields), C.POINTER(KhbFields), _P]),
    "khb_flux_dot": (_I, [_P, _I, _I, _P, _D, _P, _P]),
    "khb_ct_stage": (_I, [_P, _I, _D] + [C.POINTER(KhbFields)] * 8 + [_P, _P, _P]),
    "khb_ct_stage_fluxes": (_I, [_P, C.POINTER(KhbFields), _P]),
    "khb_ct_stage_update": (_I, [_P, _I, _D] + [C.POINTER(KhbFields)] * 8 + [_P, _P, _P]),
    "khb_ct_stage_update_part": (_I, [_P, _I, _I, _D] + [C.POINTER(KhbFields)] * 8 + [_P, _P, _P]),
    "khb_ct_ghost_from_faces": (_I, [_P, C.POINTER(KhbFields), C.POINTER(KhbFields), C.POINTER(KhbFields), _P]),
    "khb_ctmesh_create": (_I, [C.POINTER(_P), _I, _P, C.c_int64, _P, _I, _P, C.c_int64, _P, _I, _P, C.c_int64, _P,
                               C.c_int64, C.POINTER(_P)]),
    "khb_ctmesh_destroy": (_I, [_P]),
    "khb_ctmesh_correct": (_I, [_P, _P]),
    "khb_ctmesh_exchange": (_I, [_P, _P, _P, _P]),
    "khb_ctmesh_exchange_cons": (_I, [_P] * 8),
    "khb_ct_step": (_I, [_P, _D, C.POINTER(KhbFields), C.POINTER(KhbFields), C.POINTER(KhbFields), _P, _P, _P]),
    "khb_ct_boundaries": (_I, [_P, C.POINTER(KhbFields), C.POINTER(KhbFields), C.POINTER(KhbFields), _P]),
    "khb_ct_utop": (_I, [_P, C.POINTER(KhbFields), C.POINTER(KhbFields), C.POINTER(KhbFields), _P]),
    "khb_ct_faces_from_prims": (_I, [_P, C.POINTER(KhbFields), C.POINTER(KhbFields), _P]),
    "khb_ct_max_divb": (_I, [_P, C.POINTER(KhbFields), C.POINTER(_D), _P]),
    "khb_max_divb": (_I, [_P, C.POINTER(KhbFields), C.POINTER(_D), _P]),
    "khb_launch_count": (C.c_int64, [_P]),
    "khb_set_tuning": (_I, [_P, C.c_char_p, _I]),
    "khb_max_divb_noalloc": (_I, [C.POINTER(KhbConfig), C.POINTER(KhbFields), _P, _P]),
    "khb_noalloc_last_error": (C.c_char_p, []),
    "khb_build_connection": (_I, [C.POINTER(KhbCoords), C.POINTER(KhbConfig), _D, _D, _D, _P]),
    "khb_set_connection": (_I, [_P, _P]),
    "khb_emhd_ptou": (_I, [_P, C.POINTER(KhbEmhdParams), C.POINTER(KhbFields), C.POINTER(KhbFields), _P]),
    "khb_emhd_add_source": (_I, [_P, C.POINTER(KhbEmhdParams), C.POINTER(KhbFields), C.POINTER(KhbFields), _P]),
    "khb_implicit_step": (_I, [_P, C.POINTER(KhbEmhdParams), C.POINTER(KhbImplicitParams), C.POINTER(KhbFields),
                               C.POINTER(KhbFields), C.POINTER(KhbFields), C.POINTER(KhbFields),
                               C.POINTER(KhbFields), _P, _P, _D, _P]),
    "khb_implicit_stats": (_I, [_P, C.POINTER(C.c_int32), _P, _P]),
    "khb_implicit_jacobian": (_I, [_P, C.POINTER(KhbEmhdParams), C.POINTER(KhbImplicitParams),
                                   C.POINTER(KhbFields), C.POINTER(KhbFields), C.POINTER(KhbFields),
                                   C.POINTER(KhbFields), C.POINTER(KhbFields), _D, _P, _P, _P]),
    "khb_fix_solve": (_I, [_P, C.POINTER(KhbEmhdParams), C.POINTER(KhbFields), C.POINTER(KhbFields), _P, _P]),
    "khb_get_flux_emhd": (_I, [_P, C.POINTER(KhbEmhdParams), _I, C.POINTER(KhbFields), _P]),
    "khb_copy_flux_emhd": (_I, [_P, _I, C.POINTER(KhbFields), _P, _P]),
    "khb_imex_stage": (_I, [_P, C.POINTER(KhbEmhdParams), C.POINTER(KhbImplicitParams), _I, _D,
                            C.POINTER(KhbFields), C.POINTER(KhbFields), C.POINTER(KhbFields), C.POINTER(KhbFields),
                            C.POINTER(KhbFields), C.POINTER(KhbFields), _P, _P, _P]),
    "khb_imex_stage_flags": (_I, [_P, C.POINTER(KhbEmhdParams), C.POINTER(KhbImplicitParams), _I, _D,
                                  C.POINTER(KhbFields), C.POINTER(KhbFields), C.POINTER(KhbFields),
                                  C.POINTER(KhbFields), C.POINTER(KhbFields), C.POINTER(KhbFields), _P, _P, _P, _P,
                                  _P]),
    "khb_batch_create": (_I, [C.POINTER(_P), _I, C.POINTER(KhbFields), C.POINTER(KhbFields), C.POINTER(_P),
                              C.POINTER(_P), C.POINTER(_P)]),
    "khb_batch_destroy": (_I, [_P]),
    "khb_batch_step": (_I, [_P, _D, _P]),
    "khb_batch_step_graph": (_I, [_P, _D, _P]),
    "khb_batch_get_min_ndt": (_I, [_P, C.POINTER(_D), _P]),
    "khb_batch_classes": (_I, [_P, C.POINTER(C.c_int32), _P, _P, _I]),
    "khb_batch_set_tuning": (_I, [_P, _I, _I, _I]),
    "khb_batch_autotune": (_I, [_P, _I, _P, C.POINTER(C.c_int32), _P]),
    "khb_batch_launch_count": (C.c_int64, [_P]),
    "khb_batch_set_plan": (_I, [_P, _I]),
    "khb_bounds_checked": (_I, []),
    "khb_bounds_status": (_I, [_P, C.POINTER(C.c_uint64), _P]),
    "khb_batch_get_plan": (_I, [_P, C.POINTER(C.c_int32)]),
    "khb_batch_set_mesh": (_I, [_P, _P, C.c_int64, C.c_int64, _P, C.c_int64]),
    "khb_batch_mesh_exchange": (_I, [_P, _P]),
    "khb_batch_set_mesh_sync": (_I, [_P, C.c_int]),
    "khb_get_flux_planes": (_I, [_P, _I, C.POINTER(KhbFields), _I, _I, _P]),
}

_lib = None


class KhbError(RuntimeError):
    pass


def load():
    """Load libkhb.so (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise KhbError(f"{LIB_PATH} is missing: build it with `python -m kharma_b200.build`")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc, what=""):
    """Raise KhbError with the library's message on a nonzero return code."""
    if rc != 0:
        msg = load().khb_last_error().decode(errors="replace")
        raise KhbError(f"{what} failed ({rc}): {msg}")

"""The C ABI library: it loads, exports every entry point include/khb.h declares, and its host-side
geometry builder reproduces the oracle's GRCoordinates caches (CPU only, no device calls)."""
import os
import re

import numpy as np
import pytest

from kharma_b200 import _lib
from kharma_b200.block import build_geometry
from kharma_b200.spec import atmosphere_spec, mhdmodes_spec, torus_spec

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "khb.h")).read()
    return sorted(set(re.findall(r"\b(khb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, f"libkhb.so lacks {missing}"
    assert set(syms) == set(_lib.SIGNATURES), "ctypes signatures out of sync with include/khb.h"


def test_config_struct_layout():
    # offsets a C caller relies on (include/khb.h khb_config)
    assert _lib.KhbFloors.floors_switch_r.offset == 96
    assert _lib.KhbConfig.err_tol.offset == 136
    assert _lib.KhbConfig.floors.offset == 152


def test_create_rejects_bad_config():
    import ctypes as C
    lib = _lib.load()
    cfg = mhdmodes_spec(16, 16, 1).khb_config()
    cfg.nvar = 7
    ctx = C.c_void_p()
    assert lib.khb_create(C.byref(cfg), C.byref(ctx)) == -4
    assert b"nvar" in lib.khb_last_error()
    cfg = mhdmodes_spec(16, 16, 1).khb_config()
    cfg.ng = 2
    assert lib.khb_create(C.byref(cfg), C.byref(ctx)) == -1


@pytest.mark.parametrize("spec", [mhdmodes_spec(16, 16, 1), mhdmodes_spec(8, 8, 8),
                                  torus_spec(32, 24, 8), torus_spec(24, 16, 1)],
                         ids=["minkowski2d", "minkowski3d", "fmks3d", "fmks2d"])
def test_geometry_matches_oracle(oracle_mod, spec):
    go = oracle_mod.Oracle(spec).geometry()
    gp = build_geometry(spec)
    for key in go:
        assert np.array_equal(go[key], gp[key]), f"{key} differs from the oracle"


def test_emhd_struct_layout():
    # include/khb.h khb_emhd_params / khb_implicit_params
    assert C_sizeof(_lib.KhbEmhdParams) == 64 and _lib.KhbEmhdParams.tau.offset == 24
    assert C_sizeof(_lib.KhbImplicitParams) == 56 and _lib.KhbImplicitParams.jacobian_delta.offset == 24
    assert C_sizeof(_lib.KhbFields) == 8 * _lib.MAX_VARS == 80


def C_sizeof(t):
    import ctypes
    return ctypes.sizeof(t)


@pytest.mark.parametrize("spec", [atmosphere_spec(64, 8, 1), torus_spec(24, 16, 4)], ids=["mks_ks", "fmks"])
def test_connection_matches_oracle(oracle_mod, spec):
    from kharma_b200.emhd import build_connection
    assert np.array_equal(oracle_mod.Oracle(spec).connection(), build_connection(spec))

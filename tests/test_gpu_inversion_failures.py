"""Inversion failures on the GPU against the oracle: poisoned conserved states (negative D, NaN energy,
a hot state that exhausts 1D_W's iterations, superluminal momenta) at isolated zones, zones on the X1
face and the periodic x3 edge, adjacent pairs and a 3x3x3 cluster, in an FMKS torus block.

Every case asserts that zones fail (pflag > 0), that pflag and fflag equal the oracle's bit for bit and
that P and U after FixUtoP agree to 1e-12 relative per variable (the FP64 tolerance of the parity
tests).  Reference: inverter/invert_template.hpp:53 (statuses), inverter/onedw.hpp:99-101, 196-208,
inverter/kastaun.hpp, inverter/fixup.cpp:47-156, floors/floors_impl.hpp:45-128.
"""
import numpy as np
import pytest
import torch

from kharma_b200 import problems
from kharma_b200.block import Block
from kharma_b200.spec import torus_spec

import poison_cases as pc

pytestmark = pytest.mark.gpu

RTOL = 1e-12

# inverter, fix_average_neighbors, fix_atmosphere
OPTIONS = [
    ("onedw", True, True),       # the 1D_W defaults
    ("onedw", False, True),      # atmosphere only: failed zones go to the floors
    ("onedw", False, False),     # FixUtoP off: failed zones keep the guess
    ("kastaun", False, True),    # the Kastaun defaults
    ("kastaun", True, True),
]


def rel_err(a, b, sl):
    out = []
    for v in range(a.shape[0]):
        x, y = a[v][sl], b[v][sl]
        scale = np.max(np.abs(y))
        d = np.max(np.abs(x - y))
        out.append(d / scale if scale > 0 else d)
    return np.array(out)


def setup(oracle_mod, inverter, fix_avg, fix_atmo):
    spec = torus_spec(32, 24, 8, inverter=inverter)
    spec.fix_average_neighbors = fix_avg
    spec.fix_atmosphere = fix_atmo
    o = oracle_mod.Oracle(spec)
    geom = o.geometry()
    P0 = problems.fm_torus(spec, geom, seed=7)
    b = Block(spec, geometry=geom)
    b.set_prims(P0)
    Po, Uo = o.init_state(P0)
    return spec, o, b, Po, Uo


def label(opt):
    return f"{opt[0]}-avg{int(opt[1])}-atmo{int(opt[2])}"


@pytest.mark.parametrize("opt", OPTIONS, ids=label)
def test_utop_floors_fixup_match_oracle(oracle_mod, opt):
    """Package level: khb_utop, khb_apply_floors, khb_fix_utop on a poisoned U against the oracle's
    BlockUtoP, ApplyGRMHDFloors and FixUtoP."""
    spec, o, b, Po, Uo = setup(oracle_mod, *opt)
    U = Uo.copy()
    P = Po.copy()
    pc.poison(U, spec)
    b.U.copy_(torch.from_numpy(U))
    b.P.copy_(torch.from_numpy(P))
    pf_o, ff_o = o.utop(U, P)
    o.floors(P, U, pf_o, ff_o)
    b.utop(b.U, b.P, b.pflag, b.fflag)
    b.apply_floors(b.P, b.U, b.pflag, b.fflag)
    sl = spec.interior
    pf_g = b.pflag.cpu().numpy()[sl]
    ff_g = b.fflag.cpu().numpy()[sl]
    nfail = np.count_nonzero(pf_o[sl] > 0)
    assert nfail > 0
    assert np.array_equal(pf_g, pf_o[sl].astype(np.int32))
    assert np.array_equal(ff_g, ff_o[sl].astype(np.int32))
    o.fix_utop(P, U, pf_o)
    b.fix_utop(b.P, b.U, b.pflag)
    Pg, Ug = b.P.cpu().numpy(), b.U.cpu().numpy()
    psl = (slice(0, 5),) + sl
    assert np.all(np.isfinite(Pg[psl])) == np.all(np.isfinite(P[psl]))
    # zones whose fixup is off keep a NaN-free guess in P; U keeps the poison there, as in the oracle
    eP = rel_err(np.nan_to_num(Pg, nan=7.0), np.nan_to_num(P, nan=7.0), sl)
    eU = rel_err(np.nan_to_num(Ug, nan=7.0), np.nan_to_num(U, nan=7.0), sl)
    assert np.all(eP <= RTOL), eP
    assert np.all(eU <= RTOL), eU
    assert np.array_equal(np.isnan(Ug[(slice(None),) + sl]), np.isnan(U[(slice(None),) + sl]))


@pytest.mark.parametrize("opt", OPTIONS, ids=label)
def test_step_from_poisoned_state_matches_oracle(oracle_mod, opt):
    """Step level: U_0 poisoned before khb_step; both stages fail at the poisoned zones, FixUtoP and
    the lock-step P->U run inside the step.  Two more clean steps follow."""
    spec, o, b, Po, Uo = setup(oracle_mod, *opt)
    pc.poison(Uo, spec)
    b.U.copy_(torch.from_numpy(Uo))
    sl = spec.interior
    dt = spec.dt_min
    for n in range(3):
        pf_o, ff_o, dtn, mn_o = o.step(Po, Uo, dt)
        b.step(dt)
        mn_g = b.min_ndt()
        pf_g = b.pflag.cpu().numpy()[sl]
        ff_g = b.fflag.cpu().numpy()[sl]
        if n == 0:
            assert np.count_nonzero(pf_o[sl] > 0) > 0
        assert np.array_equal(pf_g, pf_o[sl].astype(np.int32)), f"step {n}: pflag differs"
        assert np.array_equal(ff_g, ff_o[sl].astype(np.int32)), f"step {n}: fflag differs"
        Pg, Ug = b.P.cpu().numpy(), b.U.cpu().numpy()
        eP = rel_err(np.nan_to_num(Pg, nan=7.0), np.nan_to_num(Po, nan=7.0), sl)
        eU = rel_err(np.nan_to_num(Ug, nan=7.0), np.nan_to_num(Uo, nan=7.0), sl)
        assert np.all(eP <= RTOL), (n, eP)
        assert np.all(eU <= RTOL), (n, eU)
        assert abs(mn_g - mn_o) <= RTOL * abs(mn_o), (mn_g, mn_o)
        dt = dtn

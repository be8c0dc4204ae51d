"""First-order flux correction in the oracle (flux/fofc.cpp:45-226, kharma_driver.cpp:292-337), CPU only.

The correction replaces the fluxes of faces next to zones whose guess update would hit floors, or
that lie within eh_buffer of the horizon, by donor-cell LLF fluxes.  So it must change nothing where
neither can happen (the Cartesian linear mode: no floors, no horizon), and on the torus it must
change the state exactly around the zones it can flag (inside the horizon plus buffer, or floored).
"""
import dataclasses

import numpy as np

from kharma_b200 import problems
from kharma_b200.spec import mhdmodes_spec, torus_spec


def run(oracle_mod, spec, P0, nsteps):
    o = oracle_mod.Oracle(spec)
    P, U = o.init_state(P0)
    dt = spec.dt_min
    for _ in range(nsteps):
        pflag, fflag, dt, _ = o.step(P, U, dt)
    return P, U, pflag, fflag, o


def test_fofc_changes_nothing_without_floors_or_horizon(oracle_mod):
    sp = mhdmodes_spec(16, 16, 1)
    P0 = problems.mhdmodes(sp, 3)
    a = run(oracle_mod, sp, P0, 5)
    b = run(oracle_mod, dataclasses.replace(sp, fofc=True), P0, 5)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_fofc_acts_near_the_horizon(oracle_mod):
    sp = torus_spec(32, 24, 8)
    o = oracle_mod.Oracle(sp)
    P0 = problems.fm_torus(sp, o.geometry(), seed=7)
    a = run(oracle_mod, sp, P0, 1)
    b = run(oracle_mod, dataclasses.replace(sp, fofc=True), P0, 1)
    sl = sp.interior
    changed = np.any(a[0][:, sl[0], sl[1], sl[2]] != b[0][:, sl[0], sl[1], sl[2]], axis=0)
    r = np.broadcast_to(o.geometry()["r_center"][None], sp.shape)[sl]
    r_mark = sp.r_horizon + sp.fofc_eh_buffer
    # every zone inside the marked radius is updated with first-order fluxes
    assert changed[r < r_mark].all()
    assert np.isfinite(b[0]).all()


def test_fofc_options_change_the_correction(oracle_mod):
    """fofc/use_glf puts the speed of light on every replaced face (fofc.cpp:200-205) and
    fofc/use_source_term adds the geometric source to the guess (kharma_driver.cpp:308-312): each
    changes the corrected torus step against the default options, and neither touches zones far from
    any flagged face."""
    sp = dataclasses.replace(torus_spec(32, 24, 8), fofc=True)
    o = oracle_mod.Oracle(sp)
    P0 = problems.fm_torus(sp, o.geometry(), seed=7)
    base = run(oracle_mod, sp, P0, 3)
    glf = run(oracle_mod, dataclasses.replace(sp, fofc_use_glf=True), P0, 3)
    src = run(oracle_mod, dataclasses.replace(sp, fofc_use_source_term=True), P0, 3)
    assert not np.array_equal(base[0], glf[0])
    assert not np.array_equal(base[0], src[0])
    assert np.isfinite(glf[0]).all() and np.isfinite(src[0]).all()
    # without floors or a horizon nothing is flagged, so neither option changes anything
    sm = mhdmodes_spec(16, 16, 1)
    Pm = problems.mhdmodes(sm, 3)
    a = run(oracle_mod, dataclasses.replace(sm, fofc=True), Pm, 3)
    for opt in ({"fofc_use_glf": True}, {"fofc_use_source_term": True}):
        b = run(oracle_mod, dataclasses.replace(sm, fofc=True, **opt), Pm, 3)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])

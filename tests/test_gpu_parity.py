"""Parity of the CUDA path (through the C ABI) with the CPU oracle on identical inputs.

Tolerance for the FP64 path: for every variable v, max |x_gpu - x_oracle| <= 1e-12 * max |x_oracle,v|
(per-variable relative L-infinity).  Inversion and floor flags must agree bit for bit.
"""
import dataclasses

import numpy as np
import pytest
import torch

from kharma_b200 import problems
from kharma_b200.block import Block
from kharma_b200.spec import mhdmodes_spec, torus_spec

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def rel_err(a, b, sl=None):
    """Per-variable max |a-b| / max |b| over the (optionally sliced) block."""
    out = []
    for v in range(a.shape[0]):
        x, y = (a[v], b[v]) if sl is None else (a[v][sl], b[v][sl])
        scale = np.max(np.abs(y))
        d = np.max(np.abs(x - y))
        out.append(d / scale if scale > 0 else d)
    return np.array(out)


def make_pair(oracle_mod, spec, P0):
    o = oracle_mod.Oracle(spec)
    geom = o.geometry()
    b = Block(spec, geometry=geom)
    b.set_prims(P0)
    Po, Uo = o.init_state(P0)
    return o, b, Po, Uo


def torus_init(spec, o):
    return problems.fm_torus(spec, o.geometry(), seed=7)


CASES = {
    "mhdmodes3d_weno5": lambda: mhdmodes_spec(16, 16, 16, recon="weno5"),
    "mhdmodes2d_ppm_hlle": lambda: mhdmodes_spec(24, 24, 1, recon="ppm", riemann="hlle"),
    "torus3d_mc": lambda: torus_spec(32, 24, 8),
}


def initial(oracle_mod, name, spec):
    if name.startswith("torus"):
        return torus_init(spec, oracle_mod.Oracle(spec))
    return problems.mhdmodes(spec, 3)


@pytest.mark.parametrize("name", list(CASES))
def test_initial_state_parity(oracle_mod, name):
    spec = CASES[name]()
    o, b, Po, Uo = make_pair(oracle_mod, spec, initial(oracle_mod, name, spec))
    torch.cuda.synchronize()
    assert np.all(rel_err(b.P.cpu().numpy(), Po) <= RTOL)
    assert np.all(rel_err(b.U.cpu().numpy(), Uo) <= RTOL)


@pytest.mark.parametrize("name", list(CASES))
def test_face_flux_parity(oracle_mod, name):
    spec = CASES[name]()
    o, b, Po, Uo = make_pair(oracle_mod, spec, initial(oracle_mod, name, spec))
    ng = spec.ng
    for d in range(1, spec.ndim + 1):
        Fo, cmax, cmin = o.get_flux(d, Po)
        b.get_flux(d)
        Fg, ctop = b.copy_flux(d)
        torch.cuda.synchronize()
        Fg = Fg.cpu().numpy()
        ctop = ctop.cpu().numpy()
        # consumer face range: [s, e+1] along d, [s-1, e+1] across
        sl = []
        for ax, (n, nx) in enumerate(zip((spec.nx3, spec.nx2, spec.nx1), (3, 2, 1))):
            if n == 1:
                sl.append(slice(0, 1))
            elif nx == d:
                sl.append(slice(ng, ng + n + 1))
            else:
                sl.append(slice(ng - 1, ng + n + 1))
        sl = tuple(sl)
        err = rel_err(Fg, Fo, sl)
        assert np.all(err <= RTOL), f"dir {d}: flux rel err {err}"
        ct_o = np.maximum(cmax, cmin)[sl]
        assert np.max(np.abs(ctop[sl] - ct_o)) <= RTOL * np.max(np.abs(ct_o))


def run_steps(o, b, Po, Uo, nsteps, spec):
    dt = spec.dt_min
    worst = np.zeros(spec.nvar)
    flags_equal = True
    for _ in range(nsteps):
        pf_o, ff_o, dtn, mn_o = o.step(Po, Uo, dt)
        b.step(dt)
        mn_g = b.min_ndt()
        U = b.U.cpu().numpy()
        P = b.P.cpu().numpy()
        sl = spec.interior
        worst = np.maximum(worst, rel_err(U, Uo))
        worst = np.maximum(worst, rel_err(P, Po))
        pf_g = b.pflag.cpu().numpy()[sl]
        ff_g = b.fflag.cpu().numpy()[sl]
        flags_equal &= np.array_equal(pf_g, pf_o[sl].astype(np.int32)) and np.array_equal(ff_g, ff_o[sl].astype(np.int32))
        assert abs(mn_g - mn_o) <= RTOL * abs(mn_o), (mn_g, mn_o)
        dt = dtn
    return worst, flags_equal


# The named workloads at their full sizes: the 64^3 fast mode (WENO5, LLF, flux-CT, RK2, CFL 0.9)
# compared after every one of 10 steps, and the 128^3 and 128^2 FM tori (MC, LLF, flux-CT, drift
# floors) over their first steps.
FULL = {
    "mhdmodes3d_weno5_64": lambda: mhdmodes_spec(64, 64, 64, recon="weno5"),
    "torus3d_mc_128": lambda: torus_spec(128, 128, 128),
    "torus2d_mc_128": lambda: torus_spec(128, 128, 1),
    # the reference's default inverter (inverter/type = kastaun, inverter.cpp:54)
    "torus3d_mc_kastaun": lambda: torus_spec(32, 24, 8, inverter="kastaun"),
    # first-order flux correction on (the production SANE deck's setting, pars/tori_3d/sane.par:80-81)
    "torus3d_mc_fofc": lambda: torus_spec(32, 24, 8, fofc=True),
    "torus3d_mc_128_fofc": lambda: torus_spec(128, 128, 128, fofc=True),
    # the FOFC options: speed-of-light LF speeds on replaced faces, geometric source in the guess
    "torus3d_mc_fofc_glf": lambda: dataclasses.replace(torus_spec(32, 24, 8, fofc=True), fofc_use_glf=True),
    "torus3d_mc_fofc_src": lambda: dataclasses.replace(torus_spec(32, 24, 8, fofc=True), fofc_use_source_term=True),
}
CASES.update(FULL)


@pytest.mark.parametrize("name,nsteps", [("mhdmodes3d_weno5", 10), ("mhdmodes2d_ppm_hlle", 10), ("torus3d_mc", 5),
                                         ("mhdmodes3d_weno5_64", 10), ("torus3d_mc_128", 3),
                                         ("torus2d_mc_128", 10), ("torus3d_mc_kastaun", 10),
                                         ("torus3d_mc_fofc", 10), ("torus3d_mc_128_fofc", 3),
                                         ("torus3d_mc_fofc_glf", 10), ("torus3d_mc_fofc_src", 10)])
def test_step_parity(oracle_mod, name, nsteps):
    spec = CASES[name]()
    o, b, Po, Uo = make_pair(oracle_mod, spec, initial(oracle_mod, name, spec))
    worst, flags_equal = run_steps(o, b, Po, Uo, nsteps, spec)
    bitwise = np.array_equal(b.U.cpu().numpy(), Uo) and np.array_equal(b.P.cpu().numpy(), Po)
    print(name, "worst per-variable relative error over steps:", worst, "bitwise equal:", bitwise)
    assert np.all(worst <= RTOL), worst
    assert flags_equal
    if name.startswith("mhdmodes"):
        # no library transcendental on this path: the FP64 build (no FMA contraction, reference
        # evaluation order) reproduces the oracle exactly
        assert bitwise


def test_second_order_convergence_fast_mode():
    """The 2D fast mode (k = (2 pi, 2 pi, 0)) advected for one period on the GPU: the L1 error of
    every perturbed variable falls with resolution at the rate the reference's tests/mhdmodes/check.py
    requires (slope in [-2.15, -1.94], [-2.3, -1.94] for u2/u3)."""
    from kharma_b200.block import Driver
    res = [16, 32, 64]
    L = []
    for n in res:
        spec = mhdmodes_spec(n, n, 1, recon="weno5")
        b = Block(spec)
        b.set_prims(problems.mhdmodes(spec, 3))
        d = Driver(b)
        tlim = problems.mhdmodes_period(3)
        while d.t < tlim:
            d.step(min(d.dt, tlim - d.t))
        ref = problems.mhdmodes_analytic(spec, 3)
        P = b.P.cpu().numpy()
        sl = spec.interior
        L.append([np.mean(np.abs(P[v][sl] - ref[v][sl])) for v in range(8)])
    L = np.array(L)
    amp = problems.MODES_DIR3[3]
    names = ["rho", "u", "u1", "u2", "u3", "B1", "B2", "B3"]
    for v, k in enumerate(("drho", "du", "du1", "du2", "du3", "dB1", "dB2", "dB3")):
        if amp[k] == 0:
            continue
        slope = np.polyfit(np.log(res), np.log(L[:, v]), 1)[0]
        lo = -2.3 if names[v] in ("u2", "u3") else -2.15
        assert lo <= slope <= -1.94, f"{names[v]}: slope {slope:.3f}; L1 {L[:, v]}"


def test_divb_stays_at_roundoff():
    spec = mhdmodes_spec(24, 24, 24)
    b = Block(spec)
    b.set_prims(problems.mhdmodes(spec, 3))
    d0 = b.max_divb()
    dt = spec.dt_min
    for _ in range(5):
        b.step(dt)
    assert b.max_divb() < 1e-12 + 10 * d0

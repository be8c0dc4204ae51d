"""The reference's known-answer tests run on the GPU path through the C ABI: the same convergence
bars the oracle meets (tests/test_oracle_pin.py), so the CUDA path is pinned to the reference's own
analytic solutions, not only to the oracle.

* Bondi steady state (tests/bondi/check.py:49-56): L1 drift of <rho>, <u>, <u^1> over t = 50 at 16-64
  zones per side, slopes in [-2.2, -1.85].
* EMHD linear mode (tests/emhdmodes/check.py:92-105): L1 error against the damped analytic wave at
  t = 2, slopes in [-3.3, -1.6]; WENO5 at 32-128 and linear MC at 64-256 as the reference runs them.
"""
import numpy as np
import pytest
import torch

from kharma_b200 import problems
from kharma_b200.block import Block, Driver
from kharma_b200.emhd import ImplicitSolver

from test_oracle_pin import (BONDI_RES, bondi_drift, bondi_pin_spec, bondi_slopes, emhd_errors, emhd_mode_setup,
                             emhd_next_dt, emhd_slopes)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("variant", [{}, {"inverter": "kastaun", "iter_max": 25, "err_tol": 1e-12},
                                     {"recon": "linear_mc"}], ids=["base", "kastaun", "linear_mc"])
def test_gpu_bondi_converges_like_reference(variant):
    L = []
    for n in BONDI_RES:
        spec = bondi_pin_spec(n, **variant)
        b = Block(spec)
        b.set_prims(problems.bondi(spec, b.geom))
        P0 = b.P.cpu().numpy()
        d = Driver(b)
        while d.t < 50.0:
            d.step(min(d.dt, 50.0 - d.t))
        L.append(bondi_drift(b.P.cpu().numpy(), P0, spec))
    for name, p in zip(("rho", "u", "u1"), bondi_slopes(L)):
        assert -2.2 <= p <= -1.85, f"{name}: slope {p:.3f}; L1 {np.array(L)}"


@pytest.mark.parametrize("recon,res", [("weno5", [32, 64, 128]), ("linear_mc", [64, 128, 256])])
def test_gpu_emhd_mode_converges_like_reference(recon, res):
    L = []
    for n in res:
        spec, emhd, imp = emhd_mode_setup(n, recon)
        b = Block(spec)
        sol = ImplicitSolver(b, emhd, imp)
        P = torch.tensor(problems.emhdmodes(spec), dtype=torch.float64, device="cuda")
        U = sol.ptou(P)
        sn, sf = sol.scalar_field(), sol.scalar_field()
        t, dt = 0.0, spec.dt_min
        while t < 2.0:
            dt = min(dt, 2.0 - t)
            sol.imex_step(P, U, dt, sn, sf)
            t += dt
            dt = emhd_next_dt(spec, b.min_ndt(), dt)
        L.append(emhd_errors(P.cpu().numpy(), spec, t))
    names = ["rho", "u", "u1", "u2", "u3", "B1", "B2", "B3", "q", "dP"]
    for v, p in emhd_slopes(L, res).items():
        assert -3.3 <= p <= -1.6, f"{recon} {names[v]}: slope {p:.3f}; L1 {np.array(L)[:, v]}"

"""The further reconstructions of flux/reconstruction.hpp (linear_vl, weno5_linear, ppmx, mp5;
donor_cell_c is donor_cell), WENO5 lowered to linear MC near the X1 block edges or the poles
(flux/low_order_edges, low_order_poles) and the floor fallback (flux/reconstruction_fallback),
against the oracle: face fluxes and 10 steps (3 on the torus), bitwise where no library
transcendental is on the path (the Cartesian modes), else to 1e-12 with identical flags."""
import dataclasses

import numpy as np
import pytest
import torch

from kharma_b200 import problems
from kharma_b200.block import Block
from kharma_b200.spec import mhdmodes_spec, torus_spec

from test_gpu_parity import RTOL, make_pair, rel_err, run_steps

pytestmark = pytest.mark.gpu

MODES = {
    "linear_vl": lambda: mhdmodes_spec(16, 16, 16, recon="linear_vl"),
    "weno5_linear": lambda: mhdmodes_spec(16, 16, 16, recon="weno5_linear"),
    "ppmx": lambda: mhdmodes_spec(16, 16, 16, recon="ppmx"),
    "mp5": lambda: mhdmodes_spec(16, 16, 16, recon="mp5"),
    "donor_cell_c": lambda: mhdmodes_spec(16, 16, 16, recon="donor_cell_c"),
    "weno5_low_order_edges": lambda: dataclasses.replace(mhdmodes_spec(16, 16, 16, recon="weno5"), low_order_edges=True),
    "mp5_fp32_flux": lambda: mhdmodes_spec(16, 16, 16, recon="mp5", precision="fp32_flux"),
}
TORI = {
    "torus_weno5_low_order_poles": lambda: dataclasses.replace(torus_spec(32, 24, 8, recon="weno5"), low_order_poles=True),
    "torus_weno5_fallback": lambda: dataclasses.replace(torus_spec(32, 24, 8, recon="weno5"), recon_fallback=True),
    "torus_mp5_recon_floors": lambda: dataclasses.replace(torus_spec(32, 24, 8, recon="mp5"), recon_floors=True),
    "torus_weno5_linear_fallback": lambda: dataclasses.replace(torus_spec(32, 24, 8, recon="weno5_linear"),
                                                               recon_fallback=True),
}


@pytest.mark.parametrize("name", list(MODES))
def test_mode_steps(oracle_mod, name):
    spec = MODES[name]()
    P0 = problems.mhdmodes(spec, 3, amp=1e-2)
    o, b, Po, Uo = make_pair(oracle_mod, spec, P0)
    if spec.precision == "fp32_flux":
        # the FP32-flux form against the FP64 oracle: the density stays within the form's bar
        ref = Block(dataclasses.replace(spec, precision="fp64"), geometry=o.geometry())
        ref.set_prims(P0)
        for _ in range(10):
            b.step(spec.dt_min)
            ref.step(spec.dt_min)
        torch.cuda.synchronize()
        sl = spec.interior
        err = float((b.P[0][sl] - ref.P[0][sl]).abs().sum() / ref.P[0][sl].abs().sum())
        assert err < 1e-6
        return
    worst, flags_equal = run_steps(o, b, Po, Uo, 10, spec)
    bitwise = np.array_equal(b.U.cpu().numpy(), Uo) and np.array_equal(b.P.cpu().numpy(), Po)
    print(name, "worst relative error:", worst.max(), "bitwise:", bitwise)
    assert bitwise
    assert flags_equal


@pytest.mark.parametrize("name", list(TORI))
def test_torus_steps(oracle_mod, name):
    spec = TORI[name]()
    o, b, Po, Uo = make_pair(oracle_mod, spec, problems.fm_torus(spec, oracle_mod.Oracle(spec).geometry(), seed=7))
    worst, flags_equal = run_steps(o, b, Po, Uo, 3, spec)
    print(name, "worst per-variable relative error:", worst)
    assert np.all(worst <= RTOL), worst
    assert flags_equal


def test_options_are_checked():
    from kharma_b200 import _lib
    with pytest.raises(_lib.KhbError, match="weno5"):
        Block(dataclasses.replace(mhdmodes_spec(16, 16, 1, recon="linear_mc"), low_order_edges=True))
    with pytest.raises(_lib.KhbError, match="high-order"):
        Block(dataclasses.replace(torus_spec(16, 16, 1, recon="linear_mc"), recon_fallback=True))

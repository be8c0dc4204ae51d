"""The FP32-flux form against the plain FP64 path, and launch-shape choices that must not change
results.

FP32-flux form: reconstruction, Riemann fluxes and EMF averaging in FP32, conserved update,
inversion and geometry in FP64.  Requirement: relative L1 density error <= 1e-5 after 100 steps
on the FM torus, both runs taking the same dt sequence.
"""
import numpy as np
import pytest
import torch

from kharma_b200 import problems
from kharma_b200.block import Block, Driver, build_geometry
from kharma_b200.spec import mhdmodes_spec, torus_spec

pytestmark = pytest.mark.gpu


def run(spec, geom, P0, dts, tuning=None):
    b = Block(spec, geometry=geom)
    for k, v in (tuning or {}).items():
        b.set_tuning(k, v)
    b.set_prims(P0)
    for dt in dts:
        b.step(dt)
    torch.cuda.synchronize()
    return b


def fp64_dts(spec, geom, P0, nsteps):
    b = Block(spec, geometry=geom)
    b.set_prims(P0)
    d = Driver(b)
    dts = []
    for _ in range(nsteps):
        dt, _ = d.step()
        dts.append(dt)
    return dts, b


def test_fp32_flux_density_error_torus():
    spec64 = torus_spec(64, 64, 64)
    geom = build_geometry(spec64)
    P0 = problems.fm_torus(spec64, geom, seed=11)
    dts, b64 = fp64_dts(spec64, geom, P0, 100)
    b32 = run(torus_spec(64, 64, 64, precision="fp32_flux"), geom, P0, dts)
    sl = spec64.interior
    r64 = b64.P[0][sl].double()
    r32 = b32.P[0][sl].double()
    err = float((r32 - r64).abs().sum() / r64.abs().sum())
    print("FP32-flux relative L1 density error after 100 steps:", err)
    assert err <= 1e-5


@pytest.mark.parametrize("spec_fn", [lambda: mhdmodes_spec(16, 16, 16), lambda: torus_spec(32, 24, 8)],
                         ids=["periodic", "torus"])
def test_zone_split_is_bitwise_neutral(spec_fn):
    spec = spec_fn()
    geom = build_geometry(spec)
    P0 = problems.fm_torus(spec, geom, seed=5) if spec.spherical else problems.mhdmodes(spec, 3)
    dts = [spec.dt_min * 2 ** k for k in range(4)]
    a = run(spec, geom, P0, dts, {"zone_split": 0})
    for split in (1, 2):
        b = run(spec, geom, P0, dts, {"zone_split": split})
        assert torch.equal(a.P, b.P) and torch.equal(a.U, b.U)
        assert torch.equal(a.pflag, b.pflag) and torch.equal(a.fflag, b.fflag)

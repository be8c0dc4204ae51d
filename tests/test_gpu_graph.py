"""Device-resident timestep and the graph-replayed step against the host-driven step (GPU).

khb_step_graph replays one RK2 step captured with the device timestep: the kernels read dt from
device memory and the next dt is set there by the reference's schedule (EstimateTimestep +
SetGlobalTimeStep).  It must reproduce the host-driven Driver (khb_step + khb_get_min_ndt + the
schedule on the host) bit for bit: same dt sequence, same state and flags, with and without FOFC.
"""
import pytest
import torch

from kharma_b200 import problems
from kharma_b200.block import Block, DeviceDriver, Driver, build_geometry
from kharma_b200.spec import mhdmodes_spec, torus_spec

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("make", [lambda: torus_spec(32, 24, 8), lambda: torus_spec(32, 24, 8, fofc=True),
                                  lambda: torus_spec(32, 24, 8, precision="fp32_flux"),
                                  lambda: mhdmodes_spec(16, 16, 16)],
                         ids=["torus", "torus_fofc", "torus_fp32", "mhdmodes"])
def test_graph_step_equals_host_driven_step(make):
    spec = make()
    geom = build_geometry(spec)
    P0 = problems.fm_torus(spec, geom, seed=3) if spec.spherical else problems.mhdmodes(spec, 3)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        a = Block(spec, geometry=geom)
        a.set_prims(P0)
        da = Driver(a)
        dts = [da.step()[0] for _ in range(8)]
        b = Block(spec, geometry=geom)
        b.set_prims(P0)
        db = DeviceDriver(b, graph=True)
        for _ in range(8):
            db.step()
        dt_next, t, last = db.timestep()
    stream.synchronize()
    assert last == dts[-1] and dt_next == da.dt and t == sum(dts) or abs(t - sum(dts)) <= 1e-15 * t
    assert torch.equal(a.P, b.P) and torch.equal(a.U, b.U)
    assert torch.equal(a.pflag, b.pflag) and torch.equal(a.fflag, b.fflag)


def test_step_host_matches_device_resident_steps():
    """khb_step_host (primitives in, U = U(P), graph step, primitives out) leaves the same state as
    the device-resident graph step, bit for bit: U = U(P) holds exactly after every step."""
    import dataclasses
    from kharma_b200 import problems
    from kharma_b200.block import Block, DeviceDriver, build_geometry
    from kharma_b200.spec import torus_spec
    spec = torus_spec(32, 24, 8)
    geom = build_geometry(spec)
    P0 = problems.fm_torus(spec, geom, seed=5)
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        a = Block(spec, geometry=geom); a.set_prims(P0)
        b = Block(spec, geometry=geom); b.set_prims(P0)
        da, db = DeviceDriver(a), DeviceDriver(b)
        hP = torch.empty(b.P.shape, dtype=torch.float64, pin_memory=True)
        hP.copy_(b.P)
        for _ in range(5):
            da.step()
            db.step_host(hP)
        torch.cuda.synchronize()
        assert torch.equal(a.P.cpu(), hP)
        assert torch.equal(a.U, b.U)
        # and the device state b holds satisfies U = U(P) exactly
        U0 = b.U.clone()
        b.ptou()
        torch.cuda.synchronize()
        assert torch.equal(U0, b.U)


def test_step_host_interior_matches_device_resident_steps():
    """khb_step_host_interior (interior primitives in, ghost zones rebuilt on the device, graph step,
    interior primitives out) leaves the device-resident graph step's state, bit for bit, ghost zones
    included; blocks with exchange faces are refused."""
    import dataclasses
    from kharma_b200 import _lib, problems
    from kharma_b200.block import Block, DeviceDriver, build_geometry
    from kharma_b200.spec import mhdmodes_spec, torus_spec
    spec = torus_spec(32, 24, 8)
    geom = build_geometry(spec)
    P0 = problems.fm_torus(spec, geom, seed=5)
    sl = (slice(None),) + spec.interior
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        a = Block(spec, geometry=geom); a.set_prims(P0)
        b = Block(spec, geometry=geom); b.set_prims(P0)
        da, db = DeviceDriver(a), DeviceDriver(b)
        hP = torch.empty(b.P[sl].shape, dtype=torch.float64, pin_memory=True)
        hP.copy_(b.P[sl])
        for _ in range(5):
            da.step()
            db.step_host_interior(hP)
        torch.cuda.synchronize()
        assert torch.equal(a.P[sl].cpu(), hP)
        assert torch.equal(a.P, b.P) and torch.equal(a.U, b.U)
        ex = Block(dataclasses.replace(mhdmodes_spec(16, 16, 1), bc=("exchange",) * 4 + ("periodic",) * 2))
        ex.set_prims(problems.mhdmodes(ex.spec, 3))
        dex = DeviceDriver(ex)
        h = torch.empty(ex.P[(slice(None),) + ex.spec.interior].shape, dtype=torch.float64, pin_memory=True)
        with pytest.raises(_lib.KhbError, match="exchange"):
            dex.step_host_interior(h)

"""x3 slab decomposition on one GPU: the block split into 2 and 4 slabs (all in this process,
exchanged by copies) steps bit for bit like the undivided periodic block, including the global
timestep."""
import numpy as np
import pytest
import torch

from kharma_b200 import problems, slabs
from kharma_b200.block import Block, Driver, build_geometry
from kharma_b200.spec import torus_spec

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nslabs", [2, 4])
def test_slabs_match_single_block(nslabs):
    spec = torus_spec(32, 24, 16)
    geom = build_geometry(spec)
    P0 = problems.fm_torus(spec, geom, seed=3)
    single = Block(spec, geometry=geom)
    single.set_prims(P0)
    ex = slabs.LocalExchange()
    parts = [slabs.SlabBlock(spec, nslabs, r, ex, geometry=geom) for r in range(nslabs)]
    ng, n = spec.ng, spec.nx3 // nslabs
    slabs.set_prims(parts, ex, [P0[:, r * n:r * n + n + 2 * ng] for r in range(nslabs)])

    def check(tag):
        torch.cuda.synchronize()
        for r, s in enumerate(parts):
            k0 = r * n
            for name in ("P", "U"):
                a = getattr(s.block, name)
                b = getattr(single, name)[:, k0:k0 + n + 2 * ng]
                assert torch.equal(a, b), f"{tag}: slab {r} {name} differs"

    check("initial state")
    drv = Driver(single)
    dt = spec.dt_min
    for step in range(4):
        dts, mn = drv.step(dt)
        slabs.step(parts, ex, dt)
        check(f"step {step}")
        assert slabs.min_ndt(parts) == mn
        dt = drv.dt

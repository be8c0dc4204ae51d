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


@pytest.mark.parametrize("overlap", [False, True])
@pytest.mark.parametrize("nslabs", [2, 4])
def test_slabs_match_single_block(nslabs, overlap):
    """overlap: the second exchange of each stage is completed by the next stage after the faces that
    read no ghost plane, across steps too (finished only every other step; the interiors are compared
    after every step, the ghost planes after each finish)."""
    spec = torus_spec(32, 24, 16)
    geom = build_geometry(spec)
    P0 = problems.fm_torus(spec, geom, seed=3)
    single = Block(spec, geometry=geom)
    single.set_prims(P0)
    ex = slabs.LocalExchange()
    parts = [slabs.SlabBlock(spec, nslabs, r, ex, geometry=geom) for r in range(nslabs)]
    ng, n = spec.ng, spec.nx3 // nslabs
    slabs.set_prims(parts, ex, [P0[:, r * n:r * n + n + 2 * ng] for r in range(nslabs)])

    def check(tag, ghosts=True):
        torch.cuda.synchronize()
        for r, s in enumerate(parts):
            k0 = r * n
            for name in ("P", "U"):
                a = getattr(s.block, name)
                b = getattr(single, name)[:, k0:k0 + n + 2 * ng]
                if not ghosts:
                    a, b = a[:, ng:ng + n], b[:, ng:ng + n]
                assert torch.equal(a, b), f"{tag}: slab {r} {name} differs"

    check("initial state")
    drv = Driver(single)
    dt = spec.dt_min
    pending = None
    for step in range(4):
        dts, mn = drv.step(dt)
        pending = slabs.step(parts, ex, dt, overlap=overlap, pending=pending)
        if step % 2:
            ex.finish(pending)
            pending = None
        check(f"step {step}", ghosts=pending is None)
        assert slabs.min_ndt(parts) == mn
        dt = drv.dt

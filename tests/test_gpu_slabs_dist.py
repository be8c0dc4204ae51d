"""The x3 slab decomposition across processes: two ranks (torch.distributed, gloo, the halo planes
staged through host memory) each step their slab of the torus on the GPU through the C ABI; after
each of 5 RK2 steps (with the global MIN of the timestep) every slab, ghost planes included, is bit
for bit the matching part of the undivided block stepped alone.  Both ranks share this run's one
GPU; they exchange on the host between kernel launches, so no kernel waits on another rank's."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

NSTEPS = 5
SHAPE = (32, 24, 16)


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _worker(rank, nranks, port, outdir, overlap):
    from datetime import timedelta

    import torch.distributed as dist
    from kharma_b200 import problems, slabs
    from kharma_b200.block import build_geometry
    from kharma_b200.spec import torus_spec
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=nranks, timeout=timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        spec = torus_spec(*SHAPE)
        geom = build_geometry(spec)
        P0 = problems.fm_torus(spec, geom, seed=3)
        ex = slabs.DistExchange(host_staged=True)
        sb = slabs.SlabBlock(spec, nranks, rank, ex, geometry=geom)
        ng, n = spec.ng, spec.nx3 // nranks
        slabs.set_prims([sb], ex, [P0[:, rank * n:rank * n + n + 2 * ng]], local=False)
        drv = slabs.SlabDriver([sb], ex, local=False, overlap=overlap)
        out = {}
        for step in range(NSTEPS):
            dt, mn = drv.step()
            drv.sync()
            torch.cuda.synchronize()
            out[f"P{step}"] = sb.block.P.cpu().numpy()
            out[f"U{step}"] = sb.block.U.cpu().numpy()
            out[f"dt{step}"] = np.array([dt, mn])
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), **out)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("overlap", [False, True])
@pytest.mark.parametrize("nranks", [2])
def test_distributed_slabs_match_single_block(nranks, overlap):
    """overlap: each stage's second exchange completes only after the next stage's faces that read no
    ghost plane have been launched."""
    from kharma_b200 import problems
    from kharma_b200.block import Block, Driver, build_geometry
    from kharma_b200.spec import torus_spec
    with tempfile.TemporaryDirectory() as outdir:
        ctx = mp.get_context("spawn")
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, nranks, port, outdir, overlap)) for r in range(nranks)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=300)
            if p.is_alive():
                p.kill()
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        ranks = [dict(np.load(os.path.join(outdir, f"rank{r}.npz"))) for r in range(nranks)]

    spec = torus_spec(*SHAPE)
    geom = build_geometry(spec)
    single = Block(spec, geometry=geom)
    single.set_prims(problems.fm_torus(spec, geom, seed=3))
    drv = Driver(single)
    ng, n = spec.ng, spec.nx3 // nranks
    for step in range(NSTEPS):
        dt, mn = drv.step()
        torch.cuda.synchronize()
        P, U = single.P.cpu().numpy(), single.U.cpu().numpy()
        for r, out in enumerate(ranks):
            k0 = r * n
            assert np.array_equal(out[f"P{step}"], P[:, k0:k0 + n + 2 * ng]), f"step {step}: rank {r} P"
            assert np.array_equal(out[f"U{step}"], U[:, k0:k0 + n + 2 * ng]), f"step {step}: rank {r} U"
            assert out[f"dt{step}"][0] == dt and out[f"dt{step}"][1] == mn, f"step {step}: rank {r} timestep"

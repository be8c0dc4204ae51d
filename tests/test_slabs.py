"""x3 slab decomposition on CPU: slab specs, and the halo exchange of the distributed exchanger
(gloo, two and three ranks as processes) against the single-process plan.  No GPU."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from kharma_b200.slabs import DistExchange, LocalExchange, plane_ranges, slab_spec
from kharma_b200.spec import torus_spec


def test_slab_specs_tile_the_block():
    spec = torus_spec(32, 24, 16)
    slabs = [slab_spec(spec, 4, r) for r in range(4)]
    assert all(s.nx3 == 4 and s.bc[4:] == ("exchange", "exchange") and s.bc[:4] == spec.bc[:4] for s in slabs)
    dx3 = (spec.x3max - spec.x3min) / spec.nx3
    for r, s in enumerate(slabs):
        assert s.x3min == pytest.approx(spec.x3min + 4 * r * dx3)
        assert (s.x3max - s.x3min) / s.nx3 == pytest.approx(dx3)
    with pytest.raises(ValueError):
        slab_spec(spec, 8, 0)          # 2 planes per slab < 4 ghosts


def global_fields(spec, nv=3):
    """Field values that identify (var, global k, j, i)."""
    n3, n2, n1 = spec.shape
    k = np.arange(n3)[:, None, None]
    j = np.arange(n2)[None, :, None]
    i = np.arange(n1)[None, None, :]
    return np.stack([1000000.0 * v + 10000 * k + 100 * j + i for v in range(nv)])


def slab_arrays(gspec, nranks, rank):
    s = slab_spec(gspec, nranks, rank)
    G = global_fields(gspec)
    ng, n = gspec.ng, s.nx3
    k0 = ng + rank * n
    P = torch.tensor(G[:, k0 - ng:k0 + n + ng].copy())
    flag = torch.tensor((G[0, k0 - ng:k0 + n + ng] % 7).astype(np.int32))
    # poison the ghosts so that only the exchange can fill them
    P[:, :ng] = -1.0
    P[:, -ng:] = -1.0
    flag[:ng] = -1
    flag[-ng:] = -1
    return s, P, flag


def expected_after_exchange(gspec, nranks, rank, nplanes):
    s, P, flag = slab_arrays(gspec, nranks, rank)
    G = global_fields(gspec)
    ng, n, N = gspec.ng, s.nx3, gspec.nx3
    for g in range(nplanes):
        # low ghost plane ks-1-g holds global interior plane (k0-1-g) wrapped
        for kk, src in ((ng - 1 - g, rank * n - 1 - g), (ng + n + g, rank * n + n + g)):
            P[:, kk] = torch.tensor(G[:, ng + src % N])
            flag[kk] = torch.tensor((G[0, ng + src % N] % 7).astype(np.int32))
    return P, flag


@pytest.mark.parametrize("nranks", [1, 2, 3])
@pytest.mark.parametrize("nplanes", [1, 4])
def test_local_exchange(nranks, nplanes):
    gspec = torus_spec(16, 8, 12)
    arrs = [slab_arrays(gspec, nranks, r) for r in range(nranks)]
    LocalExchange().exchange([[P, f] for _, P, f in arrs], arrs[0][0], nplanes)
    ng = gspec.ng
    for r, (s, P, f) in enumerate(arrs):
        eP, ef = expected_after_exchange(gspec, nranks, r, nplanes)
        sl = slice(ng - nplanes, ng + s.nx3 + nplanes)
        assert torch.equal(P[:, sl], eP[:, sl]) and torch.equal(f[sl], ef[sl])


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _worker(rank, nranks, port, nplanes, out, split=False):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=nranks)
    try:
        gspec = torus_spec(16, 8, 12)
        s, P, f = slab_arrays(gspec, nranks, rank)
        ex = DistExchange()
        ok = True
        if split:
            # started, not finished: the ghost planes are untouched until finish()
            P0, f0 = P.clone(), f.clone()
            h = ex.start([P, f], s, nplanes)
            ok = torch.equal(P, P0) and torch.equal(f, f0)
            ex.finish(h)
        else:
            ex.exchange([P, f], s, nplanes)
        eP, ef = expected_after_exchange(gspec, nranks, rank, nplanes)
        ng = gspec.ng
        sl = slice(ng - nplanes, ng + s.nx3 + nplanes)
        out[rank] = int(ok and torch.equal(P[:, sl], eP[:, sl]) and torch.equal(f[sl], ef[sl]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("nranks,nplanes,split", [(2, 4, False), (3, 1, False), (2, 4, True), (3, 2, True)])
def test_distributed_exchange_gloo(nranks, nplanes, split):
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, nranks, port, nplanes, out, split)) for r in range(nranks)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert dict(out) == {r: 1 for r in range(nranks)}

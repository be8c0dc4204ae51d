"""Domain decomposition of one block into x3 slabs, one per rank, with halo exchange.

The metric is x3-independent and x3 is periodic on the torus, so every rank holds the full
(x1, x2) extent and a contiguous range of x3 planes; the geometry tables are the same on every
rank.  Per RK stage the ranks exchange, with their two x3 neighbours:
  1. after the zone pass: one plane of the fluid primitives and of pflag, which Inverter::FixUtoP
     reads across the slab face (the reference's first boundary sync, kharma_step.cpp:209-239);
  2. after the physical boundaries: ng planes of every primitive and conserved variable (the
     second sync, kharma_step.cpp:305-317, two_sync on by default at kharma_driver.cpp:77).
Each x3 plane range of one variable is contiguous in the [n3][n2][n1] layout, so the exchange sends
the field arrays' own slices: no packing.  The global timestep is the minimum over ranks of the
per-rank minimum, max divB the maximum (kharma_driver.cpp:439-460, b_flux_ct.cpp:609-618).

Two exchangers implement the same plan: LocalExchange runs all slabs in one process (one GPU, or
CPU tensors), DistExchange uses torch.distributed point-to-point operations (NCCL between GPUs,
gloo on CPU), one rank per slab.

With overlap (step(..., overlap=True), SlabDriver(overlap=True)) the second exchange is started, not
waited for: the next stage first computes the faces that read no x3 ghost plane (x1/x2 faces of the
interior planes, x3 faces at least ng planes inside; khb_get_flux_planes), then completes the
exchange (NCCL: the compute stream waits on the communication stream; gloo: the host waits while
those kernels run) and computes the rest.  Every face is computed once either way, so the
overlapped step equals the plain one bit for bit.
"""
import dataclasses

import torch

from .block import Block, Driver
from .spec import BlockSpec


def slab_spec(spec: BlockSpec, nranks: int, rank: int) -> BlockSpec:
    """The spec of rank's slab: nx3 / nranks planes, x3 range shifted, x3 faces exchanged."""
    if spec.nx3 % nranks or spec.nx3 // nranks < spec.ng:
        raise ValueError(f"nx3 = {spec.nx3} does not split into {nranks} slabs of at least {spec.ng} planes")
    if spec.bc[4] != "periodic":
        raise ValueError("slab decomposition needs a periodic x3 direction")
    n = spec.nx3 // nranks
    dx3 = (spec.x3max - spec.x3min) / spec.nx3
    bc = tuple(spec.bc[:4]) + ("exchange", "exchange")
    return dataclasses.replace(spec, nx3=n, x3min=spec.x3min + rank * n * dx3,
                               x3max=spec.x3min + (rank + 1) * n * dx3, bc=bc)


def plane_ranges(spec: BlockSpec, nplanes: int):
    """(send_lo, send_hi, recv_lo, recv_hi) x3 slices of a slab for an exchange of nplanes."""
    ks, ke = spec.ng, spec.ng + spec.nx3 - 1
    return (slice(ks, ks + nplanes), slice(ke - nplanes + 1, ke + 1),
            slice(ks - nplanes, ks), slice(ke + 1, ke + 1 + nplanes))


class LocalExchange:
    """All slabs in this process: copies between the slabs' arrays (periodic in x3)."""

    def exchange(self, per_slab, spec, nplanes):
        """per_slab[r] = list of this slab's (..., n3, n2, n1) arrays, same order on every slab."""
        self.finish(self.start(per_slab, spec, nplanes))

    def start(self, per_slab, spec, nplanes):
        """The sent planes are copied out now; the ghost planes are written by finish()."""
        n = len(per_slab)
        slo, shi, rlo, rhi = plane_ranges(spec, nplanes)
        moves = []
        for r in range(n):
            left, right = per_slab[(r - 1) % n], per_slab[(r + 1) % n]
            for a, al, ar in zip(per_slab[r], left, right):
                moves.append((a[..., rlo, :, :], al[..., shi, :, :].clone()))
                moves.append((a[..., rhi, :, :], ar[..., slo, :, :].clone()))
        return moves

    def finish(self, moves):
        for dst, src in moves or ():
            dst.copy_(src)


class DistExchange:
    """One slab per rank of the default process group; neighbours rank -/+ 1 (periodic).

    The planes of all arrays bound for one neighbour are packed (as bytes, whatever their types) into
    one buffer, so that an exchange is two sends and two receives however many variables it carries.
    host_staged: the packed buffers travel through host memory (a backend without device
    point-to-point support, such as gloo, with the slabs on GPUs); otherwise they are sent from where
    they are (NCCL between GPUs, or gloo with CPU tensors)."""

    def __init__(self, host_staged=False):
        import torch.distributed as dist
        self.dist = dist
        self.rank = dist.get_rank()
        self.world = dist.get_world_size()
        self.host_staged = host_staged

    def exchange(self, arrays, spec, nplanes):
        """arrays: this rank's list of (n3, n2, n1) (or (nv, n3, n2, n1)) arrays."""
        self.finish(self.start(arrays, spec, nplanes))

    def start(self, arrays, spec, nplanes):
        """Pack and post the sends and receives; the ghost planes are written by finish()."""
        slo, shi, rlo, rhi = plane_ranges(spec, nplanes)
        if self.world == 1:
            return ("local", LocalExchange().start([arrays], spec, nplanes))
        dist = self.dist
        left, right = (self.rank - 1) % self.world, (self.rank + 1) % self.world
        views = []
        for a in arrays:
            views += [a[v] for v in range(a.shape[0])] if a.dim() == 4 else [a]
        # each variable's plane range is contiguous: pack them byte-wise, one buffer per neighbour
        as_bytes = lambda t: t.reshape(-1).view(torch.uint8)
        send_lo = torch.cat([as_bytes(a[slo]) for a in views])
        send_hi = torch.cat([as_bytes(a[shi]) for a in views])
        stage = self.host_staged and send_lo.is_cuda
        if stage:
            torch.cuda.current_stream().synchronize()
            send_lo, send_hi = send_lo.cpu(), send_hi.cpu()
        recv_hi, recv_lo = torch.empty_like(send_lo), torch.empty_like(send_hi)
        # Per peer the k-th send matches the k-th receive: send (low planes -> left, high planes ->
        # right) and receive (high ghosts <- right, low ghosts <- left) in this order, so that with
        # two ranks (left == right) the low planes still land in the peer's high ghosts.
        ops = [dist.P2POp(dist.isend, send_lo, left), dist.P2POp(dist.isend, send_hi, right),
               dist.P2POp(dist.irecv, recv_hi, right), dist.P2POp(dist.irecv, recv_lo, left)]
        reqs = dist.batch_isend_irecv(ops)
        return ("dist", (reqs, (send_lo, send_hi), recv_hi, recv_lo, stage, views, rhi, rlo))

    def finish(self, handle):
        if handle is None:
            return
        kind, h = handle
        if kind == "local":
            LocalExchange().finish(h)
            return
        reqs, _sends, recv_hi, recv_lo, stage, views, rhi, rlo = h
        for req in reqs:
            req.wait()
        if stage:
            dev = views[0].device
            recv_hi, recv_lo = recv_hi.to(dev), recv_lo.to(dev)
        as_bytes = lambda t: t.reshape(-1).view(torch.uint8)
        off = 0
        for a in views:
            hi, lo = a[rhi], a[rlo]
            n = hi.numel() * hi.element_size()
            as_bytes(hi).copy_(recv_hi[off:off + n])
            as_bytes(lo).copy_(recv_lo[off:off + n])
            off += n


class SlabBlock:
    """One rank's slab of a decomposed block, stepped stage by stage through the C ABI with the
    exchanges above between the pieces of each stage."""

    def __init__(self, spec: BlockSpec, nranks: int, rank: int, exchanger, geometry=None):
        self.global_spec = spec
        self.spec = slab_spec(spec, nranks, rank)
        self.block = Block(self.spec, geometry=geometry)
        self.ex = exchanger
        self.P1 = torch.zeros_like(self.block.P)
        self.U1 = torch.zeros_like(self.block.U)

    # The pieces of one stage (khb_stage = fluxes + fix_flux + zone pass + fixups + boundaries)
    def stage_fluxes(self, Pin, part):
        """The faces of a stage in two parts: 'inner' reads no x3 ghost plane (x1/x2 faces of planes
        ks..ke, x3 faces ks+ng..ke+1-ng), 'outer' the rest."""
        from .block import Fields
        from . import _lib
        b = self.block
        Pi = Fields(Pin)
        ng = self.spec.ng
        ks, ke = ng, ng + self.spec.nx3 - 1
        for d in range(1, self.spec.ndim + 1):
            if d < 3:
                inner = [(ks, ke)]
                outer = [(ks - 1, ks - 1), (ke + 1, ke + 1)]
            else:
                inner = [(ks + ng, ke + 1 - ng)]
                outer = [(ks, min(ks + ng - 1, ke + 1)), (max(ke + 2 - ng, ks + ng), ke + 1)]
            for lo, hi in (inner if part == "inner" else outer):
                if lo <= hi:
                    _lib.check(b.lib.khb_get_flux_planes(b.ctx, d, Pi.ref, lo, hi, b.stream), "khb_get_flux_planes")

    def stage_compute(self, stage, dt, Pin, Uin, Pout, Uout, fluxes=True):
        from .block import Fields
        import ctypes as C
        from . import _lib
        b = self.block
        lib, ctx, st = b.lib, b.ctx, b.stream
        Pi, Ui, Po, Uo, U0 = Fields(Pin), Fields(Uin), Fields(Pout), Fields(Uout), Fields(b.U)
        if fluxes:
            for d in range(1, self.spec.ndim + 1):
                _lib.check(lib.khb_get_flux(ctx, d, Pi.ref, st), "khb_get_flux")
        _lib.check(lib.khb_fix_flux(ctx, st), "khb_fix_flux")
        pf, ff = C.c_void_p(b.pflag.data_ptr()), C.c_void_p(b.fflag.data_ptr())
        _lib.check(lib.khb_zone_pass(ctx, stage, dt, Pi.ref, Ui.ref, U0.ref, Po.ref, Uo.ref, pf, ff, st),
                   "khb_zone_pass")
        return Po, Uo

    def stage_fix(self, Pout, Uout):
        from .block import Fields
        import ctypes as C
        from . import _lib
        b = self.block
        _lib.check(b.lib.khb_fix_utop_list(b.ctx, Fields(Pout).ref, Fields(Uout).ref,
                                           C.c_void_p(b.pflag.data_ptr()), b.stream), "khb_fix_utop_list")
        _lib.check(b.lib.khb_boundaries(b.ctx, Fields(Pout).ref, Fields(Uout).ref, b.stream), "khb_boundaries")


def set_prims(slabs, exchanger, P_slabs, local=True):
    """Initial state on every slab: U = U(P), boundaries with the exchange, U = U(P) again (the
    sequence of Block.set_prims)."""
    for s, P in zip(slabs, P_slabs):
        s.block.P.copy_(torch.as_tensor(P, dtype=torch.float64))
        s.block.ptou()
    for s in slabs:
        s.block.boundaries()
    _exchange_full(slabs, exchanger, local)
    for s in slabs:
        s.block.ptou()


def _exchange_full(slabs, exchanger, local, P=None, U=None):
    spec = slabs[0].spec
    if local:
        exchanger.exchange([[(s.block.P if P is None else P[i]), (s.block.U if U is None else U[i])]
                            for i, s in enumerate(slabs)], spec, spec.ng)
    else:
        s = slabs[0]
        exchanger.exchange([s.block.P if P is None else P[0], s.block.U if U is None else U[0]], spec, spec.ng)


def _exchange_fix(slabs, exchanger, local, P):
    spec = slabs[0].spec
    if local:
        exchanger.exchange([[P[i][0:5], s.block.pflag] for i, s in enumerate(slabs)], spec, 1)
    else:
        exchanger.exchange([P[0][0:5], slabs[0].block.pflag], spec, 1)


def _start_full(slabs, exchanger, local, P, U):
    spec = slabs[0].spec
    if local:
        return exchanger.start([[P[i], U[i]] for i in range(len(slabs))], spec, spec.ng)
    return exchanger.start([P[0], U[0]], spec, spec.ng)


def step(slabs, exchanger, dt, local=True, overlap=False, pending=None):
    """One RK2 step of every slab in this process (all slabs with LocalExchange, this rank's one
    with DistExchange).  overlap: the second exchange of each stage is left in flight and completed
    by the next stage after the faces that do not need it; pending is the one the previous step left
    (None: complete), and the return value the one this step leaves (None without overlap)."""
    for stage in (1, 2):
        Pin = [s.block.P if stage == 1 else s.P1 for s in slabs]
        Uin = [s.block.U if stage == 1 else s.U1 for s in slabs]
        Pout = [s.P1 if stage == 1 else s.block.P for s in slabs]
        Uout = [s.U1 if stage == 1 else s.block.U for s in slabs]
        if overlap:
            for i, s in enumerate(slabs):
                s.stage_fluxes(Pin[i], "inner")
            exchanger.finish(pending)
            for i, s in enumerate(slabs):
                s.stage_fluxes(Pin[i], "outer")
        for i, s in enumerate(slabs):
            s.stage_compute(stage, dt, Pin[i], Uin[i], Pout[i], Uout[i], fluxes=not overlap)
        _exchange_fix(slabs, exchanger, local, Pout)
        for i, s in enumerate(slabs):
            s.stage_fix(Pout[i], Uout[i])
        if overlap:
            pending = _start_full(slabs, exchanger, local, Pout, Uout)
        else:
            _exchange_full(slabs, exchanger, local, Pout, Uout)
    return pending


def min_ndt(slabs, local=True):
    """Global minimum zone timestep of the last stage 2 (host value)."""
    m = min(s.block.min_ndt() for s in slabs)
    if not local:
        import torch.distributed as dist
        t = torch.tensor([m], dtype=torch.float64,
                         device="cuda" if dist.get_backend() == "nccl" else "cpu")
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
        m = float(t.item())
    return m


class SlabDriver:
    """The reference's timestep schedule (Driver) over decomposed slabs: the per-rank minimum zone
    timestep is reduced over all slabs (and ranks) before the next dt is chosen."""

    def __init__(self, slabs, exchanger, local=True, dt_start=None, overlap=False):
        self.slabs = slabs
        self.ex = exchanger
        self.local = local
        self.overlap = overlap
        self.pending = None
        spec = slabs[0].spec
        self.dt = spec.dt_min if dt_start is None else dt_start
        self.nstep = 0

    def sync(self):
        """Complete the exchange the last step left in flight (the state's ghost planes)."""
        self.ex.finish(self.pending)
        self.pending = None

    def step(self, dt=None):
        dt = self.dt if dt is None else dt
        self.pending = step(self.slabs, self.ex, dt, self.local, self.overlap, self.pending)
        mn = min_ndt(self.slabs, self.local)
        s = self.slabs[0].spec
        ndt = min(max(mn * s.cfl, s.dt_min), s.max_dt_increase * dt)
        self.dt = min(2.0 * dt, ndt)
        self.nstep += 1
        return dt, mn

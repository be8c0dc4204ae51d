"""Static mesh refinement (SMR): a multi-level block mesh over a domain of native coordinates, stepped as
one batch with ghost-zone exchange and flux correction between blocks (khb_batch_set_mesh).

Parthenon owns mesh refinement in the reference (KHARMA only enables it, kharma.cpp:381-382, and
tasks the flux-correction messages, kharma_step.cpp:157-195); its cell-centred operators are
restated here as the algorithms it documents:
  * same-level neighbours: ghost zones are copies of the neighbour's zones;
  * a fine block next to a coarse one: its ghost zones are prolongated from the coarse zones, value
    plus a minmod-limited slope per active direction times +-1/4 of the coarse width
    (ProlongateCellMinMod on a uniform grid);
  * a coarse block next to fine ones: its ghost zones are the average of the 2^ndim fine zones they
    cover (RestrictCellAverage on a uniform grid);
  * flux correction: a coarse face on a fine-coarse boundary takes the average of the 2^(ndim-1)
    fine fluxes through it before the update, so the mesh conserves what the uniform scheme does.
Ghost zones are filled from primitives (then U = U(P) there), as KHARMA's simple and imex drivers
exchange them (sync_prims, kharma_driver.cpp:109-110), or, for blocks of the kharma driver, from
the updated conserved variables with the primitives as the inversion's seeds, the ghost zones then
inverted, floored and given U = U(P) like the interior (kharma_step.cpp:209-236); every block has the
same zone count,
as Parthenon requires, and the fine blocks cover whole coarse blocks (2:1 in each active direction,
neighbouring blocks at most one level apart).  Scope (any coordinates: the operators act on the
uniform native grid): hydro blocks (5 variables) through the batch,
MHD blocks with B_CT through kharma_b200/ctmesh.py; any number of levels; each direction periodic, or
outflow/reflecting on the domain faces (a block on such a face keeps it; ghost entries stop at it and
the block's boundary condition fills what lies beyond, after the exchange; refined blocks keep a
coarse block between them and a physical domain face, since prolongation near it would read
boundary values of the previous stage).

`SMRMesh.tables()` gives the device tables khb_batch_set_mesh takes:
  ghost entries (int32 x 6): dst block, dst zone, op (0 copy, 1 restrict, 2 prolong), src block,
    src zone (copy: the zone; restrict: the fine zone of lowest index; prolong: the coarse zone),
    aux (prolong: bit d set when the fine zone lies on the + side of the coarse centre along d+1,
    and the prolongation phase, the destination level less one, in bits 8 and up);
    copies and restrictions first, then the prolongations level by level (each reads coarse ghost
    zones that the copies, the restrictions or the previous level's prolongations filled);
  flux entries (int32 x 6): coarse block, direction, coarse face (zone index of the zone above it),
    fine block, fine face of lowest index, 0.
"""
import dataclasses
import math

import numpy as np

from .spec import BlockSpec

OP_COPY, OP_RESTRICT, OP_PROLONG = 0, 1, 2


@dataclasses.dataclass
class MeshBlock:
    level: int
    loc: tuple          # logical location (l1, l2, l3) at its level
    spec: BlockSpec


class SMRMesh:
    """Root grid of nb = (nb1, nb2, nb3) blocks of nx = (nx1, nx2, nx3) zones over `base`'s domain
    (a BlockSpec supplying the physics options, the coordinates and the domain extent in native
    coordinates: hydro blocks, or MHD blocks with B_CT, in any coordinate system.
    Parthenon's operators act on the uniform grid of native coordinates, so the tables are the same
    in every coordinate system; each block carries its own metric); a block
    named in `refine` is replaced by its 2^ndim children one level up.  Entries are root locations
    (l1, l2, l3), or (level, (l1, l2, l3)) for a block of that level (its logical location at that
    level); refinements apply recursively, coarsest first."""

    def __init__(self, base: BlockSpec, nb, nx, refine=()):
        assert base.nvar == 5 or base.b_ct != "none", "SMR: hydro blocks, or MHD blocks with B_CT"
        self.base = base
        self.nb = tuple(nb)
        self.nx = tuple(nx)
        self.ndim = 1 + (nx[1] > 1) + (nx[2] > 1)
        assert all(self.nb[d] == 1 or nx[d] > 1 for d in range(3))
        assert all(nx[d] >= 8 for d in range(self.ndim)), "SMR: at least 8 zones per active direction"
        self.ng = base.ng
        # directions whose domain faces are physical (outflow or reflecting): blocks on those faces
        # keep them, and no ghost entry reaches past them
        self.periodic = tuple(d >= self.ndim or base.bc[2 * d] == "periodic" for d in range(3))
        for d in range(self.ndim):
            if not self.periodic[d]:
                ok = ("outflow", "reflecting") + (("transmitting",) if d == 1 else ())
                assert base.bc[2 * d] in ok and base.bc[2 * d + 1] in ok, \
                    "SMR: domain faces periodic, outflow or reflecting (x2: or transmitting)"
            else:
                assert base.bc[2 * d + 1] == "periodic", "SMR: a periodic direction is periodic on both faces"
        if "transmitting" in base.bc[2:4]:
            # the mirror zone lies half-way round in x3 inside the block: the blocks on the poles
            # (never refined) span all of a periodic x3
            assert self.ndim == 3 and self.periodic[2] and self.nb[2] == 1 and nx[2] % 2 == 0, \
                "SMR: transmitting x2 faces need 3D root blocks spanning all of a periodic x3 (even nx3)"
        lo = (base.x1min, base.x2min, base.x3min)
        hi = (base.x1max, base.x2max, base.x3max)
        self.lo, self.size = lo, tuple(hi[d] - lo[d] for d in range(3))
        ref = set()
        for r in refine:
            if len(r) == 2 and isinstance(r[1], (tuple, list)):
                ref.add((int(r[0]), tuple(int(x) for x in r[1])))
            else:
                ref.add((0, tuple(int(x) for x in r)))
        self.blocks = []

        def place(level, loc):
            if (level, loc) not in ref:
                self._add(level, loc)
                return
            for c3 in range(2 if self.ndim > 2 else 1):
                for c2 in range(2 if self.ndim > 1 else 1):
                    for c1 in range(2):
                        place(level + 1, (2 * loc[0] + c1, 2 * loc[1] + c2, 2 * loc[2] + c3))

        for l3 in range(self.nb[2]):
            for l2 in range(self.nb[1]):
                for l1 in range(self.nb[0]):
                    place(0, (l1, l2, l3))
        self.levels = 1 + max(b.level for b in self.blocks)
        self.index = {(b.level, b.loc): n for n, b in enumerate(self.blocks)}

    def _add(self, level, loc):
        f = 2 ** level
        ext = [self.size[d] / (self.nb[d] * (f if d < self.ndim else 1)) for d in range(3)]
        x0 = [self.lo[d] + loc[d] * ext[d] for d in range(3)]
        nl = [self.nb[d] * (f if d < self.ndim else 1) for d in range(3)]

        def face_bc(face):
            d, upper = face // 2, face % 2
            if d >= self.ndim or (self.periodic[d] and nl[d] == 1):
                return "periodic"                   # the block spans the periodic direction itself
            at_edge = (loc[d] == nl[d] - 1) if upper else (loc[d] == 0)
            return self.base.bc[face] if (at_edge and not self.periodic[d]) else "exchange"
        spec = dataclasses.replace(self.base, nx1=self.nx[0], nx2=self.nx[1], nx3=self.nx[2],
                                   x1min=x0[0], x1max=x0[0] + ext[0], x2min=x0[1], x2max=x0[1] + ext[1],
                                   x3min=x0[2], x3max=x0[2] + ext[2],
                                   bc=tuple(face_bc(face) for face in range(6)))
        # prolongation reads coarse zones up to one past the fine ghost zones: a coarse block between a
        # refined block and a physical domain face keeps those reads inside the domain
        assert level == 0 or all(x in ("exchange", "periodic") for x in spec.bc), \
            "SMR: refined blocks keep a coarse block between them and a physical domain face"
        self.blocks.append(MeshBlock(level, loc, spec))

    # ------------------------------------------------------------------ topology
    def _zones_at(self, level):
        """Zones along each direction of the whole domain at a level (inactive directions: 1)."""
        return [self.nb[d] * self.nx[d] * (2 ** level if d < self.ndim else 1) for d in range(3)]

    def _owners(self, level):
        """Block id per logical location at a level (-1 where that level has no block), (l3, l2, l1)."""
        nl = [self.nb[d] * (2 ** level if d < self.ndim else 1) for d in range(3)]
        own = np.full((nl[2], nl[1], nl[0]), -1, dtype=np.int64)
        for n, b in enumerate(self.blocks):
            if b.level == level:
                own[b.loc[2], b.loc[1], b.loc[0]] = n
        return own

    def _zone_index(self, k, j, i):
        n3, n2, n1 = self.blocks[0].spec.shape      # every block has the same shape
        return (k * n2 + j) * n1 + i

    def tables(self):
        ng, ndim, nx = self.ng, self.ndim, self.nx
        own = [self._owners(L) for L in range(self.levels)]
        ghost_a, flux = [], []
        ghost_b = [[] for _ in range(self.levels)]      # prolongations by destination level
        act = [d < ndim for d in range(3)]

        def local(src_loc, g):
            # local (k, j, i) of global zone(s) g in blocks at logical locations src_loc
            return tuple((g[d] - src_loc[d] * nx[d] + ng) if act[d] else np.zeros_like(g[d]) for d in (2, 1, 0))

        def owner(level, g):
            # block id owning global zones g at `level` (-1: none, or outside a physical domain face),
            # with the logical locations
            if level < 0 or level >= self.levels:
                return np.full(len(g[0]), -1, dtype=np.int64), None
            t = self._zones_at(level)
            ok = np.ones(len(g[0]), dtype=bool)
            for d in range(3):
                if act[d] and not self.periodic[d]:
                    ok &= (g[d] >= 0) & (g[d] < t[d])
            lo = [np.clip(g[d], 0, t[d] - 1) // nx[d] if act[d] else g[d] for d in range(3)]
            return np.where(ok, own[level][lo[2], lo[1], lo[0]], -1), lo

        def wrap(v, d, t):
            return v % t if self.periodic[d] else v

        for b, blk in enumerate(self.blocks):
            n3, n2, n1 = blk.spec.shape
            L = blk.level
            tot = self._zones_at(L)
            K, J, I = np.meshgrid(np.arange(n3), np.arange(n2), np.arange(n1), indexing="ij")
            inside = np.zeros((n3, n2, n1), dtype=bool)
            inside[blk.spec.interior] = True
            K, J, I = K[~inside], J[~inside], I[~inside]
            g = [wrap(blk.loc[0] * nx[0] + I - ng, 0, tot[0]),
                 wrap(blk.loc[1] * nx[1] + J - ng, 1, tot[1]) if act[1] else np.zeros_like(I),
                 wrap(blk.loc[2] * nx[2] + K - ng, 2, tot[2]) if act[2] else np.zeros_like(I)]
            # ghost zones past a physical domain face are the block's own boundary condition's
            keep = np.ones(len(I), dtype=bool)
            for d in range(3):
                if act[d] and not self.periodic[d]:
                    keep &= (g[d] >= 0) & (g[d] < tot[d])
            K, J, I = K[keep], J[keep], I[keep]
            g = [x[keep] for x in g]
            dst = (K * n2 + J) * n1 + I
            src, loc = owner(L, g)
            same = src >= 0
            if same.any():
                sl = [loc[d][same] for d in range(3)]
                gs = [g[d][same] for d in range(3)]
                k, j, i = local(sl, gs)
                z = self._zone_index(k, j, i)
                ghost_a.append(np.stack([np.full(same.sum(), b), dst[same], np.full(same.sum(), OP_COPY),
                                         src[same], z, np.zeros(same.sum(), dtype=np.int64)], axis=1))
            rest = ~same
            if not rest.any():
                continue
            gr = [g[d][rest] for d in range(3)]
            dr = dst[rest]
            # a coarser neighbour: prolongation from level L-1
            gc = [gr[d] // 2 if act[d] else gr[d] for d in range(3)]
            s0, lc = owner(L - 1, gc)
            # a finer neighbour: restriction from level L+1
            gf = [2 * gr[d] if act[d] else gr[d] for d in range(3)]
            s1, lf = owner(L + 1, gf)
            assert ((s0 >= 0) ^ (s1 >= 0)).all(), "mesh is not 2:1 balanced"
            pm, rm = s0 >= 0, s1 >= 0
            if pm.any():
                k, j, i = local([lc[d][pm] for d in range(3)], [gc[d][pm] for d in range(3)])
                z = self._zone_index(k, j, i)
                aux = sum((gr[d][pm] % 2) << d for d in range(ndim)) + ((L - 1) << 8)
                ghost_b[L].append(np.stack([np.full(pm.sum(), b), dr[pm], np.full(pm.sum(), OP_PROLONG),
                                            s0[pm], z, aux], axis=1))
            if rm.any():
                k, j, i = local([lf[d][rm] for d in range(3)], [gf[d][rm] for d in range(3)])
                z = self._zone_index(k, j, i)
                ghost_a.append(np.stack([np.full(rm.sum(), b), dr[rm], np.full(rm.sum(), OP_RESTRICT),
                                         s1[rm], z, np.zeros(rm.sum(), dtype=np.int64)], axis=1))
        # flux correction: faces of a block bordering finer blocks
        for b, blk in enumerate(self.blocks):
            L = blk.level
            if L + 1 >= self.levels:
                continue
            tot = self._zones_at(L)
            tot1 = self._zones_at(L + 1)
            for d in range(ndim):
                # tangential global indices (level L) of the face's zones
                rng = [np.arange(blk.loc[e] * nx[e], (blk.loc[e] + 1) * nx[e]) if act[e] else np.zeros(1, dtype=np.int64)
                       for e in range(3)]
                rng[d] = np.zeros(1, dtype=np.int64)
                T3, T2, T1 = np.meshgrid(rng[2], rng[1], rng[0], indexing="ij")
                t = [T1.ravel(), T2.ravel(), T3.ravel()]
                for side in (0, 1):
                    across = list(t)
                    across[d] = np.full_like(t[0], wrap(blk.loc[d] * nx[d] + (nx[d] if side else -1), d, tot[d]))
                    if not self.periodic[d] and not (0 <= across[d][0] < tot[d]):
                        continue                            # a physical domain face
                    if (owner(L, across)[0] >= 0).all():
                        continue                            # same level
                    if (owner(L - 1, [across[e] // 2 if act[e] else across[e] for e in range(3)])[0] >= 0).all():
                        continue                            # a coarser neighbour corrects this face
                    ci = list(t)
                    ci[d] = np.full_like(t[0], blk.loc[d] * nx[d] + (nx[d] if side else 0))
                    k, j, i = local([np.full_like(t[0], blk.loc[e]) for e in range(3)], ci)
                    cface = self._zone_index(k, j, i)
                    gfz = [2 * t[e] if act[e] else t[e] for e in range(3)]
                    gfz[d] = (2 * ci[d]) % tot1[d]
                    gown = list(gfz)
                    if not side:
                        gown[d] = (gfz[d] - 1) % tot1[d]
                    fb, lo = owner(L + 1, gown)
                    assert (fb >= 0).all(), "mesh is not 2:1 balanced"
                    fk, fj, fi = local(lo, gown)
                    if not side:
                        if d == 0:
                            fi = fi + 1
                        elif d == 1:
                            fj = fj + 1
                        else:
                            fk = fk + 1
                    fz = self._zone_index(fk, fj, fi)
                    flux.append(np.stack([np.full(len(fb), b), np.full(len(fb), d + 1), cface, fb, fz,
                                          np.zeros(len(fb), dtype=np.int64)], axis=1))
        cat = lambda parts: (np.concatenate(parts) if parts else np.zeros((0, 6), dtype=np.int64)).astype(np.int32)
        ga = cat(ghost_a)
        gb = cat([x for lev in ghost_b for x in lev])
        return np.concatenate([ga, gb]), len(ga), cat(flux)

    # ------------------------------------------------------------------ helpers
    def zone_volume(self, b):
        dx = self.blocks[b].spec.dx
        return dx[0] * dx[1] * dx[2]

    @property
    def zones(self):
        return len(self.blocks) * self.nx[0] * self.nx[1] * self.nx[2]


def smr_batch(mesh: SMRMesh, init, flux_correction=True, device="cuda", conserved=None):
    """A Batch of the mesh's blocks with initial primitives init(spec) -> (5, n3, n2, n1) per block,
    the mesh tables set and the ghost zones exchanged.  flux_correction=False leaves the coarse
    faces on fine-coarse boundaries uncorrected (for tests of conservation).  conserved: the
    kharma driver's exchange of conserved variables (default: when the blocks' driver is kharma)."""
    import torch
    from .batch import Batch
    b = Batch([blk.spec for blk in mesh.blocks], init=None, device=device)
    with torch.cuda.stream(b.torch_stream):
        for blk, block in zip(mesh.blocks, b.blocks):
            block.set_prims(init(blk.spec))
    ghost, n_first, flux = mesh.tables()
    if not flux_correction:
        flux = flux[:0]
    b.set_mesh(ghost, n_first, flux)
    # the initial ghost zones from the initial primitives; the steps' exchanges as the driver's
    b.set_mesh_sync(False)
    b.mesh_exchange()
    b.set_mesh_sync(mesh.base.driver == "kharma" if conserved is None else conserved)
    return b


def conserved_totals(mesh: SMRMesh, batch):
    """Sum over the leaf blocks' interiors of U times the zone volume, per variable (host, FP64)."""
    tot = np.zeros(5)
    for n, (blk, block) in enumerate(zip(mesh.blocks, batch.blocks)):
        U = block.U.cpu().numpy()
        sl = (slice(None),) + blk.spec.interior
        tot += U[sl].reshape(5, -1).sum(axis=1) * mesh.zone_volume(n)
    return tot

"""Static mesh refinement (SMR): a two-level block mesh on a periodic Cartesian domain, stepped as one
batch with ghost-zone exchange and flux correction between blocks (khb_batch_set_mesh).

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
Ghost zones are filled from primitives (then U = U(P) there); every block has the same zone count,
as Parthenon requires, and the fine blocks cover whole coarse blocks (2:1 in each active direction).
Scope: hydro (5 variables), 2 levels, periodic domain.

`SMRMesh.tables()` gives the device tables khb_batch_set_mesh takes:
  ghost entries (int32 x 6): dst block, dst zone, op (0 copy, 1 restrict, 2 prolong), src block,
    src zone (copy: the zone; restrict: the fine zone of lowest index; prolong: the coarse zone),
    aux (prolong: bit d set when the fine zone lies on the + side of the coarse centre along d+1);
    copies and restrictions first, then prolongations (which read coarse ghost zones filled by the
    first group);
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
    (a Cartesian Minkowski BlockSpec supplying the physics options and the domain extent); root
    blocks whose logical location is in `refine` are replaced by their 2^ndim children."""

    def __init__(self, base: BlockSpec, nb, nx, refine=()):
        assert base.cart_minkowski and base.nvar == 5, "SMR: Cartesian Minkowski hydro blocks"
        self.base = base
        self.nb = tuple(nb)
        self.nx = tuple(nx)
        self.ndim = 1 + (nx[1] > 1) + (nx[2] > 1)
        assert all(self.nb[d] == 1 or nx[d] > 1 for d in range(3))
        assert all(nx[d] >= 8 for d in range(self.ndim)), "SMR: at least 8 zones per active direction"
        self.ng = base.ng
        lo = (base.x1min, base.x2min, base.x3min)
        hi = (base.x1max, base.x2max, base.x3max)
        self.lo, self.size = lo, tuple(hi[d] - lo[d] for d in range(3))
        refine = {tuple(r) for r in refine}
        self.blocks = []
        for l3 in range(self.nb[2]):
            for l2 in range(self.nb[1]):
                for l1 in range(self.nb[0]):
                    if (l1, l2, l3) in refine:
                        for c3 in range(2 if self.ndim > 2 else 1):
                            for c2 in range(2 if self.ndim > 1 else 1):
                                for c1 in range(2):
                                    self._add(1, (2 * l1 + c1, 2 * l2 + c2, 2 * l3 + c3))
                    else:
                        self._add(0, (l1, l2, l3))
        self.index = {(b.level, b.loc): n for n, b in enumerate(self.blocks)}

    def _add(self, level, loc):
        f = 2 ** level
        ext = [self.size[d] / (self.nb[d] * (f if d < self.ndim else 1)) for d in range(3)]
        x0 = [self.lo[d] + loc[d] * ext[d] for d in range(3)]
        spec = dataclasses.replace(self.base, nx1=self.nx[0], nx2=self.nx[1], nx3=self.nx[2],
                                   x1min=x0[0], x1max=x0[0] + ext[0], x2min=x0[1], x2max=x0[1] + ext[1],
                                   x3min=x0[2], x3max=x0[2] + ext[2],
                                   bc=tuple("exchange" if f // 2 < self.ndim else "periodic" for f in range(6)))
        self.blocks.append(MeshBlock(level, loc, spec))

    # ------------------------------------------------------------------ topology
    def _zones_at(self, level):
        """Zones along each direction of the whole domain at a level (inactive directions: 1)."""
        return [self.nb[d] * self.nx[d] * (2 ** level if d < self.ndim else 1) for d in range(3)]

    def _leaf(self, level, g):
        """Block covering global zone g (3 ints, wrapped) at `level`, or None."""
        loc = tuple(g[d] // self.nx[d] if d < self.ndim else 0 for d in range(3))
        return self.index.get((level, loc))

    def _local(self, b, g):
        """Local zone index (k, j, i) in block b of the global zone g at b's level."""
        blk = self.blocks[b]
        ng = self.ng
        i = g[0] - blk.loc[0] * self.nx[0] + ng
        j = g[1] - blk.loc[1] * self.nx[1] + ng if self.ndim > 1 else 0
        k = g[2] - blk.loc[2] * self.nx[2] + ng if self.ndim > 2 else 0
        return k, j, i

    def _zone(self, b, kji):
        s = self.blocks[b].spec
        n3, n2, n1 = s.shape
        k, j, i = kji
        return (k * n2 + j) * n1 + i

    def tables(self):
        ghost_a, ghost_b, flux = [], [], []
        ng, ndim = self.ng, self.ndim
        for b, blk in enumerate(self.blocks):
            s = blk.spec
            n3, n2, n1 = s.shape
            L = blk.level
            tot = self._zones_at(L)
            for k in range(n3):
                for j in range(n2):
                    for i in range(n1):
                        inside = (ng <= i < ng + self.nx[0]) and (ndim < 2 or ng <= j < ng + self.nx[1]) and \
                                 (ndim < 3 or ng <= k < ng + self.nx[2])
                        if inside:
                            continue
                        g = [(blk.loc[0] * self.nx[0] + i - ng) % tot[0],
                             ((blk.loc[1] * self.nx[1] + j - ng) % tot[1]) if ndim > 1 else 0,
                             ((blk.loc[2] * self.nx[2] + k - ng) % tot[2]) if ndim > 2 else 0]
                        dst = (k * n2 + j) * n1 + i
                        src = self._leaf(L, g)
                        if src is not None:
                            ghost_a.append((b, dst, OP_COPY, src, self._zone(src, self._local(src, g)), 0))
                            continue
                        if L == 1:
                            gc = [g[d] // 2 if d < ndim else 0 for d in range(3)]
                            src = self._leaf(0, gc)
                            assert src is not None, "mesh is not 2:1 balanced"
                            aux = sum((g[d] % 2) << d for d in range(ndim))
                            ghost_b.append((b, dst, OP_PROLONG, src, self._zone(src, self._local(src, gc)), aux))
                            continue
                        gf = [2 * g[d] if d < ndim else 0 for d in range(3)]
                        src = self._leaf(1, gf)
                        assert src is not None, "ghost zone with no covering block"
                        ghost_a.append((b, dst, OP_RESTRICT, src, self._zone(src, self._local(src, gf)), 0))
            # flux correction: faces of a coarse block bordering fine blocks
            if L == 0:
                for d in range(ndim):
                    for side in (0, 1):
                        # global coarse index of the zone just across the face
                        for t in self._face_positions(blk, d):
                            gz = list(t)
                            gz[d] = (blk.loc[d] * self.nx[d] + (self.nx[d] if side else -1)) % tot[d]
                            if self._leaf(0, gz) is not None:
                                continue
                            # the coarse face (zone index of the zone above it) in this block
                            ci = list(t)
                            ci[d] = blk.loc[d] * self.nx[d] + (self.nx[d] if side else 0)
                            kji = self._local_unwrapped(b, ci)
                            cface = self._zone(b, kji)
                            # the fine face: 2x the coarse face index, tangential 2x
                            tot1 = self._zones_at(1)
                            gf = [2 * t[e] if e < ndim else 0 for e in range(3)]
                            gf[d] = (2 * ci[d]) % tot1[d]
                            # the fine block owning the zone above (side 1) or below (side 0) the face
                            gown = list(gf)
                            if not side:
                                gown[d] = (gf[d] - 1) % tot1[d]
                            fb = self._leaf(1, gown)
                            assert fb is not None
                            fk, fj, fi = self._local(fb, gown)
                            if not side:
                                # the face above the fine zone below it
                                fi, fj, fk = (fi + 1, fj, fk) if d == 0 else ((fi, fj + 1, fk) if d == 1 else (fi, fj, fk + 1))
                            flux.append((b, d + 1, cface, fb, self._zone(fb, (fk, fj, fi)), 0))
        ghost = np.array(ghost_a + ghost_b, dtype=np.int32).reshape(-1, 6)
        flux = np.array(flux, dtype=np.int32).reshape(-1, 6)
        return ghost, len(ghost_a), flux

    def _face_positions(self, blk, d):
        """Global (unwrapped) coarse zone indices of the zones along block blk's faces normal to d
        (the normal coordinate is filled in by the caller)."""
        rng = [range(blk.loc[e] * self.nx[e], (blk.loc[e] + 1) * self.nx[e]) if e < self.ndim else range(1)
               for e in range(3)]
        rng[d] = range(1)
        for c in rng[2]:
            for bb in rng[1]:
                for a in rng[0]:
                    yield (a, bb, c)

    def _local_unwrapped(self, b, g):
        blk = self.blocks[b]
        ng = self.ng
        i = g[0] - blk.loc[0] * self.nx[0] + ng
        j = g[1] - blk.loc[1] * self.nx[1] + ng if self.ndim > 1 else 0
        k = g[2] - blk.loc[2] * self.nx[2] + ng if self.ndim > 2 else 0
        return k, j, i

    # ------------------------------------------------------------------ helpers
    def zone_volume(self, b):
        dx = self.blocks[b].spec.dx
        return dx[0] * dx[1] * dx[2]

    @property
    def zones(self):
        return len(self.blocks) * self.nx[0] * self.nx[1] * self.nx[2]


def smr_batch(mesh: SMRMesh, init, flux_correction=True, device="cuda"):
    """A Batch of the mesh's blocks with initial primitives init(spec) -> (5, n3, n2, n1) per block,
    the mesh tables set and the ghost zones exchanged.  flux_correction=False leaves the coarse
    faces on fine-coarse boundaries uncorrected (for tests of conservation)."""
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
    b.mesh_exchange()
    return b


def conserved_totals(mesh: SMRMesh, batch):
    """Sum over the leaf blocks' interiors of U times the zone volume, per variable (host, FP64)."""
    tot = np.zeros(5)
    for n, (blk, block) in enumerate(zip(mesh.blocks, batch.blocks)):
        U = block.U.cpu().numpy()
        sl = (slice(None),) + blk.spec.interior
        tot += U[sl].reshape(5, -1).sum(axis=1) * mesh.zone_volume(n)
    return tot

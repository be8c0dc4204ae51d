"""Static mesh refinement of magnetized blocks with a face-centred field (B_CT): the tables and the
driver of an SMR mesh of MHD blocks stepped with B_CT (any coordinate system: the operators act on the
native grid, the faces holding sqrt(-g) B^i).

KHARMA defaults multilevel meshes to B_CT (kharma.cpp:376-395): the field lives on faces and its
divergence stays at round-off only if every block sees the same field across a fine-coarse
boundary.  Parthenon (unvendored) and KHARMA's B_CT package do that with three pieces, restated
here as tables the library executes:

  * EMF correction (kharma_step.cpp:183-194, Parthenon's flux correction of edge variables): an
    edge of a coarse block that coincides with edges of finer blocks takes the average of the fine
    edge EMFs along it (one fine edge where the edge direction is inactive), so that the coarse face
    on the boundary changes by the average of the fine faces' changes;
  * the hydro flux correction of the cell-centred variables (the coarse face takes the average of
    the fine fluxes through it, SMRMesh.tables());
  * the face field's ghost exchange: same-level faces copied; a coarse block's ghost face covered by
    finer blocks is the area average of the 2^(ndim-1) fine faces on it (RestrictAverage; 4 in 2D
    for the x3 field, which is zone-centred there); a fine block's ghost face on a coarse face is the
    coarse value plus minmod-limited tangential slopes times +-1/4 (ProlongateSharedMinMod), and a
    fine face inside a coarse zone follows the divergence-preserving operator of Olivares et al.
    (ProlongateInternalOlivares, b_ct_functions.hpp:151-200) from the shared faces around it, its
    sub-face element el lying (el % 2) zones up along the next direction and (el // 2) along the
    third (the reference's offsets exchange the two, which in 3D leaves the fine zones with a
    divergence; in 2D both give the same faces).
The cell-centred fluid primitives are exchanged as in SMRMesh; the ghost zones then take B from
their faces and U = U(P).

Face table entries (int32 x 8): dst block, face direction d (0: x1, 1: x2, 2: x3), dst face (flat
index in the [n3][n2][n1] face array, face i being the left face of zone i), op, src block, src face,
aux, phase.  op 0 copy; 1 restriction (src: the fine face of lowest tangential indices); 2 shared
prolongation (src: the coarse face; aux bit a: + side along axis a); 3 internal prolongation (src
block = dst block, src: the lowest fine zone of the coarse zone, aux: Olivares' sub-face element).
phase 0 holds copies and restrictions; a prolongation into a level-L block has phase 2L-1 (shared)
or 2L (internal), so that each reads only faces earlier phases filled.  Internal faces whose
operator would read past the face arrays (the arrays stop at face n-1 along each direction, where
Parthenon stores face n) are left unfilled; they lie in the outermost ghost layer, which no
reconstruction stencil reaches.

EMF table entries (int32 x 6): coarse block, edge direction e, coarse edge (flat), fine block, fine
edge (flat, the sub-edge of lowest index along e), 0.  Edges follow the library's layout: E1 at
(i centre, j face, k face), E2 at (i face, j centre, k face), E3 at (i face, j face, k centre).
"""
import ctypes as C

import numpy as np

from . import _lib
from .mesh import SMRMesh

FOP_COPY, FOP_RESTRICT, FOP_SHARED, FOP_INTERNAL = 0, 1, 2, 3


class _Geo:
    """Index helpers of an SMRMesh: level-L global coordinates, owners of zones and faces."""

    def __init__(self, mesh: SMRMesh):
        self.m = mesh
        self.ng, self.nx, self.ndim = mesh.ng, mesh.nx, mesh.ndim
        self.act = [a < mesh.ndim for a in range(3)]
        self.own = [mesh._owners(L) for L in range(mesh.levels)]
        self.shape = mesh.blocks[0].spec.shape        # (n3, n2, n1)

    def tot(self, L):
        return self.m._zones_at(L)

    def zone_owner(self, L, g):
        """Block owning level-L zones g (list of 3 arrays, x1..x3; periodic directions wrap); -1 where
        none, or past a physical domain face."""
        if L < 0 or L >= self.m.levels:
            return np.full(len(g[0]), -1, dtype=np.int64)
        t = self.tot(L)
        ok = np.ones(len(g[0]), dtype=bool)
        for a in range(3):
            if self.act[a] and not self.m.periodic[a]:
                ok &= (g[a] >= 0) & (g[a] < t[a])
        lo = [(np.clip(g[a], 0, t[a] - 1) if not self.m.periodic[a] else g[a] % t[a]) // self.nx[a]
              if self.act[a] else np.zeros_like(g[a]) for a in range(3)]
        return np.where(ok, self.own[L][lo[2], lo[1], lo[0]], -1)

    def wrap(self, v, a, t):
        return v % t if self.m.periodic[a] else v

    def local(self, b, L, g):
        """Local (x1, x2, x3) indices in block b of level-L global zones g that b owns."""
        blk = self.m.blocks[b]
        t = self.tot(L)
        return [((g[a] - blk.loc[a] * self.nx[a]) % t[a]) + self.ng if self.act[a] else np.zeros_like(g[a])
                for a in range(3)]

    def flat(self, loc3):
        n3, n2, n1 = self.shape
        return (loc3[2] * n2 + loc3[1]) * n1 + loc3[0]

    def face_owner(self, L, d, g):
        """Owner and local indices of level-L faces of direction d at global coordinates g (g[d] the
        face index: the face between zones g[d]-1 and g[d]).  The block holding zone g[d] takes it
        (its lower face), else the block holding zone g[d]-1 (its upper face)."""
        if not self.act[d]:
            b = self.zone_owner(L, g)
            return b, [np.where(b >= 0, x, 0) for x in self._locals(b, L, g)]
        hi = list(g)
        lo = list(g)
        lo[d] = g[d] - 1
        bh = self.zone_owner(L, hi)
        bl = self.zone_owner(L, lo)
        b = np.where(bh >= 0, bh, bl)
        lh = self._locals(bh, L, hi)
        ll = self._locals(bl, L, lo)
        ll[d] = ll[d] + 1
        loc = [np.where(bh >= 0, lh[a], ll[a]) for a in range(3)]
        return b, loc

    def _locals(self, bs, L, g):
        out = [np.zeros_like(g[0]) for _ in range(3)]
        for b in np.unique(bs[bs >= 0]):
            m = bs == b
            lb = self.local(int(b), L, [g[a][m] for a in range(3)])
            for a in range(3):
                out[a][m] = lb[a]
        return out


def face_tables(mesh: SMRMesh):
    """(entries int32 [n, 8], phase boundaries: entries of phase p are [ends[p-1], ends[p]), number of
    internal faces skipped at the array ends)."""
    G = _Geo(mesh)
    ng, nx, act = G.ng, G.nx, G.act
    n3, n2, n1 = G.shape
    dims = (n1, n2, n3)
    rows = []
    skipped = 0
    for b, blk in enumerate(mesh.blocks):
        L = blk.level
        t = G.tot(L)
        K, J, I = np.meshgrid(np.arange(n3), np.arange(n2), np.arange(n1), indexing="ij")
        loc3 = [I.ravel(), J.ravel(), K.ravel()]
        for d in range(3):
            # owned faces: [ng, ng + nx] along an active d, the interior across
            owned = np.ones(len(loc3[0]), dtype=bool)
            for a in range(3):
                if not act[a]:
                    continue
                hi = ng + nx[a] if a == d else ng + nx[a] - 1
                owned &= (loc3[a] >= ng) & (loc3[a] <= hi)
            sel = ~owned
            lg = [loc3[a][sel] for a in range(3)]
            g = [G.wrap(blk.loc[a] * nx[a] + lg[a] - ng, a, t[a]) if act[a] else np.zeros_like(lg[a]) for a in range(3)]
            # faces past a physical domain face are the block's own boundary condition's (the domain
            # face itself, at index t along d, belongs to the last block)
            keep = np.ones(len(lg[0]), dtype=bool)
            for a in range(3):
                if act[a] and not mesh.periodic[a]:
                    keep &= (g[a] >= 0) & (g[a] <= (t[a] if a == d else t[a] - 1))
            lg = [x[keep] for x in lg]
            g = [x[keep] for x in g]
            dst = G.flat(lg)
            n = len(dst)
            ent = np.full((n, 8), -1, dtype=np.int64)
            ent[:, 0] = b
            ent[:, 1] = d
            ent[:, 2] = dst
            done = np.zeros(n, dtype=bool)
            # same level: copy
            sb, sl = G.face_owner(L, d, g)
            m = sb >= 0
            ent[m, 3] = FOP_COPY
            ent[m, 4] = sb[m]
            ent[m, 5] = G.flat([sl[a][m] for a in range(3)])
            ent[m, 6] = 0
            ent[m, 7] = 0
            done |= m
            # finer: restriction from the fine face of lowest tangential indices
            if L + 1 < mesh.levels:
                gf = [2 * g[a] if act[a] else g[a] for a in range(3)]
                fb, fl = G.face_owner(L + 1, d, gf)
                m = (~done) & (fb >= 0)
                ent[m, 3] = FOP_RESTRICT
                ent[m, 4] = fb[m]
                ent[m, 5] = G.flat([fl[a][m] for a in range(3)])
                ent[m, 6] = 0
                ent[m, 7] = 0
                done |= m
            rest = ~done
            if rest.any():
                assert L > 0, "ghost face with no source: the mesh is not 2:1 balanced"
                shared = rest.copy()
                if act[d]:
                    shared &= (g[d] % 2) == 0
                internal = rest & ~shared
                # shared faces: the coarse face and its tangential neighbours
                if shared.any():
                    gc = [g[a][shared] // 2 if act[a] else g[a][shared] for a in range(3)]
                    cb, cl = G.face_owner(L - 1, d, gc)
                    assert (cb >= 0).all(), "mesh is not 2:1 balanced"
                    aux = np.zeros(int(shared.sum()), dtype=np.int64)
                    for a in range(3):
                        if act[a] and a != d:
                            aux |= (g[a][shared] % 2) << a
                    ent[shared, 3] = FOP_SHARED
                    ent[shared, 4] = cb
                    ent[shared, 5] = G.flat(cl)
                    ent[shared, 6] = aux
                    ent[shared, 7] = 2 * L - 1
                if internal.any():
                    nxt, thd = (d + 1) % 3, (d + 2) % 3
                    base = [lg[a][internal] - (g[a][internal] % 2) if act[a] else lg[a][internal] for a in range(3)]
                    base[d] = lg[d][internal] - 1
                    par = lambda a: (g[a][internal] % 2) if act[a] else np.ones(int(internal.sum()), dtype=np.int64)
                    # element: (el % 2) along nxt, (el // 2) along thd; where a direction is inactive the
                    # operator writes the face twice and the later element stays
                    elem = 2 * par(thd) + par(nxt)
                    # the operator reads faces up to base + 2 along every active direction
                    fits = np.ones(int(internal.sum()), dtype=bool)
                    for a in range(3):
                        if act[a]:
                            fits &= base[a] + 2 <= dims[a] - 1
                    idx = np.nonzero(internal)[0]
                    skipped += int((~fits).sum())
                    ok = idx[fits]
                    ent[ok, 3] = FOP_INTERNAL
                    ent[ok, 4] = b
                    ent[ok, 5] = G.flat([base[a][fits] for a in range(3)])
                    ent[ok, 6] = elem[fits]
                    ent[ok, 7] = 2 * L
                    ent = np.delete(ent, idx[~fits], axis=0)
            rows.append(ent)
    ent = np.concatenate(rows) if rows else np.zeros((0, 8), dtype=np.int64)
    ent = ent[np.argsort(ent[:, 7], kind="stable")]
    nph = int(ent[:, 7].max()) + 1 if len(ent) else 0
    ends = np.array([int((ent[:, 7] <= p).sum()) for p in range(nph)], dtype=np.int64)
    return ent.astype(np.int32), ends, skipped


def emf_table(mesh: SMRMesh):
    """EMF correction entries (int32 [n, 6])."""
    G = _Geo(mesh)
    ng, nx, act = G.ng, G.nx, G.act
    rows = []
    for b, blk in enumerate(mesh.blocks):
        L = blk.level
        if L + 1 >= mesh.levels:
            continue
        t = G.tot(L)
        for e in range(3):
            # the block's edges: zones along e, nodes across
            rng = []
            for a in range(3):
                if not act[a]:
                    rng.append(np.zeros(1, dtype=np.int64))
                elif a == e:
                    rng.append(np.arange(ng, ng + nx[a]))
                else:
                    rng.append(np.arange(ng, ng + nx[a] + 1))
            Z3, Z2, Z1 = np.meshgrid(rng[2], rng[1], rng[0], indexing="ij")
            lc = [Z1.ravel(), Z2.ravel(), Z3.ravel()]
            bnd = np.zeros(len(lc[0]), dtype=bool)
            for a in range(3):
                if act[a] and a != e:
                    bnd |= (lc[a] == ng) | (lc[a] == ng + nx[a])
            lc = [x[bnd] for x in lc]
            if not len(lc[0]):
                continue
            g = [G.wrap(blk.loc[a] * nx[a] + lc[a] - ng, a, t[a]) if act[a] else np.zeros_like(lc[a]) for a in range(3)]
            # fine edge of lowest index along e; the fine zones around it
            gf = [2 * g[a] if act[a] else g[a] for a in range(3)]
            trans = [a for a in range(3) if a != e and act[a]]
            fb = np.full(len(g[0]), -1, dtype=np.int64)
            fl = [np.zeros_like(g[0]) for _ in range(3)]
            for shifts in ([(0, 0), (0, -1), (-1, 0), (-1, -1)] if len(trans) == 2 else [(0,), (-1,)]):
                z = list(gf)
                for a, s in zip(trans, shifts):
                    z[a] = gf[a] + s
                ob = G.zone_owner(L + 1, z)
                take = (fb < 0) & (ob >= 0)
                if not take.any():
                    continue
                zl = G._locals(np.where(take, ob, -1), L + 1, z)
                for a in range(3):
                    v = zl[a]
                    if a in trans and shifts[trans.index(a)] == -1:
                        v = v + 1          # the zone below the node: its upper node
                    fl[a] = np.where(take, v, fl[a])
                fb = np.where(take, ob, fb)
            m = fb >= 0
            if not m.any():
                continue
            n = int(m.sum())
            rows.append(np.stack([np.full(n, b), np.full(n, e), G.flat([x[m] for x in lc]), fb[m],
                                  G.flat([x[m] for x in fl]), np.zeros(n, dtype=np.int64)], axis=1))
    ent = np.concatenate(rows) if rows else np.zeros((0, 6), dtype=np.int64)
    return ent.astype(np.int32)


def cell_phase_ends(ghost, n_first):
    """Phase ends of SMRMesh.tables()'s ghost-zone entries: copies and restrictions, then the
    prolongations of each destination level (aux >> 8 = level - 1)."""
    ends = [int(n_first)]
    if len(ghost) > n_first:
        ph = ghost[n_first:, 5] >> 8
        for p in range(int(ph.max()) + 1):
            ends.append(int(n_first + (ph <= p).sum()))
    return np.array(ends, dtype=np.int64)


class CTMesh:
    """An SMRMesh of B_CT MHD blocks stepped with RK2: per block khb_ct_stage_fluxes, the mesh's flux
    and EMF corrections, khb_ct_stage_update, then the ghost exchange of the stage output.
    P_blocks: each block's primitives (8, n3, n2, n1) over the whole block; Bf_blocks: each block's
    face field (3, n3, n2, n1), or None to interpolate it from the zone B.  conserved: the kharma
    driver's exchange (default: when the blocks' driver is kharma): the update, the exchange of the
    updated conserved state with the seed primitives and the faces, the ghost zones inverted like the
    interior, then the interior's inversion and fixups (khb_ct_stage_update_part,
    khb_ctmesh_exchange_cons).  The initial ghost zones come from the initial primitives."""

    def __init__(self, mesh: SMRMesh, P_blocks, Bf_blocks=None, emf_correction=True, flux_correction=True,
                 streams=1, conserved=None):
        import torch
        from .block import Block, Fields
        self.torch = torch
        self.mesh = mesh
        self.blocks = []
        for n, blk in enumerate(mesh.blocks):
            b = Block(blk.spec)
            b.set_prims(P_blocks[n], faces=None if Bf_blocks is None else Bf_blocks[n])
            self.blocks.append(b)
        self.lib = self.blocks[0].lib
        self.conserved = (mesh.base.driver == "kharma") if conserved is None else bool(conserved)
        self._physical = [any(x not in ("exchange", "periodic") for x in blk.spec.bc) for blk in mesh.blocks]
        self.P1 = [torch.zeros_like(b.P) for b in self.blocks]
        self.U1 = [torch.zeros_like(b.U) for b in self.blocks]
        self.Bf1 = [torch.zeros_like(b.Bf) for b in self.blocks]
        self.F1 = [(Fields(p), Fields(u), Fields(f)) for p, u, f in zip(self.P1, self.U1, self.Bf1)]
        ghost, n_first, flux = mesh.tables()
        cell_ends = cell_phase_ends(ghost, n_first)
        face, face_ends, self.skipped_faces = face_tables(mesh)
        emf = emf_table(mesh)
        if not flux_correction:
            flux = flux[:0]
        if not emf_correction:
            emf = emf[:0]
        self.tables = {"cell": ghost, "face": face, "flux": flux, "emf": emf}
        self._keep = [np.ascontiguousarray(x) for x in (ghost, cell_ends, face, face_ends, flux, emf)]
        g, ce, f, fe, fl, em = self._keep
        ptr = lambda a: a.ctypes.data_as(C.c_void_p)
        ctxs = (C.c_void_p * len(self.blocks))(*[b.ctx.value for b in self.blocks])
        m = C.c_void_p()
        _lib.check(self.lib.khb_ctmesh_create(ctxs, len(self.blocks), ptr(g), len(g), ptr(ce), len(ce), ptr(f), len(f),
                                              ptr(fe), len(fe), ptr(fl), len(fl), ptr(em), len(em), C.byref(m)),
                   "khb_ctmesh_create")
        self.m = m
        self._graph = None
        # the per-block work of each phase is spread over this many streams (blocks are independent
        # there), joined before the mesh-wide corrections and exchange
        self.streams = [torch.cuda.Stream() for _ in range(max(0, int(streams) - 1))]
        self.exchange(0)

    def __del__(self):
        try:
            if getattr(self, "m", None):
                self.lib.khb_ctmesh_destroy(self.m)
                self.m = None
        except Exception:
            pass

    @property
    def stream(self):
        return self.blocks[0].stream

    def _state(self, s):
        """(P, U, Bf) Fields of every block: s = 0 the state, 1 the intermediate stage."""
        if s == 0:
            return [(b.Pf, b.Uf, b.Bff) for b in self.blocks]
        return self.F1

    def _per_block(self, fn):
        """fn(n, block) for every block, block n on stream n mod (1 + extra streams), joined back."""
        torch = self.torch
        main = torch.cuda.current_stream()
        lanes = [main] + self.streams
        for s in self.streams:
            s.wait_stream(main)
        for n, b in enumerate(self.blocks):
            with torch.cuda.stream(lanes[n % len(lanes)]):
                fn(n, b)
        for s in self.streams:
            main.wait_stream(s)

    def exchange(self, s):
        """Ghost zones and ghost faces of state s, then B and U = U(P) in every block's ghost zones."""
        st = self._state(s)
        P = (_lib.KhbFields * len(st))(*[x[0].s for x in st])
        B = (_lib.KhbFields * len(st))(*[x[2].s for x in st])
        _lib.check(self.lib.khb_ctmesh_exchange(self.m, C.cast(P, C.c_void_p), C.cast(B, C.c_void_p), self.stream),
                   "khb_ctmesh_exchange")

        def ghosts(n, b):
            Pf, Uf, Bff = st[n]
            # B from the exchanged faces in every ghost zone (MeshUtoP over the entire block, before the
            # domain conditions: kharma_step.cpp:233-249)
            _lib.check(self.lib.khb_ct_ghost_from_faces(b.ctx, Pf.ref, Uf.ref, Bff.ref, b.stream),
                       "khb_ct_ghost_from_faces")
            if self._physical[n]:
                # then the physical domain faces, over the ghost rows the exchange filled; they
                # recompute B and U only past those faces
                _lib.check(self.lib.khb_ct_boundaries(b.ctx, Pf.ref, Uf.ref, Bff.ref, b.stream), "khb_ct_boundaries")
        self._per_block(ghosts)

    def exchange_cons(self, P_s, U, P_out, Bf):
        """The kharma driver's exchange (khb_ctmesh_exchange_cons) on per-block Fields: seeds P_s, updated
        conserved state U, output primitives P_out, faces Bf."""
        n = len(self.blocks)
        arr = lambda fs: C.cast((_lib.KhbFields * n)(*[f.s for f in fs]), C.c_void_p)
        pf = (C.c_void_p * n)(*[b.pflag.data_ptr() for b in self.blocks])
        ff = (C.c_void_p * n)(*[b.fflag.data_ptr() for b in self.blocks])
        _lib.check(self.lib.khb_ctmesh_exchange_cons(self.m, arr(P_s), arr(U), arr(P_out), arr(Bf),
                                                     C.cast(pf, C.c_void_p), C.cast(ff, C.c_void_p), self.stream),
                   "khb_ctmesh_exchange_cons")

    def step(self, dt):
        for stage in (1, 2):
            src = self._state(stage - 1)
            out = self._state(1 if stage == 1 else 0)
            st0 = self._state(0)

            def fluxes(n, b):
                _lib.check(self.lib.khb_ct_stage_fluxes(b.ctx, src[n][0].ref, b.stream), "khb_ct_stage_fluxes")

            def args(n, b):
                (Ps, Us, Bs), (_, U0, B0), (Po, Uo, Bo) = src[n], st0[n], out[n]
                return (stage, float(dt), Ps.ref, Us.ref, U0.ref, Bs.ref, B0.ref, Po.ref, Uo.ref, Bo.ref,
                        C.c_void_p(b.pflag.data_ptr()), C.c_void_p(b.fflag.data_ptr()), b.stream)

            def update(n, b):
                _lib.check(self.lib.khb_ct_stage_update(b.ctx, *args(n, b)), "khb_ct_stage_update")

            def update1(n, b):
                _lib.check(self.lib.khb_ct_stage_update_part(b.ctx, 1, *args(n, b)), "khb_ct_stage_update_part")

            def update2(n, b):
                _lib.check(self.lib.khb_ct_stage_update_part(b.ctx, 2, *args(n, b)), "khb_ct_stage_update_part")
                if self._physical[n]:
                    Po, Uo, Bo = out[n]
                    _lib.check(self.lib.khb_ct_boundaries(b.ctx, Po.ref, Uo.ref, Bo.ref, b.stream), "khb_ct_boundaries")

            self._per_block(fluxes)
            _lib.check(self.lib.khb_ctmesh_correct(self.m, self.stream), "khb_ctmesh_correct")
            if self.conserved:
                self._per_block(update1)
                self.exchange_cons([x[0] for x in src], [x[1] for x in out], [x[0] for x in out],
                                   [x[2] for x in out])
                self._per_block(update2)
            else:
                self._per_block(update)
                self.exchange(1 if stage == 1 else 0)

    def step_graph(self, dt):
        """One step replayed from a CUDA graph of the whole mesh step (captured on the first call for
        this dt, after one eager step that also registers both states' descriptors with the library)."""
        torch = self.torch
        if self._graph is not None and self._graph_dt == dt:
            self._graph.replay()
            return
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            self.step(dt)
        torch.cuda.current_stream().wait_stream(side)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.step(dt)
        self._graph, self._graph_dt = g, dt

    def max_divb(self):
        """Max over the blocks of khb_ct_max_divb (interior zones)."""
        return max(b.max_divb() for b in self.blocks)

    def conserved_totals(self):
        """Sum over the blocks' interiors of U times the zone volume, per variable."""
        tot = np.zeros(8)
        for n, (blk, b) in enumerate(zip(self.mesh.blocks, self.blocks)):
            U = b.U.cpu().numpy()
            sl = (slice(None),) + blk.spec.interior
            tot += U[sl].reshape(8, -1).sum(axis=1) * self.mesh.zone_volume(n)
        return tot


# ------------------------------------------------------------------ initial data of a mesh
def cut(mesh, level_arrays):
    """Block arrays (nvar, n3, n2, n1) from whole-domain arrays level_arrays[L] (nvar, t3, t2, t1),
    ghost zones included (periodic)."""
    out = []
    ndim, ng, nx = mesh.ndim, mesh.ng, mesh.nx
    for blk in mesh.blocks:
        n3, n2, n1 = blk.spec.shape
        tot = mesh._zones_at(blk.level)
        i = (blk.loc[0] * nx[0] + np.arange(n1) - ng) % tot[0]
        j = ((blk.loc[1] * nx[1] + np.arange(n2) - ng) % tot[1]) if ndim > 1 else np.zeros(n2, dtype=int)
        k = ((blk.loc[2] * nx[2] + np.arange(n3) - ng) % tot[2]) if ndim > 2 else np.zeros(n3, dtype=int)
        K, J, I = np.meshgrid(k, j, i, indexing="ij")
        out.append(np.ascontiguousarray(level_arrays[blk.level][:, K, J, I]))
    return out


def level_dx(mesh):
    return [mesh.blocks[[b.level for b in mesh.blocks].index(L)].spec.dx for L in range(mesh.levels)]


def curl_faces_levels(mesh, B0=(1.0, 0.5, 0.25), amp=0.05, walls=False):
    """Whole-domain face arrays (3, t3, t2, t1) per level: B0 plus the discrete curl of
    A = amp (sin(2 pi x2) cos(2 pi x3), sin(2 pi x3) cos(2 pi x1), sin(2 pi x1) cos(2 pi x2)) sampled at
    each level's edges from integer corner indices, so that every level's field is divergence-free to
    rounding and a coarse face equals the mean of the fine faces on it to rounding.  walls (2D): no
    normal field on the x1 and x2 domain faces, as reflecting faces require: A_3 = amp sin(2 pi x1)
    sin(2 pi x2) and B0 along x3 only."""
    out = []
    for L in range(mesh.levels):
        t = mesh._zones_at(L)
        dx = level_dx(mesh)[L]
        d3 = mesh.ndim > 2
        # corner coordinates by integer index (periodic: index t wraps to 0)
        xs = [np.arange(t[a] + 1) * dx[a] for a in range(3)]
        X3, X2, X1 = np.meshgrid(xs[2] if d3 else np.zeros(1), xs[1], xs[0], indexing="ij")
        Z = np.zeros_like(X1)
        A1 = amp * np.sin(2 * np.pi * X2) * (np.cos(2 * np.pi * X3) if d3 else 1.0)      # at (i c, j f, k f)
        A2 = amp * (np.sin(2 * np.pi * X3) if d3 else Z) * np.cos(2 * np.pi * X1)       # at (i f, j c, k f)
        A3 = amp * np.sin(2 * np.pi * X1) * (np.sin if walls else np.cos)(2 * np.pi * X2)   # at (i f, j f, k c)
        if walls:
            B0 = (0.0, 0.0, B0[2])
        n3 = t[2]
        k1 = slice(0, n3) if d3 else slice(0, 1)
        F = np.zeros((3, n3, t[1], t[0]))
        # F1 = dA3/dx2 - dA2/dx3 at x1 faces; F2 = dA1/dx3 - dA3/dx1; F3 = dA2/dx1 - dA1/dx2
        F[0] = B0[0] + (A3[k1, 1:, :-1] - A3[k1, :-1, :-1]) / dx[1]
        F[1] = B0[1] - (A3[k1, :-1, 1:] - A3[k1, :-1, :-1]) / dx[0]
        F[2] = B0[2] + ((A2[k1, :-1, 1:] - A2[k1, :-1, :-1]) / dx[0] - (A1[k1, 1:, :-1] - A1[k1, :-1, :-1]) / dx[1])
        if d3:
            F[0] -= (A2[1:, :-1, :-1] - A2[:-1, :-1, :-1]) / dx[2]
            F[1] += (A1[1:, :-1, :-1] - A1[:-1, :-1, :-1]) / dx[2]
        out.append(F)
    return out


def potential_faces_levels(mesh, a=0.02, b=0.01):
    """Whole-domain face arrays (sqrt(-g) B^i) per level for any coordinates: the discrete curl in
    native coordinates of A_3 = a sin(pi x2^) (1 + x1^) and A_2 = b sin(2 pi x3^) sin(pi x1^), with
    x^ = corner index / zones along each direction (the same function on every level, periodic in
    x3).  A_3 does not depend on x3 nor A_2 on x2, so a coarse face is the mean of the fine faces on
    it to rounding; the normal field vanishes on the x2 faces (poles)."""
    out = []
    for L in range(mesh.levels):
        t = mesh._zones_at(L)
        dx = level_dx(mesh)[L]
        u = [np.arange(t[q] + 1) / t[q] for q in range(3)]
        I1, J2 = np.meshgrid(u[0], u[1], indexing="xy")                # (t2+1, t1+1): A3 at (i f, j f)
        A3 = a * np.sin(np.pi * J2) * (1 + I1)
        K3, I1b = np.meshgrid(u[2], u[0], indexing="ij")              # (t3+1, t1+1): A2 at (i f, k f)
        A2 = b * np.sin(2 * np.pi * K3) * np.sin(np.pi * I1b)
        F = np.zeros((3, t[2], t[1], t[0]))
        F[0] = ((A3[1:, :-1] - A3[:-1, :-1]) / dx[1])[None] - ((A2[1:, :-1] - A2[:-1, :-1]) / dx[2])[:, None, :]
        F[1] = -((A3[:-1, 1:] - A3[:-1, :-1]) / dx[0])[None]
        F[2] = ((A2[:-1, 1:] - A2[:-1, :-1]) / dx[0])[:, None, :]
        out.append(F)
    return out


def torus_blocks(mesh, seed=1234, u_jitter=0.08):
    """Each block's primitives (8, n3, n2, n1) of the FM torus (problems.fm_torus at the block's own
    zones, the density normalised by the mesh's midplane maximum, the jitter seeded per block), the
    zone field zero (it comes from the faces)."""
    import math
    from . import problems
    from .block import build_geometry
    base = mesh.base
    xs = base.x1min + np.arange(int((base.x1max - base.x1min) / 0.001) + 1) * 0.001
    rho_max = float(np.max(problems._torus_rho(base.a, 6.0, 12.0, base.gam, 1e-3, np.exp(xs),
                                               np.full_like(xs, math.pi / 2))))
    import dataclasses
    out = []
    for n, blk in enumerate(mesh.blocks):
        fluid = dataclasses.replace(blk.spec, nvar=5, b_ct="none")       # no field seeding
        P5 = problems.fm_torus(fluid, build_geometry(blk.spec), seed=seed + n, u_jitter=u_jitter, rho_max=rho_max)
        P = np.zeros((8,) + P5.shape[1:])
        P[:5] = P5
        out.append(P)
    return out


def fluid_levels(mesh, amp=0.1, v=(0.3, 0.2, 0.1)):
    """Whole-domain primitives (8, t3, t2, t1) per level: an entropy wave rho = 1 + amp sin(2 pi (x1 + x2
    (+ x3))) at uniform pressure and velocity; B slots zero (taken from the faces)."""
    out = []
    for L in range(mesh.levels):
        t = mesh._zones_at(L)
        dx = level_dx(mesh)[L]
        xc = [(np.arange(t[a]) + 0.5) * dx[a] for a in range(3)]
        X3, X2, X1 = np.meshgrid(xc[2] if mesh.ndim > 2 else np.zeros(1), xc[1], xc[0], indexing="ij")
        ph = X1 + X2 + (X3 if mesh.ndim > 2 else 0.)
        P = np.zeros((8,) + X1.shape)
        P[0] = 1.0 + amp * np.sin(2 * np.pi * ph)
        P[1] = 1.0
        W = 1.0 / np.sqrt(1.0 - sum(x * x for x in v))
        for a in range(3):
            P[2 + a] = W * v[a]
        out.append(P)
    return out

"""Test infrastructure (the oracle side of the SMR checks): a CPU restatement of the ghost zones a
static-refined mesh of any number of levels gives each block, built from whole-domain arrays rather
than from the per-zone tables the library executes.

The operators are Parthenon's cell-centred refinement operators (Parthenon, AFD-Illinois fork,
commit unpinned and absent from the reference tree) as published, on a uniform grid:
  * restriction: the average of the 2^ndim fine zones (RestrictCellAverage);
  * prolongation: the coarse value plus, per active direction, +-1/4 times the minmod of the
    left and right coarse differences (ProlongateCellMinMod).
The level-L array holds the interiors of the level-L blocks, the restriction of the level-(L+1)
blocks' interiors where level L+1 has blocks, and elsewhere the prolongation of the level-(L-1)
array (itself filled the same way, coarsest first).  With 2:1 balance a ghost zone only ever reads
positions these rules fill.  A block's ghost zone at level L takes the level-L value at its
(periodic) position.  Summation orders follow the library's kernels, so the comparison is bitwise.
"""
import numpy as np


def _minmod(a, b):
    return np.where(a * b > 0., np.where(np.abs(a) < np.abs(b), a, b), 0.)


def _restrict(f, ndim):
    q = lambda dk, dj, di: f[:, dk::2, dj::2, di::2] if ndim > 2 else (f[:, :, dj::2, di::2] if ndim > 1 else f[:, :, :, di::2])
    if ndim > 2:
        r = (q(0, 0, 0) + q(0, 0, 1)) + (q(0, 1, 0) + q(0, 1, 1))
        r = r + ((q(1, 0, 0) + q(1, 0, 1)) + (q(1, 1, 0) + q(1, 1, 1)))
        return r * 0.125
    if ndim > 1:
        return ((q(0, 0, 0) + q(0, 0, 1)) + (q(0, 1, 0) + q(0, 1, 1))) * 0.25
    return (q(0, 0, 0) + q(0, 0, 1)) * 0.5


def _prolong(G, ndim, shape):
    axes = (3, 2, 1)       # x1, x2, x3 along the array axes
    slopes = []
    for d in range(ndim):
        um = np.roll(G, 1, axis=axes[d])
        up = np.roll(G, -1, axis=axes[d])
        slopes.append(_minmod(G - um, up - G))
    pro = np.empty(shape)
    for ok in range(2 if ndim > 2 else 1):
        for oj in range(2 if ndim > 1 else 1):
            for oi in range(2):
                v = G.copy()
                for d, o in zip(range(ndim), (oi, oj, ok)):
                    v = v + (0.25 * slopes[d] if o else -0.25 * slopes[d])
                sl = (slice(None), slice(ok, None, 2) if ndim > 2 else slice(None),
                      slice(oj, None, 2) if ndim > 1 else slice(None), slice(oi, None, 2))
                pro[sl] = v
    return pro


def level_arrays(mesh, P_blocks):
    """Whole-domain primitive arrays (nvar, n3, n2, n1), one per level, coarsest first."""
    ndim, ng, nx = mesh.ndim, mesh.ng, mesh.nx
    nv = P_blocks[0].shape[0]
    G = []
    for L in range(mesh.levels):
        t = mesh._zones_at(L)
        G.append(np.full((nv, t[2], t[1], t[0]), np.nan))

    def interior(P):
        return P[(slice(None),) + (slice(ng, ng + nx[2]) if ndim > 2 else slice(0, 1),
                                   slice(ng, ng + nx[1]) if ndim > 1 else slice(0, 1),
                                   slice(ng, ng + nx[0]))]

    for blk, P in zip(mesh.blocks, P_blocks):
        sl = tuple(slice(blk.loc[d] * nx[d], (blk.loc[d] + 1) * nx[d]) if d < ndim else slice(0, 1)
                   for d in (2, 1, 0))
        G[blk.level][(slice(None),) + sl] = interior(P)
    # restriction of each level's block interiors into the level below
    inter = [g.copy() for g in G]
    for L in range(mesh.levels - 1):
        r = _restrict(inter[L + 1], ndim)
        G[L] = np.where(np.isnan(G[L]) & ~np.isnan(r), r, G[L])
    # prolongation, coarsest first, where a level has neither blocks nor restricted values
    for L in range(1, mesh.levels):
        G[L] = np.where(np.isnan(G[L]), _prolong(G[L - 1], ndim, G[L].shape), G[L])
    return G


def expected_ghosts(mesh, P_blocks):
    """For each block: (mask of its ghost zones, expected primitives there) as full-block arrays."""
    G = level_arrays(mesh, P_blocks)
    ndim, ng, nx = mesh.ndim, mesh.ng, mesh.nx
    out = []
    for blk, P in zip(mesh.blocks, P_blocks):
        n3, n2, n1 = blk.spec.shape
        tot = mesh._zones_at(blk.level)
        i = (blk.loc[0] * nx[0] + np.arange(n1) - ng) % tot[0]
        j = ((blk.loc[1] * nx[1] + np.arange(n2) - ng) % tot[1]) if ndim > 1 else np.zeros(n2, dtype=int)
        k = ((blk.loc[2] * nx[2] + np.arange(n3) - ng) % tot[2]) if ndim > 2 else np.zeros(n3, dtype=int)
        K, J, I = np.meshgrid(k, j, i, indexing="ij")
        E = G[blk.level][:, K, J, I]
        inside = np.zeros((n3, n2, n1), dtype=bool)
        inside[blk.spec.interior] = True
        out.append((~inside, E))
    return out


# ---------------------------------------------------------------------------- face fields (B_CT)
# The face field of B_CT blocks (sqrt(-g) B^d on the x_d faces, face i the lower face of zone i) on
# whole-domain level arrays, as Parthenon's face refinement operators and KHARMA's Olivares
# prolongation (b_ct_functions.hpp:151-200) fill a block's ghost faces, on a uniform Cartesian grid:
#   * faces of level-L blocks: their own values (a face two blocks share: the block above it);
#   * elsewhere, where level L+1 has blocks: the mean of the 2^(ndim-1) fine faces on the coarse face
#     (RestrictAverage; in 2D the x3 field is zone-centred: the mean of 4);
#   * elsewhere (level L-1 below), faces on a coarse face: the coarse value plus, per tangential active
#     direction, +-1/4 of the minmod of the coarse differences (ProlongateSharedMinMod); faces inside a
#     coarse zone: Olivares' operator from the faces around them (ProlongateInternalOlivares).
# Summation orders follow the library's kernels, so the comparison is bitwise.


def _face_levels_owned(mesh, Bf_blocks):
    ndim, ng, nx = mesh.ndim, mesh.ng, mesh.nx
    act = [a < ndim for a in range(3)]
    G = []
    for L in range(mesh.levels):
        t = mesh._zones_at(L)
        G.append([np.full((t[2], t[1], t[0]), np.nan) for _ in range(3)])
    for upper in (True, False):
        for blk, B in zip(mesh.blocks, Bf_blocks):
            t = mesh._zones_at(blk.level)
            for d in range(3):
                idx = []
                for a in (2, 1, 0):
                    if not act[a]:
                        idx.append((np.zeros(1, dtype=int), np.zeros(1, dtype=int)))
                        continue
                    if a == d:
                        loc = np.array([ng + nx[a]]) if upper else np.arange(ng, ng + nx[a])
                    else:
                        loc = np.arange(ng, ng + nx[a])
                    idx.append((loc, (blk.loc[a] * nx[a] + loc - ng) % t[a]))
                if upper and not act[d]:
                    continue
                (lk, gk), (lj, gj), (li, gi) = idx
                G[blk.level][d][np.ix_(gk, gj, gi)] = B[d][np.ix_(lk, lj, li)]
    return G


def face_level_arrays(mesh, Bf_blocks, dx_levels):
    """Whole-domain face arrays [level][d] (n3, n2, n1) filled by the rules above.  dx_levels[L]: the
    zone widths (dx1, dx2, dx3) at level L (dx3 of a 2D mesh: the x3 extent)."""
    ndim = mesh.ndim
    act = [a < ndim for a in range(3)]
    ax = (2, 1, 0)          # array axis of x1, x2, x3
    G = _face_levels_owned(mesh, Bf_blocks)
    owned = [[g.copy() for g in GL] for GL in G]

    def sl(a, start):
        """Slice selecting every other index along x_a from start (all of an inactive axis)."""
        s = [slice(None)] * 3
        if act[a]:
            s[ax[a]] = slice(start, None, 2)
        return tuple(s)

    # restriction from the finer level's own faces
    for L in range(mesh.levels - 1):
        for d in range(3):
            f = owned[L + 1][d]
            tr = [a for a in range(3) if act[a] and a != d]
            base = [slice(None)] * 3
            if act[d]:
                base[ax[d]] = slice(0, None, 2)
            def q(*offs):
                s = list(base)
                for a, o in zip(tr, offs):
                    s[ax[a]] = slice(o, None, 2)
                return f[tuple(s)]
            if len(tr) == 2:
                r = ((q(0, 0) + q(1, 0)) + (q(0, 1) + q(1, 1))) * 0.25
            else:
                r = (q(0) + q(1)) * 0.5
            G[L][d] = np.where(np.isnan(G[L][d]) & ~np.isnan(r), r, G[L][d])
    # prolongation, coarsest first: faces on coarse faces, then faces inside coarse zones
    for L in range(1, mesh.levels):
        for d in range(3):
            C = G[L - 1][d]
            tr = [a for a in range(3) if act[a] and a != d]
            slopes = {a: _minmod(C - np.roll(C, 1, axis=ax[a]), np.roll(C, -1, axis=ax[a]) - C) for a in tr}
            pro = np.full(G[L][d].shape, np.nan)
            for par in range(1 << len(tr)):
                v = C.copy()
                for n, a in enumerate(tr):
                    v = v + (0.25 * slopes[a] if (par >> n) & 1 else -0.25 * slopes[a])
                s = [slice(None)] * 3
                if act[d]:
                    s[ax[d]] = slice(0, None, 2)
                for n, a in enumerate(tr):
                    s[ax[a]] = slice((par >> n) & 1, None, 2)
                pro[tuple(s)] = v
            G[L][d] = np.where(np.isnan(G[L][d]) & ~np.isnan(pro), pro, G[L][d])
        dx1, dx2, dx3 = dx_levels[L]
        a3 = [(dx2*dx2 - dx3*dx3) / (dx2*dx2 + dx3*dx3), (dx3*dx3 - dx1*dx1) / (dx3*dx3 + dx1*dx1),
              (dx1*dx1 - dx2*dx2) / (dx1*dx1 + dx2*dx2)]
        area = [dx2 * dx3, dx1 * dx3, dx1 * dx2]
        for me in range(ndim):
            nxt, thd = (me + 1) % 3, (me + 2) % 3
            cf = [[3 + a3[nxt], 1 - a3[nxt], 3 - a3[thd], 1 + a3[thd]],
                  [3 + a3[nxt], 1 - a3[nxt], 1 + a3[thd], 3 - a3[thd]],
                  [1 - a3[nxt], 3 + a3[nxt], 3 - a3[thd], 1 + a3[thd]],
                  [1 - a3[nxt], 3 + a3[nxt], 1 + a3[thd], 3 - a3[thd]]]
            cur = G[L]

            def at(df, shift):
                """cur[df] at base + shift (x1, x2, x3), base = the lowest fine zone of every coarse zone."""
                s = [slice(None)] * 3
                arr = cur[df]
                for a in range(3):
                    if act[a]:
                        arr = np.roll(arr, -shift[a], axis=ax[a])
                        s[ax[a]] = slice(0, None, 2)
                return arr[tuple(s)]

            def unit(a, k=1):
                e = [0, 0, 0]
                if a is not None and 0 <= a < 3 and act[a]:
                    e[a] = k
                return e

            def term(df, ds, of):
                if not act[df]:
                    return 0.
                A = area[df]
                sh = lambda *vs: [sum(v[i] for v in vs) for i in range(3)]
                f2, s_, o_ = unit(df, 2), unit(ds), unit(of if of >= 0 else None)
                return at(df, sh(f2, s_, o_)) * A - at(df, sh(s_, o_)) * A - at(df, sh(f2, o_)) * A + at(df, o_) * A

            V = area[me]
            ta, tb = term(nxt, me, -1), term(nxt, me, thd)
            tc, td = term(thd, me, -1), term(thd, me, nxt)
            # faces inside coarse zones (neither owned, restricted nor on a coarse face); where two
            # elements write one face (an inactive direction), the later one stays, as in the operator
            inside = np.isnan(G[L][me])
            for el in range(4):
                # element el: (el % 2) zones up along nxt, (el // 2) along thd, which pairs each sub-face
                # with the coefficient row of the halves it borders (divergence-preserving; the
                # reference's b_ct_functions.hpp:194-196 exchange the two, which only matters in 3D)
                off = [0, 0, 0]
                off[me] = 1
                if act[nxt]:
                    off[nxt] = el % 2
                if act[thd]:
                    off[thd] = el // 2
                lo = [off[a] - (a == me) for a in range(3)]
                hi = [off[a] + (a == me) for a in range(3)]
                v = (0.5 * (at(me, lo) * V + at(me, hi) * V) +
                     1. / 16 * (cf[el][0] * ta + cf[el][1] * tb + cf[el][2] * tc + cf[el][3] * td)) / V
                s = [slice(None)] * 3
                for a in range(3):
                    if act[a]:
                        s[ax[a]] = slice(off[a], None, 2)
                s = tuple(s)
                G[L][me][s] = np.where(inside[s], v, G[L][me][s])
    return G


def expected_face_ghosts(mesh, Bf_blocks, dx_levels):
    """For each block: its face arrays (3, n3, n2, n1) with every ghost face replaced by the level
    arrays' value at its (periodic) position."""
    G = face_level_arrays(mesh, Bf_blocks, dx_levels)
    ndim, ng, nx = mesh.ndim, mesh.ng, mesh.nx
    out = []
    for blk, B in zip(mesh.blocks, Bf_blocks):
        n3, n2, n1 = blk.spec.shape
        tot = mesh._zones_at(blk.level)
        i = (blk.loc[0] * nx[0] + np.arange(n1) - ng) % tot[0]
        j = ((blk.loc[1] * nx[1] + np.arange(n2) - ng) % tot[1]) if ndim > 1 else np.zeros(n2, dtype=int)
        k = ((blk.loc[2] * nx[2] + np.arange(n3) - ng) % tot[2]) if ndim > 2 else np.zeros(n3, dtype=int)
        K, J, I = np.meshgrid(k, j, i, indexing="ij")
        out.append(np.stack([G[blk.level][d][K, J, I] for d in range(3)]))
    return out

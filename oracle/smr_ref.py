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

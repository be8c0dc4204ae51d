"""Test infrastructure (the oracle side of the SMR checks): a CPU restatement of the ghost zones a
static-refined two-level mesh gives each block, built from whole-domain arrays rather than from the
per-zone tables the library executes.

The operators are Parthenon's cell-centred refinement operators (Parthenon, AFD-Illinois fork,
commit unpinned and absent from the reference tree) as published, on a uniform grid:
  * restriction: the average of the 2^ndim fine zones (RestrictCellAverage);
  * prolongation: the coarse value plus, per active direction, +-1/4 times the minmod of the
    left and right coarse differences (ProlongateCellMinMod).
Level-0 values are the coarse blocks' interiors, with the restriction of the fine blocks' interiors
where the domain is refined; level-1 values are the fine interiors, with the prolongation of the
level-0 values elsewhere.  A block's ghost zone at level L takes the level-L value at its (periodic)
position.  Summation orders follow the library's kernels, so the comparison is bitwise.
"""
import numpy as np


def _minmod(a, b):
    return np.where(a * b > 0., np.where(np.abs(a) < np.abs(b), a, b), 0.)


def level_arrays(mesh, P_blocks):
    """Whole-domain primitive arrays (nvar, n3, n2, n1) at level 0 and level 1."""
    ndim, ng, nx = mesh.ndim, mesh.ng, mesh.nx
    nv = P_blocks[0].shape[0]
    t0, t1 = mesh._zones_at(0), mesh._zones_at(1)
    G0 = np.full((nv, t0[2], t0[1], t0[0]), np.nan)
    G1 = np.full((nv, t1[2], t1[1], t1[0]), np.nan)

    def interior(P):
        return P[(slice(None),) + (slice(ng, ng + nx[2]) if ndim > 2 else slice(0, 1),
                                   slice(ng, ng + nx[1]) if ndim > 1 else slice(0, 1),
                                   slice(ng, ng + nx[0]))]

    for blk, P in zip(mesh.blocks, P_blocks):
        sl = tuple(slice(blk.loc[d] * nx[d], (blk.loc[d] + 1) * nx[d]) if d < ndim else slice(0, 1)
                   for d in (2, 1, 0))
        (G0 if blk.level == 0 else G1)[(slice(None),) + sl] = interior(P)
    # restriction of the fine interiors into the level-0 array
    fine = ~np.isnan(G1[0])
    if fine.any():
        f = G1
        q = lambda dk, dj, di: f[:, dk::2, dj::2, di::2] if ndim > 2 else (f[:, :, dj::2, di::2] if ndim > 1 else f[:, :, :, di::2])
        if ndim > 2:
            r = (q(0, 0, 0) + q(0, 0, 1)) + (q(0, 1, 0) + q(0, 1, 1))
            r = r + ((q(1, 0, 0) + q(1, 0, 1)) + (q(1, 1, 0) + q(1, 1, 1)))
            r = r * 0.125
        elif ndim > 1:
            r = ((q(0, 0, 0) + q(0, 0, 1)) + (q(0, 1, 0) + q(0, 1, 1))) * 0.25
        else:
            r = (q(0, 0, 0) + q(0, 0, 1)) * 0.5
        covered = np.isnan(G0)
        G0 = np.where(covered, r, G0)
    # prolongation of the level-0 array where level 1 has no block
    axes = (3, 2, 1)       # x1, x2, x3 along the array axes
    slopes = []
    for d in range(ndim):
        um = np.roll(G0, 1, axis=axes[d])
        up = np.roll(G0, -1, axis=axes[d])
        slopes.append(_minmod(G0 - um, up - G0))
    pro = np.empty_like(G1)
    for ok in range(2 if ndim > 2 else 1):
        for oj in range(2 if ndim > 1 else 1):
            for oi in range(2):
                v = G0.copy()
                for d, o in zip(range(ndim), (oi, oj, ok)):
                    v = v + (0.25 * slopes[d] if o else -0.25 * slopes[d])
                sl = (slice(None), slice(ok, None, 2) if ndim > 2 else slice(None),
                      slice(oj, None, 2) if ndim > 1 else slice(None), slice(oi, None, 2))
                pro[sl] = v
    G1 = np.where(np.isnan(G1), pro, G1)
    return G0, G1


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

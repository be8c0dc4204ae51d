"""Host side of the B_CT SMR mesh (kharma_b200/ctmesh.py, no GPU): the ghost-face and EMF tables, and
the oracle-side restatement of the face exchange (oracle/smr_ref.py).

* Every ghost face of every block is filled once, except the internal faces of the outermost ghost
  layer whose operator would read past the arrays; phases come in order; sources are valid.
* Executing the face table in numpy, with the kernel's operations, gives bitwise the restatement's
  ghost faces on random fields (2D two and three levels, 3D two levels).
* Olivares' prolongation keeps the fine zones divergence-free: the restatement of a divergence-free
  coarse field has zero divergence in every prolongated fine zone (2D and 3D).
* EMF entries pair coarse edges with coinciding fine edges.
"""
import importlib.util
import os

import numpy as np
import pytest

from ctmesh_cases import MESHES, curl_faces_levels, cut, level_dx, random_levels
from kharma_b200 import ctmesh

_spec = importlib.util.spec_from_file_location(
    "smr_ref", os.path.join(os.path.dirname(__file__), "..", "oracle", "smr_ref.py"))
smr_ref = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(smr_ref)


def minmod(a, b):
    return (a if abs(a) < abs(b) else b) if a * b > 0 else 0.


def execute(mesh, Bf, face, ends):
    """The face table executed with the kernel's operations (k_ctm_face), in numpy."""
    n3, n2, n1 = mesh.blocks[0].spec.shape
    st = [1, n1, n1 * n2]
    ndim = mesh.ndim
    B = [b.reshape(3, -1).copy() for b in Bf]
    for e in face:
        db, fd, x, op, sb, y, aux, _ = [int(v) for v in e]
        ta = [a for a in range(ndim) if a != fd]
        if op == ctmesh.FOP_COPY:
            v = B[sb][fd][y]
        elif op == ctmesh.FOP_RESTRICT:
            f = B[sb][fd]
            if len(ta) == 2:
                v = ((f[y] + f[y + st[ta[0]]]) + (f[y + st[ta[1]]] + f[y + st[ta[0]] + st[ta[1]]])) * 0.25
            else:
                v = (f[y] + f[y + st[ta[0]]]) * 0.5
        elif op == ctmesh.FOP_SHARED:
            q = B[sb][fd]
            v = q[y]
            for a in ta:
                sl = minmod(q[y] - q[y - st[a]], q[y + st[a]] - q[y])
                v += 0.25 * sl if (aux >> a) & 1 else -0.25 * sl
        else:
            dx1, dx2, dx3 = mesh.blocks[db].spec.dx
            me, nxt, thd = fd, (fd + 1) % 3, (fd + 2) % 3
            a3 = [(dx2*dx2 - dx3*dx3) / (dx2*dx2 + dx3*dx3), (dx3*dx3 - dx1*dx1) / (dx3*dx3 + dx1*dx1),
                  (dx1*dx1 - dx2*dx2) / (dx1*dx1 + dx2*dx2)]
            cf = [[3 + a3[nxt], 1 - a3[nxt], 3 - a3[thd], 1 + a3[thd]], [3 + a3[nxt], 1 - a3[nxt], 1 + a3[thd], 3 - a3[thd]],
                  [1 - a3[nxt], 3 + a3[nxt], 3 - a3[thd], 1 + a3[thd]], [1 - a3[nxt], 3 + a3[nxt], 1 + a3[thd], 3 - a3[thd]]]
            area = [dx2 * dx3, dx1 * dx3, dx1 * dx2]
            off = [0, 0, 0]
            off[me] = 1
            if nxt < ndim:
                off[nxt] = aux % 2
            if thd < ndim:
                off[thd] = aux // 2
            tgt = y + sum(off[a] * st[a] for a in range(3))
            assert tgt == x

            def term(df, ds, of):
                if df >= ndim:
                    return 0.
                o = st[of] if 0 <= of < ndim else 0
                s = st[ds] if ds < ndim else 0
                F, A, f2 = B[db][df], area[df], 2 * st[df]
                return F[y + f2 + s + o] * A - F[y + s + o] * A - F[y + f2 + o] * A + F[y + o] * A

            V, F, dif = area[me], B[db][me], st[me]
            v = (0.5 * (F[tgt - dif] * V + F[tgt + dif] * V) +
                 1. / 16 * (cf[aux][0] * term(nxt, me, -1) + cf[aux][1] * term(nxt, me, thd) +
                            cf[aux][2] * term(thd, me, -1) + cf[aux][3] * term(thd, me, nxt))) / V
        B[db][fd][x] = v
    return [b.reshape(3, n3, n2, n1) for b in B]


@pytest.mark.parametrize("name", list(MESHES))
def test_face_table_covers_every_ghost_face_once(name):
    mesh = MESHES[name]()
    face, ends, skipped = ctmesh.face_tables(mesh)
    n3, n2, n1 = mesh.blocks[0].spec.shape
    N = n1 * n2 * n3
    key = (face[:, 0].astype(np.int64) * 3 + face[:, 1]) * N + face[:, 2]
    assert len(np.unique(key)) == len(key)
    ng, nx = mesh.ng, mesh.nx
    owned = 0
    for d in range(3):
        per = 1
        for a in range(3):
            if a < mesh.ndim:
                per *= nx[a] + (1 if a == d else 0)
        owned += per
    if all(mesh.periodic):
        assert len(face) + skipped == len(mesh.blocks) * (3 * N - owned)
    else:
        # no entry reaches past a physical domain face
        G = ctmesh._Geo(mesh)
        for e in face[:: max(1, len(face) // 2000)]:
            blk = mesh.blocks[int(e[0])]
            d = int(e[1])
            k, r = divmod(int(e[2]), n1 * n2)
            j, i = divmod(r, n1)
            t = mesh._zones_at(blk.level)
            for a, x in enumerate((i, j, k)):
                if a < mesh.ndim and not mesh.periodic[a]:
                    gg = blk.loc[a] * nx[a] + x - ng
                    assert 0 <= gg <= (t[a] if a == d else t[a] - 1)
    assert np.all(np.diff(face[:, 7]) >= 0) and ends[-1] == len(face)
    assert face[:, 3].min() >= 0 and face[:, 3].max() <= 3
    assert np.all((face[:, 2] >= 0) & (face[:, 2] < N) & (face[:, 5] >= 0) & (face[:, 5] < N))
    # a prolongation into a level-L block reads from level L-1 (shared) or from the block itself
    lev = np.array([b.level for b in mesh.blocks])
    sh = face[face[:, 3] == ctmesh.FOP_SHARED]
    assert np.all(lev[sh[:, 4]] == lev[sh[:, 0]] - 1)
    it = face[face[:, 3] == ctmesh.FOP_INTERNAL]
    assert np.all(it[:, 4] == it[:, 0])


@pytest.mark.parametrize("name", list(MESHES))
def test_executed_table_equals_restatement(name):
    mesh = MESHES[name]()
    face, ends, _ = ctmesh.face_tables(mesh)
    Bf = cut(mesh, random_levels(mesh, 3, seed=5))
    got = execute(mesh, Bf, face, ends)
    exp = smr_ref.expected_face_ghosts(mesh, Bf, level_dx(mesh))
    for e in face:
        db, fd, x = int(e[0]), int(e[1]), int(e[2])
        assert got[db][fd].reshape(-1)[x] == exp[db][fd].reshape(-1)[x], (name, e)


@pytest.mark.parametrize("name", ["2d_two_levels", "3d_two_levels"])
def test_olivares_prolongation_is_divergence_free(name):
    mesh = MESHES[name]()
    F = curl_faces_levels(mesh)
    Bf = cut(mesh, F)
    G = smr_ref.face_level_arrays(mesh, Bf, level_dx(mesh))
    dx = level_dx(mesh)[1]
    nd = mesh.ndim
    ax = (2, 1, 0)
    div = np.zeros(G[1][0].shape)
    for d in range(nd):
        div += (np.roll(G[1][d], -1, axis=ax[d]) - G[1][d]) / dx[d]
    # the level-1 zones the restatement prolongated (outside the level-1 blocks)
    own = mesh._owners(1)
    t = mesh._zones_at(1)
    Z = np.stack(np.meshgrid(np.arange(t[2]), np.arange(t[1]), np.arange(t[0]), indexing="ij"))
    lo = [Z[2] // mesh.nx[0], Z[1] // mesh.nx[1], (Z[0] // mesh.nx[2]) if nd > 2 else np.zeros_like(Z[0])]
    prolongated = own[lo[2], lo[1], lo[0]] < 0
    scale = max(np.abs(g).max() for g in G[1])
    assert prolongated.any()
    assert np.abs(div[prolongated]).max() * min(dx[:nd]) < 1e-13 * scale


@pytest.mark.parametrize("name", list(MESHES))
def test_emf_entries_pair_coinciding_edges(name):
    mesh = MESHES[name]()
    emf = ctmesh.emf_table(mesh)
    assert len(emf)
    lev = np.array([b.level for b in mesh.blocks])
    assert np.all(lev[emf[:, 3]] == lev[emf[:, 0]] + 1)
    n3, n2, n1 = mesh.blocks[0].spec.shape
    ng, nx = mesh.ng, mesh.nx
    for e in emf[:50]:
        cb, ed, cx, fb, fx = [int(v) for v in e[:5]]
        ck, r = divmod(cx, n1 * n2); cj, ci = divmod(r, n1)
        fk, r = divmod(fx, n1 * n2); fj, fi = divmod(r, n1)
        cblk, fblk = mesh.blocks[cb], mesh.blocks[fb]
        # physical position of the edges' lower ends
        for a, (cl, fl) in enumerate(zip((ci, cj, ck), (fi, fj, fk))):
            if a >= mesh.ndim:
                continue
            lo_c = (cblk.spec.x1min, cblk.spec.x2min, cblk.spec.x3min)[a] + (cl - ng) * cblk.spec.dx[a]
            lo_f = (fblk.spec.x1min, fblk.spec.x2min, fblk.spec.x3min)[a] + (fl - ng) * fblk.spec.dx[a]
            assert abs(((lo_c - lo_f) + 0.5) % 1.0 - 0.5) < 1e-12


def test_refined_block_on_a_physical_face_is_rejected():
    from ctmesh_cases import WALLS, base
    from kharma_b200.mesh import SMRMesh
    with pytest.raises(AssertionError, match="physical domain face"):
        SMRMesh(base(2, bc=WALLS), (2, 2, 1), (16, 16, 1), refine=[(0, 0, 0)])
    SMRMesh(base(2, bc=WALLS), (4, 4, 1), (16, 16, 1), refine=[(1, 1, 0)])

"""SMR mesh tables (kharma_b200.mesh), CPU only: every ghost zone of every block gets exactly one
entry, prolongations only feed fine blocks and come after the copies and restrictions, and the flux
correction covers exactly the coarse faces that border refined blocks."""
import dataclasses

import numpy as np
import pytest

from kharma_b200.mesh import OP_COPY, OP_PROLONG, OP_RESTRICT, SMRMesh
from kharma_b200.spec import BlockSpec


def hydro_base(nd):
    return BlockSpec(nx1=8, nx2=8 if nd > 1 else 1, nx3=8 if nd > 2 else 1, x1min=0., x1max=1., x2min=0., x2max=1.,
                     x3min=0., x3max=1., gam=5. / 3., nvar=5, recon="linear_mc")


@pytest.mark.parametrize("nd", [2, 3])
def test_tables_cover_every_ghost_zone_once(nd):
    nx = (8, 8, 8 if nd > 2 else 1)
    nb = (2, 2, 2 if nd > 2 else 1)
    mesh = SMRMesh(hydro_base(nd), nb, nx, refine=[(0, 0, 0)])
    ghost, n_first, flux = mesh.tables()
    assert np.all(ghost[:n_first, 2] != OP_PROLONG) and np.all(ghost[n_first:, 2] == OP_PROLONG)
    for b, blk in enumerate(mesh.blocks):
        n3, n2, n1 = blk.spec.shape
        inside = np.zeros(n3 * n2 * n1, dtype=bool)
        inside.reshape(n3, n2, n1)[blk.spec.interior] = True
        dst = ghost[ghost[:, 0] == b, 1]
        assert len(np.unique(dst)) == len(dst) == (~inside).sum()
        assert not inside[dst].any()
        ops = ghost[ghost[:, 0] == b, 2]
        if blk.level == 0:
            assert not (ops == OP_PROLONG).any()
        else:
            assert not (ops == OP_RESTRICT).any()
    # coarse faces bordering the refined root block: in 2D the two x1 neighbours of (0,0) see it on
    # both of their x1 faces (periodic), likewise the x2 neighbour; 16 faces per block side
    nface = nx[0] * (nx[2] if nd > 2 else 1)
    expect = (3 if nd > 2 else 2) * 2 * nface
    assert len(flux) == expect
    assert set(flux[:, 3]) <= {b for b, blk in enumerate(mesh.blocks) if blk.level == 1}


def three_level(nd, nx=8):
    """4^nd roots; the central 2^nd refined; the central 2^nd of those refined again."""
    c = [(a, b, e) for a in (1, 2) for b in (1, 2) for e in ((1, 2) if nd > 2 else (0,))]
    f = [(1, (a, b, e)) for a in (3, 4) for b in (3, 4) for e in ((3, 4) if nd > 2 else (0,))]
    return SMRMesh(hydro_base(nd) if nx == 8 else dataclasses.replace(hydro_base(nd), nx1=nx),
                   (4, 4, 4 if nd > 2 else 1), (nx, nx, nx if nd > 2 else 1), refine=c + f)


@pytest.mark.parametrize("nd", [2, 3])
def test_three_level_tables(nd):
    mesh = three_level(nd)
    assert mesh.levels == 3
    ghost, n_first, flux = mesh.tables()
    assert np.all(ghost[:n_first, 2] != OP_PROLONG) and np.all(ghost[n_first:, 2] == OP_PROLONG)
    # prolongation phases: the destination level less one, in order
    phase = ghost[n_first:, 5] >> 8
    assert np.all(np.diff(phase) >= 0) and set(phase) == {0, 1}
    level = np.array([blk.level for blk in mesh.blocks])
    assert np.all(level[ghost[n_first:, 0]] == phase + 1)
    assert np.all(level[ghost[n_first:, 3]] == phase)
    for b, blk in enumerate(mesh.blocks):
        n3, n2, n1 = blk.spec.shape
        inside = np.zeros(n3 * n2 * n1, dtype=bool)
        inside.reshape(n3, n2, n1)[blk.spec.interior] = True
        mine = ghost[ghost[:, 0] == b]
        assert len(np.unique(mine[:, 1])) == len(mine) == (~inside).sum()
        src_level = level[mine[:, 3]]
        assert np.all(np.abs(src_level - blk.level) <= 1)
        assert np.all((mine[:, 2] == OP_RESTRICT) == (src_level == blk.level + 1))
        assert np.all((mine[:, 2] == OP_PROLONG) == (src_level == blk.level - 1))
    # flux correction at both coarse-fine interfaces, each fine face block one level up
    assert set(level[flux[:, 0]]) == {0, 1}
    assert np.all(level[flux[:, 3]] == level[flux[:, 0]] + 1)
    # every coarse face on a fine-coarse boundary once: 2^nd refined blocks' surfaces, per interface
    per_face = 8 ** (nd - 1)
    ring = 2 * nd * 2 ** (nd - 1)            # coarse faces (block faces) around a 2^nd patch
    assert len(flux) == 2 * ring * per_face


def test_unbalanced_mesh_is_rejected():
    # a level-2 patch touching level-0 blocks
    mesh = SMRMesh(hydro_base(2), (2, 2, 1), (8, 8, 1), refine=[(0, 0, 0), (1, (0, 0, 0))])
    with pytest.raises(AssertionError, match="2:1"):
        mesh.tables()


def test_transmitting_poles_mesh():
    """Transmitting x2 faces: root blocks spanning all of a periodic x3 keep them (x3 periodic on
    the block itself); refined blocks are kept off the poles; split x3 roots are rejected."""
    import numpy as np
    from kharma_b200.spec import bondi_spec
    bc = ("outflow", "outflow", "transmitting", "transmitting", "periodic", "periodic")
    base = bondi_spec(16, 16, 16, float(np.log(3.0)), float(np.log(30.0)), 0.0, 1.0, 0.0, 2 * np.pi, bc=bc)
    mesh = SMRMesh(base, (4, 4, 1), (16, 16, 16), refine=[(1, 1, 0)])
    polar = [b for b in mesh.blocks if b.level == 0 and b.loc[1] in (0, 3)]
    assert polar and all(b.spec.bc[4:] == ("periodic", "periodic") for b in polar)
    assert all(("transmitting" in b.spec.bc[2:4]) == (b.loc[1] in (0, 3)) for b in mesh.blocks if b.level == 0)
    assert all(b.spec.bc[4:] == ("exchange", "exchange") for b in mesh.blocks if b.level == 1)
    with pytest.raises(AssertionError):
        SMRMesh(base, (4, 4, 1), (16, 16, 16), refine=[(1, 0, 0)])
    with pytest.raises(AssertionError):
        SMRMesh(base, (4, 4, 2), (16, 16, 16))

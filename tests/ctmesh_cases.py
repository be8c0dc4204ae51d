"""Shared inputs of the B_CT SMR tests: meshes and random fields; block arrays are cut from
whole-domain level arrays (kharma_b200.ctmesh) so that faces two blocks share agree bit for bit."""
import dataclasses

import numpy as np

from kharma_b200.ctmesh import curl_faces_levels, cut, fluid_levels, level_dx  # noqa: F401  (re-exported)
from kharma_b200.mesh import SMRMesh
from kharma_b200.spec import BlockSpec


def base(nd, nx=16, b_ct="gs05_c", bc=("periodic",) * 6):
    return BlockSpec(nx1=nx, nx2=nx, nx3=nx if nd > 2 else 1, x1min=0., x1max=1., x2min=0., x2max=1., x3min=0.,
                     x3max=1., gam=4. / 3., nvar=8, recon="linear_mc", riemann="llf", cfl=0.8, dt_min=1e-4,
                     b_ct=b_ct, driver="kharma", bc=bc)


WALLS = ("reflecting", "reflecting", "reflecting", "reflecting", "periodic", "periodic")
OPEN = ("outflow", "outflow", "reflecting", "reflecting", "periodic", "periodic")


REFINE_2D = [(1, 1, 0), (1, 2, 0), (2, 1, 0), (2, 2, 0)]
MESHES = {
    # 4x4 root blocks of 16^2, the central 2x2 refined
    "2d_two_levels": lambda: SMRMesh(base(2), (4, 4, 1), (16, 16, 1), refine=REFINE_2D),
    # the central 2x2 of the refined blocks refined again
    "2d_three_levels": lambda: SMRMesh(base(2), (4, 4, 1), (16, 16, 1),
                                       refine=REFINE_2D + [(1, (3, 3, 0)), (1, (4, 3, 0)), (1, (3, 4, 0)),
                                                           (1, (4, 4, 0))]),
    # 2x2x2 root blocks of 8^3, one refined
    "3d_two_levels": lambda: SMRMesh(base(3, nx=8), (2, 2, 2), (8, 8, 8), refine=[(1, 1, 1)]),
    # reflecting walls on the x1 and x2 domain faces, the central 2x2 of 4x4 roots refined
    "2d_two_levels_walls": lambda: SMRMesh(base(2, bc=WALLS), (4, 4, 1), (16, 16, 1), refine=REFINE_2D),
}


def random_levels(mesh, nvar, seed, positive=False):
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for L in range(mesh.levels):
        t = mesh._zones_at(L)
        a = rng.uniform(-1.0, 1.0, size=(nvar, t[2], t[1], t[0]))
        if positive:
            a[0] = 1.0 + 0.5 * a[0]
            a[1] = 1.0 + 0.5 * a[1]
            a[2:5] *= 0.1
        out.append(a)
    return out

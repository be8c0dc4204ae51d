"""Shared inputs of the B_CT SMR tests: meshes, and block arrays cut from whole-domain level arrays so
that faces two blocks share agree bit for bit."""
import dataclasses

import numpy as np

from kharma_b200.mesh import SMRMesh
from kharma_b200.spec import BlockSpec


def base(nd, nx=16, b_ct="gs05_c"):
    return BlockSpec(nx1=nx, nx2=nx, nx3=nx if nd > 2 else 1, x1min=0., x1max=1., x2min=0., x2max=1., x3min=0.,
                     x3max=1., gam=4. / 3., nvar=8, recon="linear_mc", riemann="llf", cfl=0.8, dt_min=1e-4,
                     b_ct=b_ct, driver="kharma")


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
}


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


def curl_faces_levels(mesh, B0=(1.0, 0.5, 0.25), amp=0.05):
    """Whole-domain face arrays (3, t3, t2, t1) per level: B0 plus the discrete curl of
    A = amp (sin(2 pi x2) cos(2 pi x3), sin(2 pi x3) cos(2 pi x1), sin(2 pi x1) cos(2 pi x2)) sampled at
    each level's edges from integer corner indices, so that every level's field is divergence-free to
    rounding and a coarse face equals the mean of the fine faces on it to rounding."""
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
        A3 = amp * np.sin(2 * np.pi * X1) * np.cos(2 * np.pi * X2)                      # at (i f, j f, k c)
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

"""Poisoned conserved states for the inversion-failure tests (host side, numpy).

Each poison rewrites the conserved variables of chosen zones so that the inversion of those zones
fails (or, for the Kastaun inverter, is floored inside the inverter):
  neg_D         D = rho u^t sqrt(-g) made negative         1D_W: neg_input (onedw.hpp:99-101)
  nan_UU        the energy T^t_t + D set to NaN             never converges: max_iter
  hot           D x 1e-2, energy x 1e2 (finite)             1D_W exhausts its 8 iterations: max_iter
  superluminal  T^t_i set to 100 (|D| + |energy|)            no physical Lorentz factor: bad_ut, or
                                                            max_iter where the secant stalls first
Sites: an isolated interior zone, a zone on the inner X1 face, a zone on the periodic x3 edge (its
neighbours wrap), a pair of adjacent zones and a 3x3x3 cluster whose centre has no good neighbour
(FixUtoP's atmosphere branch, fixup.cpp:121-124).
"""
import numpy as np


def _scale(f):
    f = np.array(f, dtype=np.float64)
    return lambda u: u * f


def _superluminal(u):
    u = u.copy()
    u[2:5] = 100.0 * (abs(u[0]) + abs(u[1]))
    return u


POISONS = {
    "neg_D": _scale([-1.0, 1, 1, 1, 1, 1, 1, 1]),
    "nan_UU": _scale([1.0, np.nan, 1, 1, 1, 1, 1, 1]),
    "hot": _scale([1e-2, 1e2, 1, 1, 1, 1, 1, 1]),
    "superluminal": _superluminal,
}


def sites(spec):
    """(name, list of (k, j, i)) of the poisoned zones of a 3D block (interior indices)."""
    ng = spec.ng
    ks, js, is_ = ng, ng, ng
    ke, je, ie = ng + spec.nx3 - 1, ng + spec.nx2 - 1, ng + spec.nx1 - 1
    kc, jc, ic = (ks + ke) // 2, (js + je) // 2, (is_ + ie) // 2
    cluster = [(kc + a, jc - 6 + b, ic + 6 + c) for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1)]
    return [
        ("isolated", [(kc, jc, ic)]),
        ("x1_face", [(kc, jc + 3, is_)]),
        ("x3_edge", [(ks, jc - 3, ic - 5)]),
        ("pair", [(kc, jc + 5, ic - 3), (kc, jc + 5, ic - 2)]),
        ("cluster", cluster),
    ]


def poison(U, spec, kinds=None):
    """Poison U (nvar, n3, n2, n1) in place: each site gets the next poison kind in turn (the cluster
    all one kind).  Returns the list of poisoned (k, j, i)."""
    kinds = list(POISONS) if kinds is None else list(kinds)
    out = []
    for n, (_, zs) in enumerate(sites(spec)):
        f = POISONS[kinds[n % len(kinds)]]
        for z in zs:
            U[(slice(0, 8),) + z] = f(U[(slice(0, 8),) + z])
            out.append(z)
    return out

"""The Bondi static-refined layout of the batching form and the Bondi initial state (CPU only).

Layout: 8 blocks of 64^3, 48 of 32^3, 128 of 16^3 on three levels whose zone widths halve per level;
within a level blocks tile their region without overlap.  Bondi: the analytic solution of
prob/bondi.hpp (sonic point r_s = 8, mdot = 1, gamma = 5/3), and a block whose ghost zones hold it
stays at the steady state under the oracle's step.
"""
import math

import numpy as np

from kharma_b200 import problems
from kharma_b200.batch import bondi_smr_layout
from kharma_b200.spec import bondi_spec


def test_layout_counts_sizes_and_refinement():
    specs = bondi_smr_layout()
    assert len(specs) == 184
    by = {}
    for s in specs:
        by.setdefault(s.nx1, []).append(s)
        assert s.nx1 == s.nx2 == s.nx3 and s.nvar == 5 and s.bc == ("exchange",) * 6
    assert {k: len(v) for k, v in by.items()} == {64: 8, 32: 48, 16: 128}
    assert sum(s.nx1 * s.nx2 * s.nx3 for s in specs) == 4194304
    dx = {k: v[0].dx for k, v in by.items()}
    for a, b in ((64, 32), (32, 16)):
        for x in range(3):
            assert math.isclose(dx[a][x], 2 * dx[b][x], rel_tol=1e-12)
    # no two blocks of a level overlap
    for lvl in by.values():
        boxes = [(s.x1min, s.x1max, s.x2min, s.x2max, s.x3min, s.x3max) for s in lvl]
        for i in range(len(boxes)):
            for j in range(i + 1, len(boxes)):
                a, b = boxes[i], boxes[j]
                overlap = all(min(a[2 * d + 1], b[2 * d + 1]) - max(a[2 * d], b[2 * d]) > 1e-12 for d in range(3))
                assert not overlap
    # radial shells: level 2 at r_in, level 0 reaching r_out
    assert math.isclose(min(s.x1min for s in by[16]), math.log(3.0))
    assert math.isclose(max(s.x1max for s in by[64]), math.log(30.0))


def test_bondi_solution_sonic_point():
    # at the sonic radius u^r = -sqrt(1 / (2 r_s)) (bondi.hpp: uc); the two solution branches cross
    # there, which limits the bisection to about 1e-7
    rho, u, ur = problems.bondi_solution(np.array([8.0]), rs=8.0, mdot=1.0, gam=5.0 / 3.0)
    assert math.isclose(ur[0], -math.sqrt(1 / 16.0), rel_tol=1e-6)
    # the accretion rate 4 pi r^2 rho u^r is -mdot at every radius
    r = np.array([3.0, 5.0, 8.0, 13.0, 30.0])
    rho, u, ur = problems.bondi_solution(r)
    assert np.allclose(4 * math.pi * r * r * rho * ur, -1.0, rtol=1e-9)


def test_bondi_block_stays_steady_under_the_oracle(oracle_mod):
    sp = bondi_spec(12, 12, 12, math.log(3.0), math.log(3.0) + 0.25, 0.375, 0.5, 0.0, math.pi / 8)
    o = oracle_mod.Oracle(sp)
    P0 = problems.bondi(sp, o.geometry())
    P, U = o.init_state(P0)
    for _ in range(4):
        pflag, _, _, _ = o.step(P, U, 2e-3)
    assert not (pflag > 0).any()
    sl = sp.interior
    for v in range(2):
        assert np.max(np.abs(P[v][sl] - P0[v][sl])) / np.max(np.abs(P0[v][sl])) < 1e-6

"""The oracle's inversion-failure path on poisoned states (CPU): the statuses the reference's 1D_W
returns (invert_template.hpp:53, onedw.hpp:99-101, 196-208) and FixUtoP's neighbour average and
atmosphere fallback (fixup.cpp:47-156), checked against a numpy restatement of the average."""
import numpy as np

from kharma_b200 import problems
from kharma_b200.spec import torus_spec

import poison_cases as pc

NEG_INPUT, MAX_ITER, BAD_UT = 1, 2, 3


def state(orc, **kw):
    spec = torus_spec(32, 24, 8, **kw)
    o = orc.Oracle(spec)
    P0 = problems.fm_torus(spec, o.geometry(), seed=7)
    Po, Uo = o.init_state(P0)
    return spec, o, Po, Uo


def test_onedw_statuses(oracle_mod):
    spec, o, Po, Uo = state(oracle_mod)
    expect = {"neg_D": {NEG_INPUT}, "nan_UU": {MAX_ITER}, "hot": {MAX_ITER}, "superluminal": {BAD_UT, MAX_ITER}}
    for kind, status in expect.items():
        U = Uo.copy()
        P = Po.copy()
        zs = pc.poison(U, spec, kinds=[kind])
        pflag, fflag = o.utop(U, P)
        for z in zs:
            assert int(pflag[z]) in status, (kind, z, pflag[z])
        # the zones not poisoned invert
        mask = np.zeros(spec.shape, bool)
        for z in zs:
            mask[z] = True
        assert np.all(pflag[spec.interior][~mask[spec.interior]] == 0)
        # P is left as the guess where the inversion failed (onedw.hpp:196-208 write only on success)
        for z in zs:
            assert np.array_equal(P[(slice(0, 5),) + z], Po[(slice(0, 5),) + z])


def test_fixup_average_and_atmosphere(oracle_mod):
    spec, o, Po, Uo = state(oracle_mod)
    U = Uo.copy()
    P = Po.copy()
    pc.poison(U, spec)
    pflag, fflag = o.utop(U, P)
    o.floors(P, U, pflag, fflag)
    P_before = P.copy()
    fail = pflag > 0
    assert np.count_nonzero(fail[spec.interior]) >= 30
    o.fix_utop(P, U, pflag)
    assert np.all(np.isfinite(P[:, spec.interior[0], spec.interior[1], spec.interior[2]]))
    # an isolated failed zone: the 1/(Manhattan distance + 1) weighted average of its 26 good
    # neighbours, then the geometric floors (it sits in the torus, above them)
    k, j, i = pc.sites(spec)[0][1][0]
    w = np.zeros((3, 3, 3))
    for a in (-1, 0, 1):
        for b in (-1, 0, 1):
            for c in (-1, 0, 1):
                w[a + 1, b + 1, c + 1] = 0.0 if fail[k + a, j + b, i + c] else 1.0 / (abs(a) + abs(b) + abs(c) + 1)
    avg = np.array([np.sum(w * P_before[p, k - 1:k + 2, j - 1:j + 2, i - 1:i + 2]) / np.sum(w) for p in range(5)])
    np.testing.assert_allclose(P[:5, k, j, i], avg, rtol=1e-13)
    # the centre of the 3x3x3 cluster has no good neighbour: atmosphere (zero velocity, floors)
    kc, jc, ic = pc.sites(spec)[4][1][13]
    assert np.all(P[2:5, kc, jc, ic] == 0.0)
    assert P[0, kc, jc, ic] > 0 and P[1, kc, jc, ic] > 0
    # U follows P in every fixed zone (lock step)
    U2 = o.ptou(P)
    for z in zip(*np.nonzero(fail)):
        if all(s.start <= x < s.stop for s, x in zip(spec.interior, z)):
            np.testing.assert_allclose(U[(slice(0, 5),) + z], U2[(slice(0, 5),) + z], rtol=1e-14, atol=0)


def test_fixup_off_leaves_guess(oracle_mod):
    """With fix_average_neighbors and fix_atmosphere both false FixUtoP does nothing (fixup.cpp:52-55)."""
    spec, o, Po, Uo = state(oracle_mod)
    spec.fix_average_neighbors = False
    spec.fix_atmosphere = False
    o = oracle_mod.Oracle(spec)
    U = Uo.copy()
    P = Po.copy()
    pc.poison(U, spec)
    pflag, fflag = o.utop(U, P)
    P1, U1 = P.copy(), U.copy()
    o.fix_utop(P, U, pflag)
    sl = spec.interior
    assert np.array_equal(P[(slice(None),) + sl], P1[(slice(None),) + sl])


def test_step_with_poisoned_state_recovers(oracle_mod):
    """A step from a poisoned U_0 fails in both stages at the poisoned zones, and FixUtoP plus the
    lock-step P->U leave a finite state; Kastaun floors neg_D/hot/superluminal inside the inverter and
    fails only on NaN."""
    for inv, must_fail in (("onedw", ["neg_D", "nan_UU", "hot", "superluminal"]), ("kastaun", ["nan_UU"])):
        spec, o, Po, Uo = state(oracle_mod, inverter=inv)
        U = Uo.copy()
        P = Po.copy()
        pc.poison(U, spec)
        pf, ff, dtn, mn = o.step(P, U, spec.dt_min)
        sl = spec.interior
        assert np.count_nonzero(pf[sl] > 0) > 0, inv
        assert np.all(np.isfinite(P)) and np.all(np.isfinite(U))
        assert np.isfinite(dtn)
        for n, (name, zs) in enumerate(pc.sites(spec)):
            kind = list(pc.POISONS)[n % len(pc.POISONS)]
            if kind in must_fail and name != "cluster":
                assert all(pf[z] > 0 for z in zs), (inv, name, kind)

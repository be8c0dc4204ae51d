"""The oracle's EMHD and implicit-solve restatement on CPU: pinned by the reference's own
conducting-atmosphere profile check, checked for self-consistency (exact vs finite-difference
Jacobian, dense solves vs numpy) and for Newton convergence.  No GPU."""
import numpy as np
import pytest

from emhd_cases import EMHD_VARIANTS, atmosphere_case, implicit, profile, source
from kharma_b200.spec import atmosphere_spec


@pytest.mark.parametrize("n1", [64, 128])
def test_atmosphere_profile_matches_grid(oracle_mod, n1):
    # conducting_atmosphere.cpp:139-152 aborts unless every rCoords row is within 1e-10 of the grid r
    spec = atmosphere_spec(n1, 4, 1)
    r = oracle_mod.Oracle(spec).geometry()["r_center"]
    prof = profile(n1)
    assert len(prof["rCoords"]) == n1 + 8
    assert np.max(np.abs(r[:, :] - prof["rCoords"][None, :])) < 1e-10


def test_qr_solve_matches_numpy(oracle_mod):
    rng = np.random.Generator(np.random.PCG64(3))
    for n in (5, 6, 7):
        for _ in range(20):
            A = rng.normal(size=(n, n)) + n * np.eye(n) * rng.uniform(0.1, 2)
            A[:, rng.integers(n)] *= 1e3          # badly scaled column, exercises the pivoting
            b = rng.normal(size=n)
            x = oracle_mod.dense_solve(A, b, use_qr=True)
            ref = np.linalg.solve(A, b)
            assert np.allclose(x, ref, rtol=1e-10, atol=1e-12 * np.abs(ref).max())


def test_lu_path_is_upper_solve_only(oracle_mod):
    # implicit.cpp:387-401 factorises without pivoting and then solves with U alone
    rng = np.random.Generator(np.random.PCG64(4))
    n = 7
    A = rng.normal(size=(n, n)) + 5 * np.eye(n)
    b = rng.normal(size=n)
    U = A.copy()
    for p in range(n):
        U[p, p] += 1e-20 if U[p, p] >= 0 else -1e-20
        for r in range(p + 1, n):
            U[r, p] /= U[p, p]
            U[r, p + 1:] -= U[r, p] * U[p, p + 1:]
    ref = np.linalg.solve(np.triu(U), b)
    x = oracle_mod.dense_solve(A, b, use_qr=False)
    assert np.allclose(x, ref, rtol=1e-12, atol=1e-14)


def _case(oracle_mod, variant, n1=64, n2=6, n3=1):
    spec, emhd, P, dt, xi = atmosphere_case(n1, n2, n3, EMHD_VARIANTS[variant])
    o = oracle_mod.Oracle(spec)
    U = o.emhd_ptou(emhd, P)
    S_e = o.zeros10()
    o.emhd_add_source(emhd, P, S_e)
    S = source(U, S_e, xi, dt)
    return spec, emhd, o, P, U, S, dt


@pytest.mark.parametrize("variant", ["kappa_eta_ho", "constant", "soundspeed_q_only", "dp_only", "grmhd_only"])
def test_exact_jacobian_matches_central_differences(oracle_mod, variant):
    spec, emhd, o, P, U, S, dt = _case(oracle_mod, variant)
    Psol = P.copy()
    Psol[[0, 1]] *= 1.002                                 # away from the initial state
    J, r = o.implicit_jacobian(emhd, implicit("exact"), P, U, P, S, Psol, dt)
    nf = emhd.nfvar
    slots = [0, 1, 2, 3, 4] + ([8] if emhd.conduction else []) + ([9] if emhd.viscosity else [])
    sl = spec.interior
    Jc = np.zeros((nf, nf) + P.shape[1:])
    for col, s in enumerate(slots):
        h = 1e-6 * np.maximum(np.abs(Psol[s]), 1e-3)
        Pp, Pm = Psol.copy(), Psol.copy()
        Pp[s] += h
        Pm[s] -= h
        rp = o.implicit_residual(emhd, P, U, P, S, Pp, dt)
        rm = o.implicit_residual(emhd, P, U, P, S, Pm, dt)
        Jc[:, col] = (rp - rm) / (2 * h)
    Je = J.reshape((nf, nf) + P.shape[1:])
    for row in range(nf):
        scale = np.abs(Je[row][(slice(None),) + sl]).max(axis=0) + 1e-300
        err = np.abs(Je[row][(slice(None),) + sl] - Jc[row][(slice(None),) + sl]).max(axis=0) / scale
        assert err.max() < 1e-6, (row, err.max())


@pytest.mark.parametrize("variant", ["kappa_eta_ho", "constant", "grmhd_only"])
def test_fd_jacobian_residual_equals_exact_residual(oracle_mod, variant):
    spec, emhd, o, P, U, S, dt = _case(oracle_mod, variant)
    Jf, rf = o.implicit_jacobian(emhd, implicit("fd"), P, U, P, S, P, dt)
    Je, re = o.implicit_jacobian(emhd, implicit("exact"), P, U, P, S, P, dt)
    assert np.array_equal(rf, re)          # the dual evaluation's value part is the plain residual
    sl = (slice(None),) + spec.interior
    assert np.abs(Jf[sl] - Je[sl]).max() <= 1e-4 * np.abs(Je[sl]).max()


@pytest.mark.parametrize("variant", ["kappa_eta_ho", "constant", "soundspeed_q_only"])
def test_newton_converges_with_either_jacobian(oracle_mod, variant):
    spec, emhd, o, P, U, S, dt = _case(oracle_mod, variant)
    sl = (slice(None),) + spec.interior
    # The residual is absolute and scales with |U|/dt (~1e9 here: sqrt(-g) ~ r^3); round-off bounds
    # it near 1e-16 of that, so the tolerance is set relative to it.
    tol = 1e-12 * np.abs(U[sl]).max() / dt
    out = {}
    for jac in ("fd", "exact"):
        Psol = P.copy()
        norm = np.zeros(spec.shape)
        fail = np.zeros(spec.shape)
        it, mx = o.implicit_step(emhd, implicit(jac, rootfind_tol=tol), P, U, P, S, Psol, norm, fail, dt)
        out[jac] = (it, mx, Psol)
        assert mx[-1] < tol, (jac, mx)
        assert np.all(fail[spec.interior] != 1)
        r = o.implicit_residual(emhd, P, U, P, S, Psol, dt)
        assert np.abs(r[sl]).max() < tol
    # both reach the same root; iteration counts agree within one (the first steps are limited by the
    # residual's curvature, not by the 1e-8 error of the forward-difference Jacobian)
    assert abs(out["exact"][0] - out["fd"][0]) <= 1
    d = np.abs(out["exact"][2] - out["fd"][2])[sl].max() / np.abs(P[sl]).max()
    assert d < 1e-10


def test_backtracking_failure_and_fix_solve(oracle_mod):
    spec, emhd, o, P, U, S, dt = _case(oracle_mod, "kappa_eta_ho")
    sl = spec.interior
    k, j = sl[0].start, sl[1].start + 2
    bad = [(k, j, sl[2].start + 5), (k, j + 1, sl[2].start + 17)]
    for z in bad:
        S[(0,) + z] = -50.0 * U[(0,) + z] / dt          # asks for rho to drop far below zero
    Psol = P.copy()
    norm = np.zeros(spec.shape)
    fail = np.zeros(spec.shape)
    o.implicit_step(emhd, implicit("fd", max_nonlinear_iter=3), P, U, P, S, Psol, norm, fail, dt)
    for z in bad:
        assert fail[z] == 1
        for s in (0, 1, 2, 3, 4, 8, 9):
            assert Psol[(s,) + z] == P[(s,) + z]        # reset to the sub-step state
    assert np.count_nonzero(fail == 1) == len(bad)
    # FixSolve: distance-weighted average of the good neighbours (fix_solve.cpp:70-107)
    Pfix, Ufix = Psol.copy(), o.emhd_ptou(emhd, Psol)
    o.fix_solve(emhd, Pfix, Ufix, fail)
    for z in bad:
        kk, jj, ii = z
        wsum, acc = 0.0, np.zeros(10)
        for n in (-1, 0, 1):
            for m in (-1, 0, 1):
                for l in (-1, 0, 1):
                    zz = (kk + n, jj + m, ii + l)
                    if not (0 <= zz[0] < spec.shape[0] and 0 <= zz[1] < spec.shape[1] and 0 <= zz[2] < spec.shape[2]):
                        continue
                    if fail[zz] == 1:
                        continue
                    w = 1.0 / (abs(l) + abs(m) + abs(n) + 1)
                    wsum += w
                    acc += w * Psol[(slice(None),) + zz]
        for s in (0, 1, 2, 3, 4, 8, 9):
            assert Pfix[(s,) + z] == pytest.approx(acc[s] / wsum, rel=1e-14, abs=1e-300)
        for s in (5, 6, 7):
            assert Pfix[(s,) + z] == Psol[(s,) + z]
    Uref = o.emhd_ptou(emhd, Pfix)
    for z in bad:
        assert np.array_equal(Ufix[(slice(None),) + z], Uref[(slice(None),) + z])


def test_imex_keeps_conducting_atmosphere_in_equilibrium(oracle_mod):
    """The reference's conducting atmosphere (tests/conducting_atmosphere) is a steady state of the
    EMHD equations: its ODE profile (heat flux phi included) balances the explicit fluxes, the
    geometric source with the EMHD stress tensor, and the implicit q relaxation.  Ten vl2 ImEx steps
    of the oracle (imex_step.cpp:58-356) must leave rho, u and q~ within 1e-4 of the profile."""
    import dataclasses
    from emhd_cases import EMHD_VARIANTS, implicit, profile
    from kharma_b200 import problems
    from kharma_b200.block import build_geometry
    from kharma_b200.spec import atmosphere_spec
    n1 = 64
    spec = dataclasses.replace(atmosphere_spec(n1, 8, 1), bc=("exchange",) * 4 + ("periodic",) * 2)
    emhd = EMHD_VARIANTS["kappa_eta_ho"]
    P = problems.conducting_atmosphere(spec, build_geometry(spec), emhd, profile(n1), jitter=0.0)
    o = oracle_mod.Oracle(spec)
    U = o.emhd_ptou(emhd, P)
    imp = implicit("fd", max_nonlinear_iter=3, rootfind_tol=1e-12)
    sn, sf = np.zeros(spec.shape), np.zeros(spec.shape)
    P0 = P.copy()
    for _ in range(10):
        P1, U1, _, _ = o.imex_stage(emhd, imp, 1, 0.5, P, U, P, U, sn, sf)
        P, U, _, _ = o.imex_stage(emhd, imp, 2, 0.5, P, U, P1, U1, sn, sf)
    sl = spec.interior
    assert not (sf[sl] == 1).any()
    for v in (0, 1, 8):
        assert np.max(np.abs(P[v][sl] - P0[v][sl])) / np.max(np.abs(P0[v][sl])) < 1e-4, v


@pytest.mark.parametrize("name", ["constant", "kappa_eta_ho"])
def test_imex_stage_floors_limits_and_physical_faces(oracle_mod, name):
    """An ImEx stage on a block with physical faces, floors and the EMHD stability limits
    (imex_step.cpp:269-298, emhd_limits.hpp:55-130): the limit bits are all hit, a zone the heat-flux
    limit scaled holds |q| = 1.07 rho cs^3 (constant closure: q = q~), and the ghost zones of q~ / dP~
    copy the boundary zones (outflow X1) or their mirror images (reflecting X2) without a sign change."""
    import dataclasses
    from emhd_cases import atmosphere_limits_case
    spec, emhd, P = atmosphere_limits_case(name)
    o = oracle_mod.Oracle(spec)
    U = o.emhd_ptou(emhd, P)
    imp = implicit("fd", max_nonlinear_iter=3, rootfind_tol=1e-12)
    sn, sf = np.zeros(spec.shape), np.zeros(spec.shape)
    Pout, Uout, _, _, ff, ef = o.imex_stage_flags(emhd, imp, 1, 0.5, P, U, P, U, sn, sf)
    sl = spec.interior
    ef_i, ff_i = ef[sl].astype(int), ff[sl].astype(int)
    assert (ef_i & 1).any() and (ef_i & 2).any() and (ef_i & 4).any()
    assert ff_i.any() and not ff_i.all()
    assert np.isfinite(Pout).all() and np.isfinite(Uout).all()
    ok = sf[sl] != 1          # zones FixSolve left alone
    gam = spec.gam

    def qmax(Q):
        rho, u = Q[0][sl], Q[1][sl]
        return 1.07 * rho * np.sqrt(gam * (gam - 1.) * u / (rho + gam * u)) ** 3

    if name == "constant":
        hit = ((ef_i & 1) != 0) & ok
        assert hit.any()
        np.testing.assert_allclose(np.abs(Pout[8][sl][hit]), qmax(Pout)[hit], rtol=1e-12)
        assert np.all(np.abs(Pout[8][sl][ok]) <= qmax(Pout)[ok] * (1 + 1e-12))
    # the same stage without the limits leaves the flags clear (and, constant closure, the bound broken)
    free = dataclasses.replace(emhd, stability_limits=False)
    sn2, sf2 = np.zeros(spec.shape), np.zeros(spec.shape)
    Pfree, _, _, _, _, ef2 = o.imex_stage_flags(free, imp, 1, 0.5, P, U, P, U, sn2, sf2)
    assert not ef2.any()
    if name == "constant":
        assert np.any(np.abs(Pfree[8][sl]) > qmax(Pfree) * (1 + 1e-6))
    # ghost zones of the scalar slots (2D block: one k plane)
    ng = spec.ng
    js, je, is_, ie = ng, ng + spec.nx2 - 1, ng, ng + spec.nx1 - 1
    for s in (8, 9):
        A = Pout[s][0]
        for g in range(ng):
            np.testing.assert_array_equal(A[js:je + 1, g], A[js:je + 1, is_])
            np.testing.assert_array_equal(A[js:je + 1, ie + 1 + g], A[js:je + 1, ie])
            np.testing.assert_array_equal(A[g, is_:ie + 1], A[2 * js - 1 - g, is_:ie + 1])
            np.testing.assert_array_equal(A[je + 1 + g, is_:ie + 1], A[je - g, is_:ie + 1])

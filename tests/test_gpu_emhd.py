"""EMHD sources and the implicit Newton solve on the GPU against the oracle.

With the reference's forward-difference Jacobian every output (primitives, solve_norm, solve_fail,
iteration count and per-iteration maximum norms) must agree bit for bit: the kernels are compiled
without FMA contraction in the reference's evaluation order.  The exact-Jacobian form is compared
with the oracle's dual-number Jacobian to 1e-12 relative (Jacobian) and 1e-11 (converged iterates).  The torus closure calls exp, whose CUDA
and glibc results differ in the last bits, so it is compared to 1e-12 relative.
"""
import numpy as np
import pytest
import torch

from emhd_cases import EMHD_VARIANTS, atmosphere_case, implicit, source
from kharma_b200.block import Block
from kharma_b200.emhd import ImplicitSolver

pytestmark = pytest.mark.gpu

SLOTS = {True: [8], False: []}


def setup(oracle_mod, variant, shape=(64, 6, 1)):
    spec, emhd, P, dt, xi = atmosphere_case(*shape, emhd=EMHD_VARIANTS[variant])
    o = oracle_mod.Oracle(spec)
    b = Block(spec, geometry=o.geometry())
    sol = ImplicitSolver(b, emhd, conn=o.connection())
    U = o.emhd_ptou(emhd, P)
    S_e = o.zeros10()
    o.emhd_add_source(emhd, P, S_e)
    S = source(U, S_e, xi, dt)
    return spec, emhd, o, b, sol, P, U, S_e, S, dt


def dev(a):
    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def slots(emhd):
    return [0, 1, 2, 3, 4, 5, 6, 7] + ([8] if emhd.conduction else []) + ([9] if emhd.viscosity else [])


def rel_err(a, b):
    scale = np.abs(b).max() + 1e-300
    return np.abs(a - b).max() / scale


SHAPES = {"2d": (64, 6, 1), "3d": (64, 4, 4)}


@pytest.mark.parametrize("shape", ["2d", "3d"])
@pytest.mark.parametrize("variant", ["kappa_eta_ho", "constant", "soundspeed_q_only", "dp_only", "grmhd_only"])
def test_emhd_ptou_and_explicit_sources_bitwise(oracle_mod, variant, shape):
    spec, emhd, o, b, sol, P, U, S_e, S, dt = setup(oracle_mod, variant, SHAPES[shape])
    Pd = dev(P)
    Ud = sol.ptou(Pd)
    Sd = torch.zeros_like(Pd)
    sol.add_source(Pd, Sd)
    torch.cuda.synchronize()
    for s in slots(emhd):
        assert np.array_equal(Ud[s].cpu().numpy(), U[s]), f"U slot {s}"
    assert np.array_equal(Sd.cpu().numpy(), S_e), "explicit EMHD sources differ"


@pytest.mark.parametrize("variant", ["kappa_eta_ho", "constant", "soundspeed_q_only", "dp_only", "grmhd_only"])
def test_jacobian_fd_bitwise_and_exact_close(oracle_mod, variant):
    spec, emhd, o, b, sol, P, U, S_e, S, dt = setup(oracle_mod, variant)
    Psol = P.copy()
    Psol[[0, 1]] *= 1.002
    sl = (slice(None),) + spec.interior
    for jac in ("fd", "exact"):
        sol.set_implicit(implicit(jac))
        Jd, rd = sol.jacobian(dev(P), dev(U), dev(P), dev(S), dev(Psol), dt)
        Jo, ro = o.implicit_jacobian(emhd, implicit(jac), P, U, P, S, Psol, dt)
        torch.cuda.synchronize()
        Jd, rd = Jd.cpu().numpy(), rd.cpu().numpy()
        assert np.array_equal(rd[sl], ro[sl]), f"{jac}: residual differs"
        if jac == "fd":
            assert np.array_equal(Jd[sl], Jo[sl]), "forward-difference Jacobian differs"
        else:
            nf = emhd.nfvar
            for row in range(nf):
                a = Jd[row * nf:(row + 1) * nf][sl]
                c = Jo[row * nf:(row + 1) * nf][sl]
                assert rel_err(a, c) < 1e-12, (row, rel_err(a, c))


def run_step(sol, o, emhd, imp, spec, P, U, S, dt, P_guess=None, fail0=None):
    Psol = (P if P_guess is None else P_guess).copy()
    norm = np.zeros(spec.shape)
    fail = np.zeros(spec.shape) if fail0 is None else fail0.copy()
    Psd, nd, fd = dev(Psol), dev(norm), dev(fail)
    sol.set_implicit(imp)
    sol.step(dev(P), dev(U), dev(P), dev(S), Psd, nd, fd, dt)
    it_d, mx_d = sol.stats()
    it_o, mx_o = o.implicit_step(emhd, imp, P, U, P, S, Psol, norm, fail, dt)
    return (Psd.cpu().numpy(), nd.cpu().numpy(), fd.cpu().numpy(), it_d, mx_d), (Psol, norm, fail, it_o, mx_o)


@pytest.mark.parametrize("solver", ["qr", "lu"])
@pytest.mark.parametrize("variant", ["kappa_eta_ho", "constant", "soundspeed_q_only", "dp_only", "grmhd_only"])
def test_implicit_step_fd_bitwise(oracle_mod, variant, solver):
    spec, emhd, o, b, sol, P, U, S_e, S, dt = setup(oracle_mod, variant)
    tol = 1e-12 * np.abs(U[(slice(None),) + spec.interior]).max() / dt
    imp = implicit("fd", rootfind_tol=tol, use_qr=(solver == "qr"))
    (Pd, nd, fd, itd, mxd), (Po, no, fo, ito, mxo) = run_step(sol, o, emhd, imp, spec, P, U, S, dt)
    sl = spec.interior
    print(variant, solver, "iterations", ito, "max norms", mxo)
    assert itd == ito
    assert np.array_equal(mxd, mxo)
    assert np.array_equal(fd[sl], fo[sl])
    assert np.array_equal(nd[sl], no[sl])
    for s in slots(emhd):
        assert np.array_equal(Pd[s][sl], Po[s][sl]), f"slot {s}"


@pytest.mark.parametrize("variant", ["kappa_eta_ho", "constant", "grmhd_only"])
def test_implicit_step_exact_close(oracle_mod, variant):
    spec, emhd, o, b, sol, P, U, S_e, S, dt = setup(oracle_mod, variant, SHAPES["3d"])
    imp = implicit("exact", rootfind_tol=0.0, max_nonlinear_iter=4)      # a fixed number of iterations
    (Pd, nd, fd, itd, mxd), (Po, no, fo, ito, mxo) = run_step(sol, o, emhd, imp, spec, P, U, S, dt)
    sl = spec.interior
    assert itd == ito == 4
    assert np.array_equal(fd[sl], fo[sl])
    # the two exact Jacobians differ by rounding (~1e-15); after the iterates reach the residual's
    # round-off floor they differ by up to ~1e-12 of the smallest variable's scale (dP~ ~ 1e-5)
    for s in slots(emhd):
        assert rel_err(Pd[s][sl], Po[s][sl]) < 1e-11, s
    assert np.abs(mxd[-1] - mxo[-1]) <= 1e-12 * np.abs(U[(slice(None),) + sl]).max() / dt


def test_failures_backtracking_and_fix_solve_bitwise(oracle_mod):
    spec, emhd, o, b, sol, P, U, S_e, S, dt = setup(oracle_mod, "kappa_eta_ho")
    sl = spec.interior
    k, j = sl[0].start, sl[1].start + 2
    bad = [(k, j, sl[2].start + 5), (k, j + 1, sl[2].start + 17), (k, j + 1, sl[2].start + 18)]
    for z in bad:
        S[(0,) + z] = -50.0 * U[(0,) + z] / dt
    z2 = (k, j + 3, sl[2].start + 30)
    S[(0,) + z2] = -3.0 * U[(0,) + z2] / dt        # recovers by backtracking (lambda = 0.1)
    fail0 = np.zeros(spec.shape)
    fail0[k, j + 2, sl[2].start + 40] = 1.0         # failed in an earlier stage: skipped
    imp = implicit("fd", max_nonlinear_iter=3)
    (Pd, nd, fd, itd, mxd), (Po, no, fo, ito, mxo) = run_step(sol, o, emhd, imp, spec, P, U, S, dt, fail0=fail0)
    assert np.count_nonzero(fo[sl] == 1) == len(bad) + 1
    assert np.array_equal(fd[sl], fo[sl]) and np.array_equal(nd[sl], no[sl])
    for s in slots(emhd):
        assert np.array_equal(Pd[s][sl], Po[s][sl])
    # FixSolve over the whole block
    Uo = o.emhd_ptou(emhd, Po)
    Pdd, Udd = dev(Po), dev(Uo)
    sol.fix_solve(Pdd, Udd, dev(fo))
    o.fix_solve(emhd, Po, Uo, fo)
    torch.cuda.synchronize()
    assert np.array_equal(Pdd.cpu().numpy(), Po)
    for s in slots(emhd):
        assert np.array_equal(Udd[s].cpu().numpy(), Uo[s])


def test_torus_closure_close(oracle_mod):
    spec, emhd, o, b, sol, P, U, S_e, S, dt = setup(oracle_mod, "torus")
    Pd = dev(P)
    Sd = torch.zeros_like(Pd)
    sol.add_source(Pd, Sd)
    torch.cuda.synchronize()
    sl = (slice(None),) + spec.interior
    for s in slots(emhd)[8:]:
        assert rel_err(Sd[s].cpu().numpy()[spec.interior], S_e[s][spec.interior]) < 1e-12
    imp = implicit("fd", rootfind_tol=0.0, max_nonlinear_iter=3)
    (Pd_, nd, fd, itd, mxd), (Po, no, fo, ito, mxo) = run_step(sol, o, emhd, imp, spec, P, U, S, dt)
    for s in slots(emhd):
        assert rel_err(Pd_[s][spec.interior], Po[s][spec.interior]) < 1e-10, s


# ---------------------------------------------------------------------------- explicit EMHD step and ImEx
IMEX_BC = ("exchange",) * 4 + ("periodic",) * 2


def imex_setup(oracle_mod, variant, shape):
    import dataclasses
    spec, emhd, P, dt, xi = atmosphere_case(*shape, emhd=EMHD_VARIANTS[variant])
    spec = dataclasses.replace(spec, bc=IMEX_BC)
    o = oracle_mod.Oracle(spec)
    b = Block(spec, geometry=o.geometry())
    sol = ImplicitSolver(b, emhd, conn=o.connection())
    U = o.emhd_ptou(emhd, P)
    return spec, emhd, o, b, sol, P, U


@pytest.mark.parametrize("shape", ["2d", "3d"])
@pytest.mark.parametrize("variant", ["kappa_eta_ho", "constant", "soundspeed_q_only", "dp_only", "grmhd_only"])
def test_emhd_face_fluxes_match_oracle(oracle_mod, variant, shape):
    """Flux::GetFlux with the EMHD variables: every active slot of every face the stage consumes, and
    the signal speeds, bitwise equal to the oracle (no library transcendental on this path)."""
    spec, emhd, o, b, sol, P, U = imex_setup(oracle_mod, variant, SHAPES[shape])
    ng = spec.ng
    for d in range(1, spec.ndim + 1):
        Fo, cmax, cmin = o.get_flux_emhd(emhd, d, P)
        Fd, ctop = sol.get_flux(d, dev(P))
        torch.cuda.synchronize()
        Fd, ctop = Fd.cpu().numpy(), ctop.cpu().numpy()
        sl = []
        for n, ax in zip((spec.nx3, spec.nx2, spec.nx1), (3, 2, 1)):
            if n == 1:
                sl.append(slice(0, 1))
            elif ax == d:
                sl.append(slice(ng, ng + n + 1))
            else:
                sl.append(slice(ng - 1, ng + n + 1))
        sl = tuple(sl)
        for s in slots(emhd):
            assert np.array_equal(Fd[s][sl], Fo[s][sl]), f"dir {d} slot {s}: max diff {np.abs(Fd[s][sl] - Fo[s][sl]).max()}"
        assert np.array_equal(ctop[sl], np.maximum(cmax, cmin)[sl])


@pytest.mark.parametrize("variant", ["kappa_eta_ho", "constant", "soundspeed_q_only", "dp_only", "grmhd_only", "torus"])
def test_imex_step_matches_oracle(oracle_mod, variant):
    """Two vl2 ImEx steps (imex_step.cpp:58-356): fluxes, EMHD geometric and explicit sources, explicit
    B update, forward-difference Newton solve, FixSolve, periodic ghosts, P -> U.  Primitives and
    conserved variables within 1e-12 of the oracle per slot (the torus closure calls exp: 1e-10),
    solver status and the zone timestep minimum the same."""
    spec, emhd, o, b, sol, P, U = imex_setup(oracle_mod, variant, (64, 6, 4))
    imp = implicit("fd", max_nonlinear_iter=3, rootfind_tol=1e-12)
    sol.set_implicit(imp)
    tol = 1e-10 if variant == "torus" else 1e-12
    dt = 0.5
    Pd, Ud = dev(P), dev(U)
    sn_d, sf_d = sol.scalar_field(), sol.scalar_field()
    sn = np.zeros(spec.shape)
    sf = np.zeros(spec.shape)
    for _ in range(2):
        P1, U1, _, _ = o.imex_stage(emhd, imp, 1, dt, P, U, P, U, sn, sf)
        P, U, _, mn = o.imex_stage(emhd, imp, 2, dt, P, U, P1, U1, sn, sf)
        sol.imex_step(Pd, Ud, dt, sn_d, sf_d)
    mn_d = b.min_ndt()
    sl = (slice(None),) + spec.interior
    Pg, Ug = Pd.cpu().numpy(), Ud.cpu().numpy()
    for s in slots(emhd):
        assert rel_err(Pg[s][sl[1:]], P[s][sl[1:]]) <= tol, f"P slot {s}"
        assert rel_err(Ug[s][sl[1:]], U[s][sl[1:]]) <= tol, f"U slot {s}"
    assert np.array_equal(sf_d.cpu().numpy()[spec.interior], sf[spec.interior])
    assert abs(mn_d - mn) <= 1e-12 * abs(mn)


@pytest.mark.parametrize("shape", ["2d", "3d"])
@pytest.mark.parametrize("name", ["constant", "kappa_eta_ho"])
def test_imex_floors_limits_physical_faces_match_oracle(oracle_mod, name, shape):
    """Two vl2 ImEx steps on a block with outflow X1 (inflow checks), reflecting X2 (polar flux fixes,
    corner fix) and periodic X3 faces, drift-frame floors and the EMHD stability limits: the flux fixes
    of all 10 slots, the floors and limits after the solve, FixSolve and the 10-slot ghost zones
    (imex_step.cpp:58-356).  Primitives and conserved variables over the whole block, ghost zones
    included, within 1e-12 of the oracle per slot; floor and limit flags and solver status equal; the
    zone timestep minimum within 1e-12."""
    from emhd_cases import atmosphere_limits_case
    n1, n2, n3 = SHAPES[shape]
    spec, emhd, P = atmosphere_limits_case(name, n1, n2, n3)
    o = oracle_mod.Oracle(spec)
    b = Block(spec, geometry=o.geometry())
    sol = ImplicitSolver(b, emhd, conn=o.connection())
    U = o.emhd_ptou(emhd, P)
    imp = implicit("fd", max_nonlinear_iter=3, rootfind_tol=1e-12)
    sol.set_implicit(imp)
    dt = 0.5
    Pd, Ud = dev(P), dev(U)
    sn_d, sf_d = sol.scalar_field(), sol.scalar_field()
    sn, sf = np.zeros(spec.shape), np.zeros(spec.shape)
    sl = spec.interior
    seen = 0
    for _ in range(2):
        P1, U1, _, _, ff1, ef1 = o.imex_stage_flags(emhd, imp, 1, dt, P, U, P, U, sn, sf)
        P1d, U1d = sol.zeros(), sol.zeros()
        sol.imex_stage(1, dt, Pd, Ud, Pd, Ud, P1d, U1d, sn_d, sf_d)
        assert np.array_equal(b.fflag.cpu().numpy()[sl], ff1[sl].astype(np.int32))
        assert np.array_equal(sol.eflag.cpu().numpy()[sl], ef1[sl].astype(np.int32))
        P, U, _, mn, ff2, ef2 = o.imex_stage_flags(emhd, imp, 2, dt, P, U, P1, U1, sn, sf)
        P2d, U2d = sol.zeros(), sol.zeros()
        sol.imex_stage(2, dt, Pd, Ud, P1d, U1d, P2d, U2d, sn_d, sf_d)
        assert np.array_equal(b.fflag.cpu().numpy()[sl], ff2[sl].astype(np.int32))
        assert np.array_equal(sol.eflag.cpu().numpy()[sl], ef2[sl].astype(np.int32))
        seen |= int(np.bitwise_or.reduce(ef2[sl].astype(int), axis=None))
        Pd, Ud = P2d, U2d
        mn_d = b.min_ndt()
        assert abs(mn_d - mn) <= 1e-12 * abs(mn)
        Pg, Ug = Pd.cpu().numpy(), Ud.cpu().numpy()
        for s in slots(emhd):
            assert rel_err(Pg[s], P[s]) <= 1e-12, f"P slot {s}: {rel_err(Pg[s], P[s])}"
            assert rel_err(Ug[s], U[s]) <= 1e-12, f"U slot {s}: {rel_err(Ug[s], U[s])}"
        assert np.array_equal(sf_d.cpu().numpy()[sl], sf[sl])
    assert seen & 1 and seen & 2


def test_imex_stage_flag_arguments(oracle_mod):
    """khb_imex_stage_flags without flag fields rejects floors or limits that would write them
    (KHB_ERR_ARG), and the normal-observer floor frame is rejected on the EMHD state
    (KHB_ERR_UNSUPPORTED)."""
    import ctypes as C
    import dataclasses
    from emhd_cases import atmosphere_limits_case
    from kharma_b200.block import Fields
    OK, ERR_ARG, ERR_UNSUPPORTED = 0, -1, -4      # khb.h return codes
    spec, emhd, P = atmosphere_limits_case("constant")
    o = oracle_mod.Oracle(spec)
    U = o.emhd_ptou(emhd, P)

    def call(spec, emhd, with_flags):
        b = Block(spec, geometry=o.geometry())
        sol = ImplicitSolver(b, emhd, conn=o.connection())
        Pd, Ud = dev(P), dev(U)
        Po, Uo = sol.zeros(), sol.zeros()
        sn, sf = sol.scalar_field(), sol.scalar_field()
        fl = [C.c_void_p(b.fflag.data_ptr()), C.c_void_p(sol.eflag.data_ptr())] if with_flags else [None, None]
        rc = sol.lib.khb_imex_stage_flags(b.ctx, C.byref(sol._e), C.byref(sol._i), 1, 0.5, Fields(Pd).ref,
                                          Fields(Ud).ref, Fields(Pd).ref, Fields(Ud).ref, Fields(Po).ref,
                                          Fields(Uo).ref, C.c_void_p(sn.data_ptr()), C.c_void_p(sf.data_ptr()),
                                          fl[0], fl[1], b.stream)
        torch.cuda.synchronize()
        return rc

    assert call(spec, emhd, True) == OK
    assert call(spec, emhd, False) == ERR_ARG
    assert call(dataclasses.replace(spec, floors_on=False), emhd, False) == ERR_ARG   # the limits are on
    assert call(dataclasses.replace(spec, floors_on=False), dataclasses.replace(emhd, stability_limits=False),
                False) == OK
    assert call(dataclasses.replace(spec, floor_frame="normal"), emhd, True) == ERR_UNSUPPORTED

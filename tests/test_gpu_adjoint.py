"""Full-step adjoint (khb_adjoint_step) with checkpoint-and-recompute, wrapped in a
torch.autograd.Function here in the test harness only.

Checks:
  * directional derivatives of the objective against central finite differences of the FP64
    forward run on seeded random directions (a Bondi block in KS/MKS coordinates with the mass flux
    through the x1 face layer nearest r = 5 as the objective, a magnetized block inside the FM torus
    in FMKS coordinates, the periodic MHD linear-mode box with a functional of the final state);
  * the FP32-flux form's adjoint against the FP64 adjoint;
  * checkpoint spacing does not change the gradient (recompute reproduces the forward states).
Floors in the fluid and drift frames, and outflow and reflecting X1/X2 faces, are differentiated;
fixups, FOFC, normal-frame floors and transmitting faces are outside the differentiated scope; the
cases below keep every inversion successful (the harness raises otherwise).

The MC limiter and the LLF speed maxima are piecewise smooth: the adjoint is the derivative of the
branch each face takes.  Central differences agree with it where a perturbation crosses no branch
point, so the initial states carry smooth ramps in every variable and direction (no zone has a flat
neighbourhood, where the limited slope is not differentiable at all), and each direction is
differenced at up to three step sizes, the best agreement counting.
"""
import dataclasses
import math

import numpy as np
import pytest
import torch

from kharma_b200 import problems
from kharma_b200.adjoint import Run
from kharma_b200.block import Block, build_geometry
from kharma_b200.problems import cell_centers
from kharma_b200.spec import bondi_spec, mhdmodes_spec, torus_spec

pytestmark = pytest.mark.gpu


class KharmaRun(torch.autograd.Function):
    """J(P0) for a block run over fixed dts; backward through khb_adjoint_step."""

    @staticmethod
    def forward(ctx, P0, block, dts, weight, Pw, every):
        block.set_prims(P0)
        P0_full = block.P.clone()
        run = Run(block, dts, weight=weight, Pw=Pw, checkpoint_every=every)
        J = run.forward()
        ctx.run, ctx.P0_full = run, P0_full
        return torch.tensor(J, dtype=torch.float64, device=P0.device)

    @staticmethod
    def backward(ctx, g):
        grad = ctx.run.gradient_prims(ctx.P0_full)
        return g * grad, None, None, None, None, None


def objective(block, P0, dts, weight, Pw=None, every=5):
    block.set_prims(P0)
    return Run(block, dts, weight=weight, Pw=Pw, checkpoint_every=every).forward()


def gradient(block, P0, dts, weight, Pw=None, every=5):
    P = P0.clone().requires_grad_(True)
    J = KharmaRun.apply(P, block, dts, weight, Pw, every)
    J.backward()
    return float(J.detach()), P.grad.detach().clone()


def mdot_weight(spec, r_face=5.0):
    """dx2 dx3 on the x1 face layer nearest r = r_face (faces indexed like zones: face i is the
    left face of zone i), zero elsewhere."""
    n3, n2, n1 = spec.shape
    dx1, dx2, dx3 = spec.dx
    i_f = spec.ng + int(round((math.log(r_face) - spec.x1min) / dx1))
    assert spec.ng < i_f < spec.ng + spec.nx1
    w = np.zeros(spec.shape)
    sk, sj, _ = spec.interior
    w[sk, sj, i_f] = dx2 * dx3
    return torch.as_tensor(w.reshape(-1), device="cuda")


def directions(spec, P0, n, seed):
    """Seeded random interior directions scaled per variable by the variable's rms."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sl = (slice(None),) + spec.interior
    scale = P0[sl].pow(2).mean(dim=(1, 2, 3)).sqrt().cpu().numpy() + 1e-6
    out = []
    for _ in range(n):
        v = np.zeros(tuple(P0.shape))
        v[sl] = rng.standard_normal(v[sl].shape) * scale[:, None, None, None]
        out.append(torch.as_tensor(v, device="cuda"))
    return out


def ramps(spec, P):
    return problems.add_ramps(spec, P)


def check_fd(block, P0, dts, weight, Pw, ndir, seed, eps=(1e-6, 1e-7, 1e-8), tol=1e-5):
    """Adjoint directional derivatives against central differences; per direction the best of the
    step sizes counts (a branch point crossed at one size is rarely crossed at all three)."""
    J, g = gradient(block, P0, dts, weight, Pw)
    rels = []
    for v in directions(block.spec, P0, ndir, seed):
        ad = float((g * v).sum())
        best = math.inf
        for e in eps:
            fd = (objective(block, P0 + e * v, dts, weight, Pw) - objective(block, P0 - e * v, dts, weight, Pw)) / (2 * e)
            best = min(best, abs(fd - ad) / max(abs(fd), abs(ad), 1e-300))
            if best < 1e-7:
                break
        rels.append(best)
    rels = np.array(rels)
    print(f"J = {J:.6e}; adjoint vs central FD over {ndir} directions: median {np.median(rels):.1e}, "
          f"worst {rels.max():.1e}; all: {' '.join(f'{r:.0e}' for r in rels)}")
    assert rels.max() < tol
    assert np.median(rels) < 1e-6
    return g


def stable_dt(block, P0):
    """Half the CFL timestep of the initial state (the run's fixed dt)."""
    block.set_prims(P0)
    block.step(block.spec.dt_min)
    return 0.5 * block.spec.cfl * block.min_ndt()


def bondi_case(precision="fp64"):
    spec = bondi_spec(16, 8, 8, math.log(4.0), math.log(8.0), 0.3, 0.7, 0.0, math.pi / 2,
                      precision=precision, recon="linear_mc")
    geom = build_geometry(spec)
    P0 = torch.as_tensor(ramps(spec, problems.bondi(spec, geom)), device="cuda")
    b = Block(spec, geometry=geom)
    dts = [stable_dt(Block(dataclasses.replace(spec, precision="fp64"), geometry=geom), P0)] * 12
    return b, P0, dts, mdot_weight(spec)


def torus_block_case(precision="fp64"):
    full = torus_spec(128, 128, 64)
    # beyond the pressure maximum (r = 12) and off the midplane: monotone in x1 and x2
    spec = dataclasses.replace(full, nx1=12, nx2=12, nx3=8, x1min=math.log(13.0), x1max=math.log(18.0),
                               x2min=0.40, x2max=0.48, x3min=0.0, x3max=math.pi / 4, precision=precision,
                               bc=("exchange",) * 6, floors_on=False, check_inflow_inner_x1=False,
                               check_inflow_outer_x1=False, zero_polar_flux=False, fix_polar_flux=False,
                               fix_corner_inner=False)
    geom = build_geometry(spec)
    P0 = torch.as_tensor(ramps(spec, problems.fm_torus(spec, geom, u_jitter=0.0)), device="cuda")
    b = Block(spec, geometry=geom)
    dts = [stable_dt(Block(dataclasses.replace(spec, precision="fp64"), geometry=geom), P0)] * 8
    return b, P0, dts, mdot_weight(spec, r_face=15.0)


def test_adjoint_bondi_vs_fd():
    b, P0, dts, w = bondi_case()
    check_fd(b, P0, dts, w, None, ndir=64, seed=1)


def test_adjoint_bondi_physical_faces_vs_fd():
    """Outflow X1 faces with inflow checks (the outer face takes inflow: its ghost velocities are
    reset and its mass flux clipped), reflecting X2 faces with zero polar fluxes and the corner fix,
    periodic X3: the ghost fills' and flux fixes' adjoints against central differences."""
    b, P0, dts, w = bondi_case()
    spec = dataclasses.replace(b.spec, bc=("outflow", "outflow", "reflecting", "reflecting", "periodic", "periodic"),
                               check_inflow_inner_x1=True, check_inflow_outer_x1=True, zero_polar_flux=True,
                               fix_corner_inner=True)
    bp = Block(spec, geometry=b.geom)
    check_fd(bp, P0, dts, w, None, ndir=16, seed=3)


def test_adjoint_torus_block_mhd_vs_fd():
    # magnetized MC faces sit close to limiter branch points more often: 1e-4 on the worst direction
    b, P0, dts, w = torus_block_case()
    check_fd(b, P0, dts, w, None, ndir=8, seed=2, tol=1e-4)


@pytest.mark.parametrize("frame", ["drift", "fluid"])
def test_adjoint_torus_block_floors_vs_fd(frame):
    """The magnetized torus block with the floors on and the geometric density floor raised so that
    they bind on about half of the zones at every stage (drift frame: density, internal energy and
    velocity change; fluid frame: density and internal energy): the floors' adjoint (one dual
    evaluation of the floor map per input at the inverted, pre-floor primitives the recompute keeps)
    against central differences."""
    b, P0, dts, w = torus_block_case()
    spec = dataclasses.replace(b.spec, floors_on=True, floor_frame=frame,
                               floors=dataclasses.replace(b.spec.floors, rho_min_geom=50.0))
    bf = Block(spec, geometry=b.geom)
    bf.set_prims(P0)
    bf.step(dts[0])
    floored = float((bf.fflag[spec.interior] != 0).float().mean())
    assert 0.2 < floored < 0.8, floored
    check_fd(bf, P0, dts, w, None, ndir=8, seed=5, tol=1e-4)


def test_adjoint_through_fixups_vs_fd():
    """Inversion failures and FixUtoP: three zones of the torus block's initial conserved state are
    poisoned (two hot, 1D_W max_iter; one with negative D, neg_input) after U = U(P0), so that their
    inversions fail and the fixup replaces them by the weighted average of their neighbours; the
    adjoint through the fixup (to the neighbours' primitives and the zone's own B) against central
    differences in directions that leave the poisoned zones' P0 alone (their U0 is not U(P0))."""
    import poison_cases
    b, P0, dts, w = torus_block_case()
    spec = b.spec
    ng = spec.ng
    zs = [(ng + 3, ng + 4, ng + 5), (ng + 4, ng + 7, ng + 6), (ng + 5, ng + 5, ng + 8)]
    kinds = ["hot", "hot", "neg_D"]

    def prepare(P):
        b.set_prims(P)
        U = b.U.cpu().numpy()
        for z, kind in zip(zs, kinds):
            U[(slice(0, 8),) + z] = poison_cases.POISONS[kind](U[(slice(0, 8),) + z])
        b.U.copy_(torch.as_tensor(U, device="cuda"))

    def objective_p(P):
        prepare(P)
        return Run(b, dts, weight=w, checkpoint_every=5).forward()

    prepare(P0)
    P0_full = b.P.clone()
    run = Run(b, dts, weight=w, checkpoint_every=5)
    J = run.forward()
    assert run.failures >= len(zs), run.failures
    g = run.gradient_prims(P0_full)
    rng = np.random.Generator(np.random.PCG64(7))
    sl = (slice(None),) + spec.interior
    scale = P0[sl].pow(2).mean(dim=(1, 2, 3)).sqrt().cpu().numpy() + 1e-6
    rels = []
    for _ in range(8):
        v = np.zeros(tuple(P0.shape))
        v[sl] = rng.standard_normal(v[sl].shape) * scale[:, None, None, None]
        for z in zs:
            v[(slice(None),) + z] = 0.
        v = torch.as_tensor(v, device="cuda")
        ad = float((g * v).sum())
        best = math.inf
        for e in (1e-6, 1e-7, 1e-8):
            fd = (objective_p(P0 + e * v) - objective_p(P0 - e * v)) / (2 * e)
            best = min(best, abs(fd - ad) / max(abs(fd), abs(ad), 1e-300))
            if best < 1e-7:
                break
        rels.append(best)
    rels = np.array(rels)
    print(f"J = {J:.6e}, {run.failures} failed inversions; adjoint vs central FD: median {np.median(rels):.1e}, "
          f"worst {rels.max():.1e}")
    assert rels.max() < 1e-4
    assert np.median(rels) < 1e-6


@pytest.mark.parametrize("nsteps,tol,tol_median", [(1, 1e-4, 1e-5), (6, 2e-3, 5e-4)])
def test_adjoint_fm_torus_floored_vs_fd(nsteps, tol, tol_median):
    """The adjoint workload's physics on a small FM torus block (FMKS a = 0.9375, SANE field, u jittered
    +-4%, linear MC, LLF, flux-CT, 1D_W, drift-frame floors and ceilings, outflow X1 faces with inflow
    checks, reflecting X2 faces with both polar flux fixes and the corner fix, periodic X3; a few
    hundred inversions fail and are fixed up): gradient of the mass through r = 5 with respect to the
    initial internal-energy perturbation, against central differences in directions of that
    perturbation field (u (1 + eps xi) where the jitter acts, rho above the floor).  Outside the torus
    the initial state is exactly axisymmetric, so its x3 MC slopes sit at the limiter's non-smooth
    point (both differences zero) and a perturbation there has no derivative; the perturbation
    field's support avoids that.  Over several steps central differences themselves stop
    converging below about 1e-4 (the inverter's 1e-8 tolerance, zones hovering at the floors): the
    bar widens with the steps."""
    spec = torus_spec(32, 24, 8)
    geom = build_geometry(spec)
    P0 = torch.as_tensor(problems.fm_torus(spec, geom, seed=11), device="cuda")
    b = Block(spec, geometry=geom)
    dts = [stable_dt(Block(spec, geometry=geom), P0)] * nsteps
    w = mdot_weight(spec)
    J, g = gradient(b, P0, dts, w)
    run = Run(b, dts, weight=w)
    b.set_prims(P0)
    run.forward()
    b.set_prims(P0)
    b.step(dts[0])
    assert int((b.fflag[spec.interior] != 0).sum()) > 0
    jittered = P0[0] > spec.floors.rho_min_geom
    rng = np.random.Generator(np.random.PCG64(9))
    rels = []
    for _ in range(8):
        v = torch.zeros_like(P0)
        xi = torch.as_tensor(rng.standard_normal(tuple(P0[1][spec.interior].shape)), device="cuda")
        v[1][spec.interior] = xi * P0[1][spec.interior]
        v[1] = torch.where(jittered, v[1], torch.zeros_like(v[1]))
        ad = float((g * v).sum())
        best = math.inf
        for e in (1e-5, 1e-6, 1e-7):
            fd = (objective(b, P0 + e * v, dts, w) - objective(b, P0 - e * v, dts, w)) / (2 * e)
            best = min(best, abs(fd - ad) / max(abs(fd), abs(ad), 1e-300))
        rels.append(best)
    rels = np.array(rels)
    print(f"J = {J:.6e}, {run.failures} failed inversions; adjoint vs central FD (u perturbation field, {nsteps} "
          f"steps): median {np.median(rels):.1e}, worst {rels.max():.1e}")
    assert rels.max() < tol
    assert np.median(rels) < tol_median


@pytest.mark.parametrize("recon", ["donor_cell", "linear_mc"])
def test_adjoint_mhdmodes_periodic_final_state_vs_fd(recon):
    """Periodic MHD box (flux-CT, folded periodic ghost adjoints) with a smooth mode along every
    direction in every variable, objective a random functional of the final primitives."""
    spec = mhdmodes_spec(16, 16, 8, recon=recon)
    b = Block(spec)
    P0 = problems.mhdmodes(spec, 3, amp=1e-2)
    x1, x2, x3 = cell_centers(spec)
    X3, X2, X1 = np.meshgrid(x3, x2, x1, indexing="ij")
    rng = np.random.Generator(np.random.PCG64(7))
    for q in range(spec.nvar):
        P0[q] += 1e-2 * np.sin(2 * np.pi * (X1 + X2 + X3) + rng.uniform(0, 2 * np.pi))
    P0 = torch.as_tensor(P0, device="cuda")
    Pw = np.zeros(tuple(P0.shape))
    sl = (slice(None),) + spec.interior
    Pw[sl] = rng.standard_normal(Pw[sl].shape)
    Pw = torch.as_tensor(Pw, device="cuda")
    dts = [stable_dt(b, P0)] * 10
    check_fd(b, P0, dts, None, Pw, ndir=8, seed=3)


def test_adjoint_cartesian_exchange_mhd_vs_fd():
    """Minkowski MHD block with exchange faces (constant ghosts), several steps, final-state objective.
    Donor-cell faces: the strongly magnetized mode puts many MC faces next to limiter branch points,
    where central differences stop resolving the derivative (the MC path is covered above)."""
    spec = dataclasses.replace(mhdmodes_spec(12, 12, 8, recon="donor_cell"), bc=("exchange",) * 6)
    b = Block(spec)
    P0 = torch.as_tensor(ramps(spec, problems.mhdmodes(spec, 3, amp=1e-2)), device="cuda")
    rng = np.random.Generator(np.random.PCG64(8))
    Pw = np.zeros(tuple(P0.shape))
    sl = (slice(None),) + spec.interior
    Pw[sl] = rng.standard_normal(Pw[sl].shape)
    Pw = torch.as_tensor(Pw, device="cuda")
    dts = [stable_dt(b, P0)] * 6
    check_fd(b, P0, dts, None, Pw, ndir=8, seed=5)


def test_adjoint_cartesian_physical_faces_mhd_vs_fd():
    """Minkowski MHD block with outflow X1 faces (inflow checks), reflecting X2 faces (zero polar
    fluxes, the corner fix) and periodic X3: the ghost fills of P and of U_B (the ghost B_P = U_B/gdet)
    and the flux fixes, against central differences of a final-state objective (donor-cell faces)."""
    spec = dataclasses.replace(mhdmodes_spec(12, 12, 8, recon="donor_cell"),
                               bc=("outflow", "outflow", "reflecting", "reflecting", "periodic", "periodic"),
                               check_inflow_inner_x1=True, check_inflow_outer_x1=True, zero_polar_flux=True,
                               fix_corner_inner=True)
    b = Block(spec)
    P0 = torch.as_tensor(ramps(spec, problems.mhdmodes(spec, 3, amp=1e-2)), device="cuda")
    rng = np.random.Generator(np.random.PCG64(9))
    Pw = np.zeros(tuple(P0.shape))
    sl = (slice(None),) + spec.interior
    Pw[sl] = rng.standard_normal(Pw[sl].shape)
    Pw = torch.as_tensor(Pw, device="cuda")
    dts = [stable_dt(b, P0)] * 6
    check_fd(b, P0, dts, None, Pw, ndir=8, seed=6)


def test_adjoint_polar_mhd_vs_fd():
    """A magnetized FMKS block on the pole (reflecting X2 faces with B_FluxCT's polar B-flux fix and
    zero polar fluxes, outflow X1 faces with inflow checks, floors off; a ramped magnetized gas),
    final-state objective."""
    full = torus_spec(128, 128, 64)
    spec = dataclasses.replace(full, nx1=12, nx2=8, nx3=8, x1min=math.log(13.0), x1max=math.log(18.0),
                               x2min=0.0, x2max=0.1, x3min=0.0, x3max=math.pi / 4, floors_on=False,
                               recon="donor_cell")
    geom = build_geometry(spec)
    # a gas at rest with a radial field, ramped in every variable (the torus itself is atmosphere here)
    P = np.zeros((8,) + spec.shape)
    P[0], P[1], P[5] = 1.0, 0.1, 0.05
    P0 = torch.as_tensor(ramps(spec, P), device="cuda")
    b = Block(spec, geometry=geom)
    rng = np.random.Generator(np.random.PCG64(10))
    Pw = np.zeros(tuple(P0.shape))
    sl = (slice(None),) + spec.interior
    Pw[sl] = rng.standard_normal(Pw[sl].shape)
    Pw = torch.as_tensor(Pw, device="cuda")
    dts = [stable_dt(Block(spec, geometry=geom), P0)] * 4
    check_fd(b, P0, dts, None, Pw, ndir=8, seed=7, tol=1e-4)


def test_adjoint_donor_cell_vs_fd():
    b, P0, dts, w = bondi_case()
    spec = dataclasses.replace(b.spec, recon="donor_cell")
    b = Block(spec, geometry=b.geom)
    check_fd(b, P0, dts, w, None, ndir=8, seed=4)


def test_adjoint_checkpoint_spacing():
    b, P0, dts, w = bondi_case()
    J1, g1 = gradient(b, P0, dts, w, every=1)
    J5, g5 = gradient(b, P0, dts, w, every=5)
    Jall, gall = gradient(b, P0, dts, w, every=100)
    assert J1 == J5 == Jall
    scale = float(gall.abs().max())
    # the adjoint scatters with atomics: equal to rounding, not bitwise
    assert float((g1 - gall).abs().max()) <= 1e-12 * scale
    assert float((g5 - gall).abs().max()) <= 1e-12 * scale


@pytest.mark.parametrize("case", [bondi_case, torus_block_case], ids=["bondi", "torus_block"])
def test_adjoint_fp32_flux_vs_fp64(case):
    b64, P0, dts, w = case("fp64")
    b32, _, _, _ = case("fp32_flux")
    J64, g64 = gradient(b64, P0, dts, w)
    J32, g32 = gradient(b32, P0, dts, w)
    relJ = abs(J32 - J64) / abs(J64)
    relg = float((g32 - g64).norm() / g64.norm())
    print(f"FP32-flux vs FP64: objective {relJ:.2e}, gradient (relative L2) {relg:.2e}")
    assert relJ < 1e-5
    assert relg < 1e-3


def test_adjoint_rejects_unsupported():
    from kharma_b200 import _lib
    spec = bondi_spec(8, 8, 8, math.log(4.0), math.log(8.0), 0.3, 0.7, 0.0, math.pi / 2)   # WENO5
    b = Block(spec)
    b.set_prims(problems.bondi(spec, b.geom))
    run = Run(b, [0.01], weight=None, Pw=torch.ones_like(b.P))
    run.forward()
    with pytest.raises(_lib.KhbError, match="reconstruction"):
        run.adjoint()
    # floors in the normal-observer frame (their re-inversion is not differentiated)
    tb, P0, dts, w = torus_block_case()
    spec = dataclasses.replace(tb.spec, floors_on=True, floor_frame="normal")
    nb = Block(spec, geometry=tb.geom)
    nb.set_prims(P0)
    run = Run(nb, dts[:1], weight=w)
    run.forward()
    with pytest.raises(_lib.KhbError, match="drift frames"):
        run.adjoint()

"""Static mesh refinement through the batch (khb_batch_set_mesh): two- and three-level hydro meshes on
a periodic box, and one-level meshes with outflow or reflecting domain faces.

* The ghost zones the library fills after an exchange equal, bitwise, the oracle-side restatement
  built from whole-domain arrays (oracle/smr_ref.py).
* With flux correction the mesh conserves mass to rounding, and energy and momentum as well as the
  unrefined mesh does (the lock-step U = U(P) after the inversion limits both to the inversion's
  tolerance); without it, mass is not conserved (the check has teeth).
* A uniform state stays exactly uniform across the refinement boundary.
* An entropy wave advected across the refined patch: the mesh's error lies between those of the
  uniform coarse and uniform fine meshes.
* 2x2 blocks with physical domain faces step bitwise as one block of the whole domain.
* The kharma driver's exchange (conserved variables and inversion seeds, the ghost zones inverted
  like the interior): ghost zones equal the oracle's inversion of the restated conserved state from
  the restated seed; one level steps bitwise as one block; conservation and uniformity as above.
* MKS (spherical KS) meshes: exchange bitwise as restated, one level as one block to 1e-9.
* The FP32-flux form on a mesh stays within 1e-5 relative L1 density of the FP64 mesh.
"""
import dataclasses
import importlib.util
import os

import numpy as np
import pytest
import torch

from kharma_b200 import problems
from kharma_b200.mesh import SMRMesh, conserved_totals, smr_batch
from kharma_b200.spec import BlockSpec

pytestmark = pytest.mark.gpu

_spec = importlib.util.spec_from_file_location(
    "smr_ref", os.path.join(os.path.dirname(__file__), "..", "oracle", "smr_ref.py"))
smr_ref = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(smr_ref)


def base(nd, recon="linear_mc"):
    return BlockSpec(nx1=16, nx2=16 if nd > 1 else 1, nx3=16 if nd > 2 else 1, x1min=0., x1max=1., x2min=0.,
                     x2max=1., x3min=0., x3max=1., gam=5. / 3., nvar=5, recon=recon, cfl=0.8, dt_min=1e-4)


def mesh_of(nd, refine=((0, 0, 0),), nx=16, nb=2, recon="linear_mc"):
    return SMRMesh(base(nd, recon), (nb, nb, nb if nd > 2 else 1), (nx, nx, nx if nd > 2 else 1), refine=refine)


def random_smooth(spec, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    P = problems.entropy_wave(spec, amp=0.1)
    P[0] *= 1 + 0.05 * rng.standard_normal(P[0].shape)
    P[1] *= 1 + 0.05 * rng.standard_normal(P[1].shape)
    P[2:5] += 0.05 * rng.standard_normal(P[2:5].shape)
    return P


@pytest.mark.parametrize("nd", [2, 3])
def test_exchange_matches_restatement(nd):
    mesh = mesh_of(nd)
    seeds = iter(range(1000))
    b = smr_batch(mesh, lambda s: random_smooth(s, next(seeds)))
    torch.cuda.synchronize()
    P = [blk.P.cpu().numpy() for blk in b.blocks]
    for n, ((mask, E), Pb) in enumerate(zip(smr_ref.expected_ghosts(mesh, P), P)):
        got, want = Pb[:, mask], E[:, mask]
        assert np.array_equal(got, want), (n, mesh.blocks[n].level, np.abs(got - want).max())


def run(mesh, flux_correction, steps=10, init=None, conserved=None):
    b = smr_batch(mesh, init or (lambda s: random_smooth(s, 3)), flux_correction=flux_correction,
                  conserved=conserved)
    t0 = conserved_totals(mesh, b)
    dt = 0.2 * min(blk.spec.dx[0] for blk in mesh.blocks)
    for _ in range(steps):
        b.step(dt)
    torch.cuda.synchronize()
    assert not any(blk.pflag.any() for blk in b.blocks)
    return b, t0, conserved_totals(mesh, b)


@pytest.mark.parametrize("nd,conserved", [(2, False), (3, False), (2, True), (3, True)])
def test_flux_correction_conserves(nd, conserved):
    _, r0, r1 = run(mesh_of(nd, refine=()), True, conserved=conserved)
    mesh = mesh_of(nd)
    _, t0, t1 = run(mesh, True, conserved=conserved)
    scale = np.abs(t0).max()
    uniform = np.abs(r1 - r0) / scale
    refined = np.abs(t1 - t0) / scale
    print("relative change of the conserved totals, unrefined:", uniform, "refined:", refined)
    assert refined[0] <= 1e-13
    assert np.all(refined <= 10 * uniform + 1e-13)
    _, u0, u1 = run(mesh, False, conserved=conserved)
    print("refined without flux correction:", np.abs(u1 - u0) / scale)
    assert np.abs(u1[0] - u0[0]) > 1e-9 * abs(u0[0])


@pytest.mark.parametrize("conserved", [False, True])
def test_uniform_state_stays_uniform(conserved):
    mesh = mesh_of(2)

    def uniform(s):
        P = np.zeros((5,) + s.shape)
        P[0], P[1], P[2], P[3] = 1.0, 2.0, 0.2, -0.1
        return P

    b, _, _ = run(mesh, True, steps=5, init=uniform, conserved=conserved)
    for blk in b.blocks:
        P = blk.P.cpu().numpy()
        ref = uniform(blk.spec)
        assert np.abs(P - ref).max() <= 1e-14


def test_entropy_wave_error_between_coarse_and_fine():
    """The wave crosses the refined patch: the L1 density error of the mesh (over all leaf zones,
    volume-weighted) lies between the uniform-coarse and uniform-fine errors."""
    t_end = 0.5
    errs = {}
    for name, mesh in (("coarse", mesh_of(2, refine=())), ("fine", mesh_of(2, refine=(), nb=4)),
                       ("smr", mesh_of(2))):
        b = smr_batch(mesh, lambda s: problems.entropy_wave(s, amp=0.1))
        dx = min(blk.spec.dx[0] for blk in mesh.blocks)
        n = int(np.ceil(t_end / (0.3 * dx)))
        for _ in range(n):
            b.step(t_end / n)
        torch.cuda.synchronize()
        e, vol = 0.0, 0.0
        for k, (mb, blk) in enumerate(zip(mesh.blocks, b.blocks)):
            ref = problems.entropy_wave(mb.spec, amp=0.1, t=t_end)
            sl = mb.spec.interior
            v = mesh.zone_volume(k)
            e += np.abs(blk.P.cpu().numpy()[0][sl] - ref[0][sl]).sum() * v
            vol += ref[0][sl].size * v
        errs[name] = e / vol
    print("entropy wave L1 errors:", errs)
    assert errs["fine"] < errs["smr"] < errs["coarse"]


def three_level(nd, nx=8):
    """4^nd roots of nx^nd zones, the central 2^nd refined, the central 2^nd of those refined again."""
    c = [(a, b, e) for a in (1, 2) for b in (1, 2) for e in ((1, 2) if nd > 2 else (0,))]
    f = [(1, (a, b, e)) for a in (3, 4) for b in (3, 4) for e in ((3, 4) if nd > 2 else (0,))]
    return SMRMesh(base(nd), (4, 4, 4 if nd > 2 else 1), (nx, nx, nx if nd > 2 else 1), refine=c + f)


@pytest.mark.parametrize("nd", [2, 3])
def test_three_levels_exchange_matches_restatement(nd):
    """The level-2 ghost zones prolongated from level-1 zones, some of which are level-1 ghost zones
    prolongated from level 0 in the phase before: bitwise against the whole-domain restatement."""
    mesh = three_level(nd)
    seeds = iter(range(1000))
    b = smr_batch(mesh, lambda s: random_smooth(s, next(seeds)))
    torch.cuda.synchronize()
    P = [blk.P.cpu().numpy() for blk in b.blocks]
    for n, ((mask, E), Pb) in enumerate(zip(smr_ref.expected_ghosts(mesh, P), P)):
        got, want = Pb[:, mask], E[:, mask]
        assert np.array_equal(got, want), (n, mesh.blocks[n].level, np.abs(got - want).max())


@pytest.mark.parametrize("nd", [2, 3])
def test_three_levels_conserve(nd):
    mesh = three_level(nd)
    _, t0, t1 = run(mesh, True, steps=6)
    scale = np.abs(t0).max()
    refined = np.abs(t1 - t0) / scale
    print("three levels, relative change of the conserved totals:", refined)
    assert refined[0] <= 1e-13
    _, u0, u1 = run(mesh, False, steps=6)
    assert np.abs(u1[0] - u0[0]) > 1e-9 * abs(u0[0])


@pytest.mark.parametrize("driver", ["simple", "kharma"])
@pytest.mark.parametrize("faces", [("periodic",) * 6,
                                   ("outflow", "outflow", "reflecting", "reflecting", "periodic", "periodic"),
                                   ("reflecting",) * 4 + ("periodic",) * 2])
def test_one_level_steps_as_one_block(faces, driver):
    """2x2 blocks of one level, the domain periodic or with outflow or reflecting faces: each block on
    a domain face applies it after the exchange, over the ghost rows the exchange filled; the mesh
    steps bitwise as one block of the whole domain with those faces.  With the kharma driver the
    exchange moves the updated conserved variables and the seeds, and each ghost zone's inversion
    repeats its source zone's."""
    from kharma_b200.batch import Batch
    spec = dataclasses.replace(base(2), bc=faces, driver=driver)
    mesh = SMRMesh(spec, (2, 2, 1), (16, 16, 1))
    big = dataclasses.replace(spec, nx1=32, nx2=32)
    ng = big.ng
    Pbig = problems.entropy_wave(big, amp=0.1)
    J, I = np.meshgrid(np.arange(Pbig.shape[2]), np.arange(Pbig.shape[3]), indexing="ij")
    Pbig[2] += 0.05 * np.sin(2 * np.pi * (J - ng + 0.5) / 32)
    Pbig[3] += 0.05 * np.cos(2 * np.pi * (I - ng + 0.5) / 32)

    def init(s):
        lx, ly = round(s.x1min * 2), round(s.x2min * 2)
        return Pbig[:, :, ly * 16:ly * 16 + 16 + 2 * ng, lx * 16:lx * 16 + 16 + 2 * ng]
    b = smr_batch(mesh, init)
    one = Batch([big], init=None)
    with torch.cuda.stream(one.torch_stream):
        one.blocks[0].set_prims(Pbig)
    dt = 0.2 / 32
    for _ in range(5):
        b.step(dt)
        one.step(dt)
    torch.cuda.synchronize()
    Pone = one.blocks[0].P.cpu().numpy()
    for n, (blk, mb) in enumerate(zip(mesh.blocks, b.blocks)):
        sl = (slice(None), slice(0, 1), slice(ng + blk.loc[1] * 16, ng + blk.loc[1] * 16 + 16),
              slice(ng + blk.loc[0] * 16, ng + blk.loc[0] * 16 + 16))
        assert np.array_equal(mb.P.cpu().numpy()[(slice(None),) + blk.spec.interior], Pone[sl]), f"block {n}"


@pytest.mark.parametrize("nd", [2, 3])
def test_conserved_exchange_matches_restatement(oracle_mod, nd):
    """The kharma driver's exchange outside a stage (khb_batch_mesh_exchange with KHB_SYNC_CONSERVED):
    on block states whose U is not U(P), so that every inversion moves its seed, each ghost zone's
    primitives equal the oracle's inversion of the restated conserved state (copy, restriction or
    prolongation of the blocks' U) from the restated seed, with no failure, and its U is U(P)."""
    mesh = mesh_of(nd)
    seeds = iter(range(1000))
    b = smr_batch(mesh, lambda s: random_smooth(s, next(seeds)), conserved=True)
    torch.cuda.synchronize()
    rng = np.random.Generator(np.random.PCG64(11))
    P, U = [], []
    for blk in b.blocks:
        u = blk.U.cpu().numpy()
        u = u * (1 + 1e-3 * rng.standard_normal(u.shape))
        blk.U.copy_(torch.as_tensor(u))
        P.append(blk.P.cpu().numpy())
        U.append(u)
    torch.cuda.synchronize()
    b.mesh_exchange()
    torch.cuda.synchronize()
    o = oracle_mod.Oracle(mesh.blocks[0].spec)
    worst, checked = 0.0, 0
    for n, ((mask, Eu), (_, Ep), blk) in enumerate(zip(smr_ref.expected_ghosts(mesh, U),
                                                       smr_ref.expected_ghosts(mesh, P), b.blocks)):
        Pg, Ug = blk.P.cpu().numpy(), blk.U.cpu().numpy()
        pf = blk.pflag.cpu().numpy()
        for k, j, i in np.argwhere(mask):
            uz = np.ascontiguousarray(Eu[:, k, j, i])
            pz = np.ascontiguousarray(Ep[:, k, j, i])
            flag = o.lib.orc_utop_cell(o.h, int(j), int(i), oracle_mod._ptr(uz), oracle_mod._ptr(pz))
            assert flag == 0 and pf[k, j, i] == 0
            worst = max(worst, float(np.max(np.abs(Pg[:, k, j, i] - pz) / np.maximum(np.abs(pz), 1.0))))
            checked += 1
        Uo = o.ptou(Pg)
        assert np.array_equal(Ug[:, mask], Uo[:, mask]), n
    print("conserved exchange:", checked, "ghost zones, worst relative P difference", worst)
    assert checked > 0 and worst <= 1e-12


def mks_base(nx, bc=("outflow", "outflow", "reflecting", "reflecting", "periodic", "periodic")):
    from kharma_b200.spec import bondi_spec
    return bondi_spec(nx, nx, nx, np.log(3.0), np.log(30.0), 0.0, 1.0, 0.0, 2 * np.pi, recon="linear_mc", bc=bc)


def test_mks_exchange_matches_restatement():
    """A two-level mesh of spherical-KS (MKS) hydro blocks, outflow x1 and reflecting x2 domain faces:
    the exchanged ghost zones equal the restatement on the native grid bitwise (Parthenon's operators
    do not see the metric)."""
    mesh = SMRMesh(mks_base(16), (4, 4, 2), (16, 16, 16), refine=[(1, 1, 0)])
    seeds = iter(range(1000))
    b = smr_batch(mesh, lambda s: random_smooth(s, next(seeds)), conserved=False)
    torch.cuda.synchronize()
    P = [blk.P.cpu().numpy() for blk in b.blocks]
    cell = mesh.tables()[0]
    for n, ((mask, E), Pb) in enumerate(zip(smr_ref.expected_ghosts(mesh, P), P)):
        filled = np.zeros(mask.size, dtype=bool)
        filled[cell[cell[:, 0] == n, 1]] = True
        m = mask & filled.reshape(mask.shape)
        assert m.any() and np.array_equal(Pb[:, m], E[:, m]), n


@pytest.mark.parametrize("conserved", [False, True])
@pytest.mark.parametrize("poles", ["reflecting", "transmitting"])
def test_mks_one_level_steps_as_one_block(conserved, poles):
    """2x2x2 MKS blocks of the Bondi problem (outflow x1, reflecting x2, periodic x3) — or 2x2x1
    blocks spanning x3 with transmitting poles — step as the
    single block of the domain, with either exchange, to 1e-9 of each variable's (velocities: the
    velocity's) largest magnitude over 3 steps.  Not bitwise: each block evaluates its metric at its
    own zone centres, which differ from the single block's by rounding, and the connection is a
    centred difference of the metric with step 1e-8 (as the reference forms it), so rounding-level
    shifts of the centres move it by up to ~1e-8 of its size; over 3 steps that leaves ~1e-11."""
    from kharma_b200.batch import Batch
    from kharma_b200.block import build_geometry
    bc = ("outflow", "outflow", poles, poles, "periodic", "periodic")
    base_ = mks_base(16, bc=bc)
    nb3 = 2 if poles == "reflecting" else 1
    mesh = SMRMesh(base_, (2, 2, nb3), (16, 16, 16))
    big = dataclasses.replace(base_, nx1=32, nx2=32, nx3=16 * nb3)
    ng = big.ng
    Pbig = problems.bondi(big, build_geometry(big))

    def init(s):
        blk = next(x for x in mesh.blocks if x.spec is s)
        lx, ly, lz = blk.loc
        return Pbig[:, lz * 16:lz * 16 + 16 + 2 * ng, ly * 16:ly * 16 + 16 + 2 * ng, lx * 16:lx * 16 + 16 + 2 * ng]
    b = smr_batch(mesh, init, conserved=conserved)
    one = Batch([big], init=None)
    with torch.cuda.stream(one.torch_stream):
        one.blocks[0].set_prims(Pbig)
    dt = 1e-3
    for _ in range(3):
        b.step(dt)
        one.step(dt)
    torch.cuda.synchronize()
    Pone = one.blocks[0].P.cpu().numpy()
    # per variable: max |difference| over max |value| (the parity tests' measure)
    diff, scale = np.zeros(5), np.zeros(5)
    for blk, mb in zip(mesh.blocks, b.blocks):
        lx, ly, lz = blk.loc
        sl = (slice(None), slice(ng + lz * 16, ng + lz * 16 + 16), slice(ng + ly * 16, ng + ly * 16 + 16),
              slice(ng + lx * 16, ng + lx * 16 + 16))
        a, e = mb.P.cpu().numpy()[(slice(None),) + blk.spec.interior], Pone[sl]
        diff = np.maximum(diff, np.abs(a - e).reshape(5, -1).max(axis=1))
        scale = np.maximum(scale, np.abs(e).reshape(5, -1).max(axis=1))
        assert not mb.pflag.cpu().numpy().any()
    scale[2:] = scale[2:].max()             # u2, u3 vanish in Bondi: measure them against |u|
    worst = float(np.max(diff / scale))
    print("MKS one level vs one block: per-variable relative difference", diff / scale)
    assert worst <= 1e-9


@pytest.mark.parametrize("conserved", [False, True])
def test_fp32_flux_mesh_close_to_fp64(conserved):
    """The FP32-flux form on a two-level mesh (the flux correction and the exchange on FP32 fluxes):
    after 20 steps its density is within 1e-5 relative L1 of the FP64 mesh's, with either exchange."""
    import dataclasses
    out = {}
    for prec in ("fp64", "fp32_flux"):
        base_ = dataclasses.replace(base(2), precision=prec)
        mesh = SMRMesh(base_, (2, 2, 1), (16, 16, 1), refine=[(0, 0, 0)])
        b = smr_batch(mesh, lambda s: random_smooth(s, 5), conserved=conserved)
        dt = 0.2 * min(blk.spec.dx[0] for blk in mesh.blocks)
        for _ in range(20):
            b.step(dt)
        torch.cuda.synchronize()
        out[prec] = [blk.P.cpu().numpy()[(0,) + mb.spec.interior] for blk, mb in zip(b.blocks, mesh.blocks)]
    num = sum(float(np.abs(x - y).sum()) for x, y in zip(out["fp32_flux"], out["fp64"]))
    den = sum(float(np.abs(y).sum()) for y in out["fp64"])
    print("FP32-flux mesh vs FP64 mesh: relative L1 density difference", num / den)
    assert 0 < num / den < 1e-5

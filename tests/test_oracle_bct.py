"""B_CT (face-centred field, b_ct/b_ct.cpp) in the oracle, CPU only.

Constrained transport changes each face by the circulation of the edge EMFs, so the discrete face
divergence of every zone keeps its initial value to rounding whatever the EMF scheme; a face field
built as a discrete curl therefore stays divergence-free.  The three EMF schemes differ only in the
corrections they add to the Balsara-Spicer average, so on a smooth mode they agree with each other
to the truncation error.
"""
import dataclasses

import numpy as np
import pytest

from kharma_b200 import problems
from kharma_b200.spec import mhdmodes_spec


def run(oracle_mod, spec, P0, Bf0, nsteps, dt=0.01):
    o = oracle_mod.Oracle(spec)
    P, U, Bf = o.ct_init_state(P0, Bf0)
    for _ in range(nsteps):
        pflag, fflag, _, _ = o.ct_step(P, U, Bf, dt)
        assert not pflag.any()
    return o, P, U, Bf


@pytest.mark.parametrize("scheme", ["bs99", "gs05_0", "gs05_c"])
@pytest.mark.parametrize("dims", [(16, 16, 1), (12, 12, 8)], ids=["2d", "3d"])
def test_face_divergence_stays_at_rounding(oracle_mod, scheme, dims):
    spec = dataclasses.replace(mhdmodes_spec(*dims, recon="linear_mc"), b_ct=scheme)
    P0 = problems.mhdmodes(spec, 3, amp=1e-2)
    Bf0 = problems.ct_curl_faces(spec)
    o, P, U, Bf = run(oracle_mod, spec, P0, Bf0, 5)
    assert o.ct_max_divb(Bf0) < 1e-12
    assert o.ct_max_divb(Bf) < 1e-12
    # the field did evolve
    assert np.abs(Bf - Bf0).max() > 1e-6


def test_face_divergence_is_conserved_zone_by_zone(oracle_mod):
    """Faces interpolated from a zone B that is not divergence-free (the reference's DangerousPtoU)
    carry a divergence; CT keeps every zone's value."""
    spec = dataclasses.replace(mhdmodes_spec(16, 16, 1, recon="linear_mc"), b_ct="gs05_c")
    P0 = problems.mhdmodes(spec, 3, amp=1e-2)
    # a seeded non-solenoidal perturbation of the zone field, so that the interpolated faces carry a
    # divergence
    rng = np.random.Generator(np.random.PCG64(3))
    P0[5:7] += 1e-3 * rng.standard_normal(P0[5:7].shape)
    o = oracle_mod.Oracle(spec)
    P, U, Bf = o.ct_init_state(P0)
    sl = spec.interior
    ng = spec.ng

    def div(Bf):
        dx1, dx2, _ = spec.dx
        return ((Bf[0][0, ng:-ng, ng + 1:-ng + 1] - Bf[0][0, ng:-ng, ng:-ng]) / dx1
                + (Bf[1][0, ng + 1:-ng + 1, ng:-ng] - Bf[1][0, ng:-ng, ng:-ng]) / dx2)

    d0 = div(Bf)
    assert np.abs(d0).max() > 1e-8
    for _ in range(5):
        o.ct_step(P, U, Bf, 0.01)
    assert np.abs(div(Bf) - d0).max() < 1e-12 * max(1.0, np.abs(d0).max())


def test_schemes_agree_on_a_smooth_mode(oracle_mod):
    base = mhdmodes_spec(24, 24, 1, recon="linear_mc")
    P0 = problems.mhdmodes(base, 3, amp=1e-4)
    out = {}
    for scheme in ("bs99", "gs05_0", "gs05_c"):
        spec = dataclasses.replace(base, b_ct=scheme)
        _, P, _, _ = run(oracle_mod, spec, P0, None, 10)
        out[scheme] = P
    pert = np.abs(P0[:, 0] - P0[:, 0].mean(axis=(1, 2), keepdims=True)).max()
    for a in ("gs05_0", "gs05_c"):
        assert np.abs(out[a] - out["bs99"]).max() < 0.05 * pert


def test_x3_outflow_cleaning_closes_the_ghost_zones(oracle_mod):
    """Outflow X3 faces (clean_face_B along x3, b_ct_boundaries.cpp:249-268): after the boundaries
    every ghost zone whose faces are all stored, in the X3 ghost layers, has zero face divergence to
    rounding, and the interior field keeps its rounding-level divergence over 5 steps."""
    spec = dataclasses.replace(mhdmodes_spec(12, 12, 12, recon="linear_mc"), b_ct="gs05_c",
                               bc=("periodic", "periodic", "periodic", "periodic", "outflow", "outflow"))
    P0 = problems.add_ramps(spec, problems.mhdmodes(spec, 3, amp=1e-2))
    Bf0 = problems.ct_curl_faces(spec)
    o, P, U, Bf = run(oracle_mod, spec, P0, Bf0, 5)
    assert o.ct_max_divb(Bf) < 1e-12
    dx1, dx2, dx3 = spec.dx
    F1, F2, F3 = Bf
    # zone (k, j, i) closed by faces i, i+1 / j, j+1 / k, k+1 (all stored for i < n1-1, j < n2-1, k < n3-1)
    div = ((F1[:-1, :-1, 1:] - F1[:-1, :-1, :-1]) / dx1 + (F2[:-1, 1:, :-1] - F2[:-1, :-1, :-1]) / dx2
           + (F3[1:, :-1, :-1] - F3[:-1, :-1, :-1]) / dx3)
    ng = spec.ng
    scale = np.abs(Bf).max() / min(spec.dx)
    for kz in list(range(0, ng)) + list(range(ng + spec.nx3, spec.shape[0] - 1)):
        assert np.abs(div[kz]).max() < 1e-12 * scale, kz

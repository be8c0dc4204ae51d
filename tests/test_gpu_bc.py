"""Transmitting polar boundaries (boundaries/one_block_transmit.cpp) on the GPU against the oracle:
a 3D MKS torus block over all of x3 with transmitting X2 faces, 3 steps to 1e-12 with identical
flags; and the ghost zones it fills are the mirrored zones half-way round in x3 with u^2, u^3, B^2,
B^3 inverted."""
import dataclasses

import numpy as np
import pytest
import torch

from kharma_b200 import problems
from kharma_b200.block import Block
from kharma_b200.spec import torus_spec

from test_gpu_parity import RTOL, make_pair, run_steps

pytestmark = pytest.mark.gpu


def transmit_spec():
    return dataclasses.replace(torus_spec(32, 24, 16), transform="mks",
                               bc=("outflow", "outflow", "transmitting", "transmitting", "periodic", "periodic"))


def test_transmitting_steps(oracle_mod):
    spec = transmit_spec()
    o, b, Po, Uo = make_pair(oracle_mod, spec, problems.fm_torus(spec, oracle_mod.Oracle(spec).geometry(), seed=3))
    worst, flags_equal = run_steps(o, b, Po, Uo, 3, spec)
    print("transmitting poles, worst per-variable relative error:", worst)
    assert np.all(worst <= RTOL), worst
    assert flags_equal


def test_transmitting_ghosts_are_mirrored_images():
    spec = transmit_spec()
    b = Block(spec)
    b.set_prims(problems.fm_torus(spec, b.geom, seed=3))
    torch.cuda.synchronize()
    P, U = b.P.cpu().numpy(), b.U.cpu().numpy()
    ng, n3 = spec.ng, spec.nx3
    sp = np.array([1, 1, 1, -1, -1])[:, None]          # fluid primitives: u^2, u^3 inverted
    sb = np.array([1, -1, -1])[:, None]                # conserved field: B^2, B^3 inverted
    for jg in range(ng):
        js = ng + (ng - 1 - jg)                        # inner pole: ghost row jg mirrors row 2 ng - 1 - jg
        for k in range(ng, ng + n3):
            ki = ((k - ng + n3 // 2) % n3) + ng
            assert np.array_equal(P[:5, k, jg, ng:-ng], sp * P[:5, ki, js, ng:-ng])
            assert np.array_equal(U[5:, k, jg, ng:-ng], sb * U[5:, ki, js, ng:-ng])


# Physical X3 faces (KBoundaries on inner/outer_x3, boundaries.cpp:369-589; Parthenon's face order
# x1, x2, x3): the X3 ghost planes copy (outflow) or mirror with u^3 and B^3 inverted (reflecting)
# the boundary planes over the whole (j, i) plane, after the X1/X2 faces.
X3_CASES = {
    "outflow": ("periodic", "periodic", "periodic", "periodic", "outflow", "outflow"),
    "reflecting": ("periodic", "periodic", "periodic", "periodic", "reflecting", "reflecting"),
    "mixed": ("outflow", "outflow", "periodic", "periodic", "reflecting", "outflow"),
}


@pytest.mark.parametrize("name", list(X3_CASES))
def test_x3_physical_faces_match_oracle(oracle_mod, name):
    from kharma_b200.spec import mhdmodes_spec
    spec = dataclasses.replace(mhdmodes_spec(16, 12, 12, recon="linear_mc"), bc=X3_CASES[name])
    # seeded smooth ramps on every variable, so that the state varies along x3 and u^3, B^3 are nonzero
    P0 = problems.add_ramps(spec, problems.mhdmodes(spec, 3, amp=1e-2))
    o, b, Po, Uo = make_pair(oracle_mod, spec, P0)
    worst, flags_equal = run_steps(o, b, Po, Uo, 5, spec)
    assert np.all(worst <= RTOL), worst
    assert flags_equal
    # the ghost planes themselves, after the last step's boundaries
    P, U = b.P.cpu().numpy(), b.U.cpu().numpy()
    assert np.max(np.abs(P - Po)) <= RTOL * np.max(np.abs(Po))
    assert np.max(np.abs(U - Uo)) <= RTOL * np.max(np.abs(Uo))
    ng, ke = spec.ng, spec.ng + spec.nx3 - 1
    if name == "reflecting":
        for g in range(ng):
            assert np.array_equal(P[4, ng - 1 - g], -P[4, ng + g])          # u^3 inverted
            assert np.array_equal(P[0, ke + 1 + g], P[0, ke - g])

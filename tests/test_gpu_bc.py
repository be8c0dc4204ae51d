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

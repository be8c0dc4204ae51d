"""B_FluxCT::MaxDivB by value (b_flux_ct.cpp:554-607, corner_div b_flux_ct_functions.hpp:52-75): the
GPU maximum against the oracle's on conserved fields whose divergence is O(1) or larger, in 2D and 3D,
Cartesian and FMKS torus blocks.  Spikes of B_U in single zones at the block edges check that both
take the same corner range (ValidDivBX1: the X1 corners of physical faces are left out).
Tolerance: relative 1e-12."""
import numpy as np
import pytest
import torch

from kharma_b200.block import Block
from kharma_b200.spec import mhdmodes_spec, torus_spec

pytestmark = pytest.mark.gpu

RTOL = 1e-12

SPECS = {
    "cart3d": lambda: mhdmodes_spec(24, 20, 16),
    "cart2d": lambda: mhdmodes_spec(24, 20, 1),
    "torus3d": lambda: torus_spec(32, 24, 8),
    "torus2d": lambda: torus_spec(32, 32, 1),
}


def oracle_divb(o, spec, U):
    phys = lambda bc: bc in ("outflow", "reflecting", "transmitting")
    return o.max_divb(np.ascontiguousarray(U), avoid_inner=phys(spec.bc[0]), avoid_outer=phys(spec.bc[1]))


def gpu_divb(b, U):
    b.U.copy_(torch.from_numpy(U))
    return b.max_divb()


@pytest.mark.parametrize("name", list(SPECS))
def test_max_divb_random_field_matches_oracle(oracle_mod, name):
    spec = SPECS[name]()
    o = oracle_mod.Oracle(spec)
    b = Block(spec, geometry=o.geometry())
    rng = np.random.default_rng(11)
    for trial in range(3):
        U = np.zeros((spec.nvar,) + spec.shape)
        U[5:8] = rng.uniform(-1.0, 1.0, size=(3,) + spec.shape)
        ref = oracle_divb(o, spec, U)
        got = gpu_divb(b, U)
        assert ref > 1.0
        assert abs(got - ref) <= RTOL * ref, (trial, got, ref)


@pytest.mark.parametrize("name", list(SPECS))
def test_max_divb_corner_range_matches_oracle(oracle_mod, name):
    spec = SPECS[name]()
    o = oracle_mod.Oracle(spec)
    b = Block(spec, geometry=o.geometry())
    ng = spec.ng
    is_, ie = ng, ng + spec.nx1 - 1
    js, je = ng, ng + spec.nx2 - 1
    ks, ke = (ng, ng + spec.nx3 - 1) if spec.nx3 > 1 else (0, 0)
    sites = [(ks, js, is_), (ke, je, ie), (ks, je, is_ + 1), (ke, js, ie - 1), (ks, (js + je) // 2, is_ - 1),
             (ke, (js + je) // 2, ie + 1)]
    seen_nonzero = 0
    for (k, j, i) in sites:
        for v in (5, 6, 7):
            if v == 7 and spec.nx3 == 1:
                continue
            U = np.zeros((spec.nvar,) + spec.shape)
            U[v, k, j, i] = 3.0
            ref = oracle_divb(o, spec, U)
            got = gpu_divb(b, U)
            assert abs(got - ref) <= RTOL * max(ref, 1e-300), ((k, j, i), v, got, ref)
            seen_nonzero += ref > 0
    assert seen_nonzero > 0

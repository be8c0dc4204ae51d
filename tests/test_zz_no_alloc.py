"""khb_max_divb_noalloc: the divB diagnostic for callers that cannot allocate device memory.

Callers whose device memory comes only from their own framework's pre-reserved pool, and diagnostic
hooks that hold field pointers but no khb_ctx, cannot use khb_max_divb (it needs a context, and
creating one allocates).  The no-allocation variant keeps its per-block partial maxima in a static
device array; these tests check, through the C ABI, that two calls in a row return what the
context-based entry point returns (relative 1e-12), that both equal the oracle's maximum on a field
with O(1) divergence, and that blocks without a field or without corners give 0 as khb_max_divb does.
The file is collected last, so that a run stopping at the first failure has already run every
other test.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from kharma_b200 import _lib, problems
from kharma_b200.block import Block
from kharma_b200.spec import bondi_spec, mhdmodes_spec, torus_spec

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def noalloc_divb(block, out):
    lib = _lib.load()
    cfg = block.spec.khb_config()
    rc = lib.khb_max_divb_noalloc(C.byref(cfg), block.Uf.ref, C.c_void_p(out.data_ptr()), block.stream)
    if rc != 0:
        raise _lib.KhbError(lib.khb_noalloc_last_error().decode())
    torch.cuda.synchronize()
    return float(out.item())


@pytest.mark.parametrize("spec", [mhdmodes_spec(24, 24, 24), torus_spec(32, 24, 8), mhdmodes_spec(32, 32, 1)],
                         ids=["periodic3d", "torus3d", "periodic2d"])
def test_noalloc_divb_matches_context_version(spec):
    b = Block(spec)
    if spec.spherical:
        b.set_prims(problems.fm_torus(spec, b.geom, seed=3))
    else:
        b.set_prims(problems.mhdmodes(spec, 3))
    # evolve a little so the field has structure beyond the initial condition
    dt = spec.dt_min
    for _ in range(3):
        b.step(dt)
        dt *= 2
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    for call in range(2):
        ref = b.max_divb()
        got = noalloc_divb(b, out)
        assert abs(got - ref) <= RTOL * max(abs(ref), 1e-300), f"call {call}: {got} vs {ref}"
        # move the state on so the second call sees different data
        b.step(dt)


@pytest.mark.parametrize("spec", [mhdmodes_spec(24, 20, 16), torus_spec(32, 24, 8)], ids=["cart3d", "torus3d"])
def test_noalloc_divb_matches_oracle(oracle_mod, spec):
    o = oracle_mod.Oracle(spec)
    b = Block(spec, geometry=o.geometry())
    rng = np.random.default_rng(5)
    phys = lambda bc: bc in ("outflow", "reflecting", "transmitting")
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    for call in range(2):
        U = np.zeros((spec.nvar,) + spec.shape)
        U[5:8] = rng.uniform(-1.0, 1.0, size=(3,) + spec.shape)
        b.U.copy_(torch.from_numpy(U))
        ref = o.max_divb(U, avoid_inner=phys(spec.bc[0]), avoid_outer=phys(spec.bc[1]))
        got = noalloc_divb(b, out)
        assert ref > 1.0
        assert abs(got - ref) <= RTOL * ref, f"call {call}: {got} vs {ref}"


@pytest.mark.parametrize("spec", [mhdmodes_spec(32, 1, 1), bondi_spec(16, 8, 8, 3.0, 30.0)], ids=["1d", "hydro"])
def test_noalloc_divb_zero_without_corners_or_field(spec):
    """A 1D block has no corners and a hydro block (nvar = 5) no field: 0, as khb_max_divb gives."""
    b = Block(spec)
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    assert noalloc_divb(b, out) == 0.0
    assert b.max_divb() == 0.0


def test_noalloc_rejects_oversized_block():
    spec = mhdmodes_spec(256, 256, 256)
    lib = _lib.load()
    cfg = spec.khb_config()
    fields = _lib.KhbFields()
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    for v in range(8):
        fields.v[v] = dummy.data_ptr()
    rc = lib.khb_max_divb_noalloc(C.byref(cfg), C.byref(fields), C.c_void_p(dummy.data_ptr()), None)
    assert rc == -1
    assert b"static scratch" in lib.khb_noalloc_last_error()

"""The batching form on the GPU: every block of the three-level Bondi mesh in one launch per kernel
per stage (khb_batch_step), replayed from a CUDA graph (khb_batch_step_graph), after autotuning.

Requirements: a batch step is bitwise identical to khb_step on each block in turn (the per-block
launch path), in both precisions and both launch plans (one launch per kernel per stage, or three
launches per stage); graph replay and any tile shape or plan chosen by the autotuner change
nothing; autotuning leaves the state alone; and each block matches the CPU oracle stepped with the
same ghost inputs to 1e-12 per variable (max |gpu - oracle| <= 1e-12 max |oracle|), flags exactly.
The mesh here has the production block counts (8 + 48 + 128) with 16^3, 8^3 and 4^3 blocks.
Blocks with physical and periodic faces (FM torus, Bondi, a periodic box), whose boundary work the
batch runs as one launch per boundary phase, also step bitwise as khb_step on each block.
"""
import numpy as np
import pytest
import torch

from kharma_b200 import problems
from kharma_b200.batch import Batch, bondi_smr_layout

pytestmark = pytest.mark.gpu

SMALL = (16, 8, 4)
DTS = [1e-3, 2e-3, 4e-3]


def assert_same(a, b):
    for x, (sa, sb) in enumerate(zip(a.state(), b.state())):
        for q in range(4):
            assert np.array_equal(sa[q], sb[q]), f"block {x} array {q} differs"


@pytest.mark.parametrize("plan", [0, 1])
@pytest.mark.parametrize("precision", ["fp64", "fp32_flux"])
def test_batch_step_equals_per_block_steps(precision, plan):
    specs = bondi_smr_layout(SMALL, precision=precision)
    a, b = Batch(specs), Batch(specs)
    a.set_plan(plan)
    for dt in DTS:
        a.step(dt)
        b.step_per_block(dt)
    assert_same(a, b)
    with torch.cuda.stream(b.torch_stream):
        per_block = min(blk.min_ndt() for blk in b.blocks)
    assert a.min_ndt() == per_block


def test_graph_replay_and_autotune_keep_results():
    specs = bondi_smr_layout(SMALL)
    a, b = Batch(specs), Batch(specs)
    kz, persistent = b.autotune(reps=2)
    assert set(kz) == {str((16, 16, 16)), str((8, 8, 8)), str((4, 4, 4))}
    assert all(v in (1, 2, 4) for v in kz.values()) and persistent in (0, 1)
    assert_same(a, b)                      # autotuning times stage 1 only: the state is untouched
    l0 = b.launch_count()
    for dt in DTS:
        a.step(dt)
        b.step_graph(dt)
    assert_same(a, b)
    per_step = (b.launch_count() - l0) / len(DTS)
    assert 0 < per_step <= 20             # a handful of launches per step, whatever the block count
    # other tile shapes and the other launch mode give the same bits
    for shape in (1, 2):
        c = Batch(specs)
        for q in range(3):
            c.set_tuning(q, shape, 1 - persistent)
        for dt in DTS:
            c.step(dt)
        assert_same(a, c)


def test_batch_blocks_match_oracle(oracle_mod):
    specs = bondi_smr_layout(SMALL)
    pick = [0, 8, 56]                      # one block of each size
    sub = [specs[i] for i in pick]
    batch = Batch(sub)
    for dt in DTS:
        batch.step(dt)
    for x, sp in enumerate(sub):
        o = oracle_mod.Oracle(sp)
        P, U = o.init_state(problems.bondi(sp, o.geometry()))
        for dt in DTS:
            pflag, fflag, _, _ = o.step(P, U, dt)
        Pg, Ug, pg, fg = batch.state()[x]
        sl = sp.interior
        for v in range(sp.nvar):
            for got, ref in ((Pg[v], P[v]), (Ug[v], U[v])):
                scale = np.max(np.abs(ref))
                assert np.max(np.abs(got - ref)) <= 1e-12 * scale, f"block {pick[x]} variable {v}"
        assert np.array_equal(pg[sl], pflag[sl].astype(np.int32))
        assert np.array_equal(fg[sl], fflag[sl].astype(np.int32))


@pytest.mark.parametrize("persistent", [0, 1])
def test_fused_plan_three_launches_per_stage(persistent):
    """The fused plan replays a step of the exchange-face Bondi mesh as 6 graph nodes (3 per stage),
    bitwise equal to the one-launch-per-kernel plan, flat or persistent grid."""
    specs = bondi_smr_layout(SMALL)
    a, b = Batch(specs), Batch(specs)
    b.set_tuning(-1, 0, persistent)
    b.set_plan(1)
    l0 = b.launch_count()
    for dt in DTS:
        a.step(dt)
        b.step_graph(dt)
    assert_same(a, b)
    assert (b.launch_count() - l0) / len(DTS) == 6


@pytest.mark.parametrize("plan", [0, 1])
def test_physical_and_periodic_faces_equal_per_block(plan):
    """Blocks with outflow, reflecting and periodic faces, whose boundary work (faces by direction,
    ghost P->U, periodic images) the batch runs as one launch per phase over all of them, step
    bitwise as khb_step on each block: two FM torus blocks of different sizes (flux-CT MHD: outflow
    x1 with the inflow checks, reflecting x2, periodic x3), and a hydro batch of a Bondi block
    (outflow x1, reflecting x2, periodic x3) beside a periodic Cartesian block."""
    from kharma_b200.block import build_geometry
    from kharma_b200.spec import BlockSpec, bondi_spec, torus_spec

    def pair(specs, inits):
        out = []
        for _ in range(2):
            bb = Batch(specs, init=None)
            with torch.cuda.stream(bb.torch_stream):
                for blk, P in zip(bb.blocks, inits):
                    blk.set_prims(P)
            out.append(bb)
        return out

    torus = [torus_spec(32, 24, 16), torus_spec(24, 16, 8)]
    bondi = bondi_spec(16, 16, 8, float(np.log(3.0)), float(np.log(30.0)), recon="linear_mc",
                       bc=("outflow", "outflow", "reflecting", "reflecting", "periodic", "periodic"))
    box = BlockSpec(nx1=16, nx2=8, nx3=8, x1min=0., x1max=1., x2min=0., x2max=1., x3min=0., x3max=1., gam=5. / 3.,
                    nvar=5, recon="linear_mc")
    cases = [(torus, [problems.fm_torus(s, build_geometry(s), seed=3 + n) for n, s in enumerate(torus)]),
             ([bondi, box], [problems.bondi(bondi, build_geometry(bondi)), problems.entropy_wave(box, amp=0.1)])]
    for specs, inits in cases:
        a, b = pair(specs, inits)
        a.set_plan(plan)
        for dt in (1e-3, 2e-3):
            a.step(dt)
            b.step_per_block(dt)
        assert_same(a, b)

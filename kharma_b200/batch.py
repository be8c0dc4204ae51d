"""Batches of meshblocks: every block of a static-refined mesh, of uneven sizes, stepped together.

`Batch` wraps khb_batch_* (include/khb.h): one launch per kernel per RK stage for all blocks, the
step optionally replayed from a CUDA graph, and the tile shape per block size chosen by the
library's autotuner.  `bondi_smr_layout` builds the Bondi workload: a three-level static-refined
arrangement of 8 blocks of 64^3, 48 of 32^3 and 128 of 16^3 zones (resolution doubling per level)
on spherical Kerr-Schild (a = 0) MKS coordinates.  Parthenon meshes have uniform block sizes, so
the reference has no such mesh; each block here has exchange faces whose ghost zones hold the
analytic Bondi solution (prob/bondi.hpp), i.e. the blocks are advanced independently with
identical ghost inputs, as the per-block comparison with the oracle needs.
"""
import ctypes as C
import math

import numpy as np
import torch

from . import _lib, problems
from .block import Block, build_geometry
from .spec import bondi_spec

_P = C.c_void_p


def bondi_smr_layout(sizes=(64, 32, 16), r_in=3.0, r_out=30.0, precision="fp64"):
    """Block specs of the three-level Bondi mesh, coarsest level first.

    Level l has blocks of sizes[l]^3 zones and native zone widths dx0 / 2^l.  With the default sizes:
      level 0: 2 x 2 x 2 blocks of 64^3 over x1 in [X_in + 20 dx0, X_out], all x2 and x3;
      level 1: 1 x 6 x 8 blocks of 32^3 over x1 in [X_in + 4 dx0, X_in + 20 dx0], x2 in [1/8, 7/8];
      level 2: 1 x 8 x 16 blocks of 16^3 over x1 in [X_in, X_in + 4 dx0], x2 in [3/8, 5/8], x3 in [0, pi];
    184 blocks, 4,194,304 zones; dx0 = (log r_out - log r_in) / 148 along x1, 1/128 along x2 and
    2 pi / 128 along x3.  Other sizes scale the zone counts with the same block counts.
    """
    s0, s1, s2 = sizes
    assert s0 == 2 * s1 == 4 * s2, "block sizes must halve per level"
    X_in, X_out = math.log(r_in), math.log(r_out)
    n1_0 = 2 * s0                       # level-0 zones along x1
    w1 = s1 / 2 / n1_0                  # x1 width of levels 1 and 2, in units of the level-0 span
    w2 = s2 / 4 / n1_0
    dx0 = (X_out - X_in) / (n1_0 * (1 + w1 + w2))
    specs = []
    # level 0
    x1a = X_in + (s1 / 2 + s2 / 4) * dx0
    for k in range(2):
        for j in range(2):
            for i in range(2):
                specs.append(bondi_spec(s0, s0, s0, x1a + i * s0 * dx0, x1a + (i + 1) * s0 * dx0,
                                        j * 0.5, (j + 1) * 0.5, k * math.pi, (k + 1) * math.pi, precision=precision))
    # level 1: one radial layer, x2 in [1/8, 7/8] (6 blocks), all x3 (8 blocks)
    x1b = X_in + (s2 / 4) * dx0
    for k in range(8):
        for j in range(6):
            specs.append(bondi_spec(s1, s1, s1, x1b, x1b + s1 * dx0 / 2, 0.125 + j * 0.125, 0.125 + (j + 1) * 0.125,
                                    k * math.pi / 4, (k + 1) * math.pi / 4, precision=precision))
    # level 2: one radial layer, x2 in [3/8, 5/8] (8 blocks), x3 in [0, pi] (16 blocks)
    for k in range(16):
        for j in range(8):
            specs.append(bondi_spec(s2, s2, s2, X_in, X_in + s2 * dx0 / 4, 0.375 + j / 32, 0.375 + (j + 1) / 32,
                                    k * math.pi / 16, (k + 1) * math.pi / 16, precision=precision))
    return specs


def _geom_key(spec):
    # the geometry is x3-independent: blocks differing only in x3 share it
    return (spec.nx1, spec.nx2, spec.nx3, spec.x1min, spec.x1max, spec.x2min, spec.x2max)


class Batch:
    """Blocks (kharma_b200.block.Block, each with its own context and state) under one khb_batch.

    All calls go on the batch's own CUDA stream (`self.stream`), which graph capture needs."""

    def __init__(self, specs, init="bondi", device="cuda"):
        self.lib = _lib.load()
        self.specs = list(specs)
        self.torch_stream = torch.cuda.Stream(device=device)
        geoms = {}
        self.blocks = []
        with torch.cuda.stream(self.torch_stream):
            for s in self.specs:
                key = _geom_key(s)
                if key not in geoms:
                    geoms[key] = build_geometry(s)
                g = geoms[key]
                b = Block(s, geometry=g, device=device)
                if init == "bondi":
                    b.set_prims(problems.bondi(s, g))
                self.blocks.append(b)
        self.geoms = geoms
        n = len(self.blocks)
        ctxs = (_P * n)(*[b.ctx.value for b in self.blocks])
        self._Pf = (_lib.KhbFields * n)(*[b.Pf.s for b in self.blocks])
        self._Uf = (_lib.KhbFields * n)(*[b.Uf.s for b in self.blocks])
        pf = (_P * n)(*[b.pflag.data_ptr() for b in self.blocks])
        ff = (_P * n)(*[b.fflag.data_ptr() for b in self.blocks])
        h = _P()
        _lib.check(self.lib.khb_batch_create(ctxs, n, self._Pf, self._Uf, pf, ff, C.byref(h)), "khb_batch_create")
        self.h = h
        self.zones = sum(s.nx1 * s.nx2 * s.nx3 for s in self.specs)

    def __del__(self):
        try:
            if getattr(self, "h", None):
                self.lib.khb_batch_destroy(self.h)
                self.h = None
        except Exception:
            pass

    @property
    def stream(self):
        return C.c_void_p(self.torch_stream.cuda_stream)

    def step(self, dt):
        _lib.check(self.lib.khb_batch_step(self.h, float(dt), self.stream), "khb_batch_step")

    def step_graph(self, dt):
        _lib.check(self.lib.khb_batch_step_graph(self.h, float(dt), self.stream), "khb_batch_step_graph")

    def step_per_block(self, dt):
        """The plain per-block launch path: khb_step on each block in turn (same stream)."""
        with torch.cuda.stream(self.torch_stream):
            for b in self.blocks:
                b.step(dt)

    def min_ndt(self):
        out = C.c_double()
        _lib.check(self.lib.khb_batch_get_min_ndt(self.h, C.byref(out), self.stream), "khb_batch_get_min_ndt")
        return out.value

    def classes(self):
        n = C.c_int32()
        sizes = (C.c_int32 * (3 * 64))()
        kz = (C.c_int32 * 64)()
        _lib.check(self.lib.khb_batch_classes(self.h, C.byref(n), sizes, kz, 64), "khb_batch_classes")
        return [((sizes[3 * q], sizes[3 * q + 1], sizes[3 * q + 2]), kz[q]) for q in range(n.value)]

    def set_tuning(self, size_class=-1, kz=0, persistent=0):
        _lib.check(self.lib.khb_batch_set_tuning(self.h, size_class, kz, persistent), "khb_batch_set_tuning")

    def autotune(self, reps=5):
        """Returns ({class size: planes per CTA}, persistent)."""
        ncls = len(self.classes())
        kz = (C.c_int32 * max(ncls, 1))()
        pers = C.c_int32()
        _lib.check(self.lib.khb_batch_autotune(self.h, reps, kz, C.byref(pers), self.stream), "khb_batch_autotune")
        return {str(c[0]): kz[q] for q, c in enumerate(self.classes())}, int(pers.value)

    def launch_count(self):
        return int(self.lib.khb_batch_launch_count(self.h))

    def set_plan(self, plan):
        """0: one launch per kernel per stage; 1: three launches per stage (khb_batch_set_plan)."""
        _lib.check(self.lib.khb_batch_set_plan(self.h, int(plan)), "khb_batch_set_plan")

    def plan(self):
        out = C.c_int32()
        _lib.check(self.lib.khb_batch_get_plan(self.h, C.byref(out)), "khb_batch_get_plan")
        return int(out.value)

    def set_mesh(self, ghost, n_ghost_first, flux):
        """SMR tables (kharma_b200.mesh.SMRMesh.tables): ghost exchange after every stage and flux
        correction before every update."""
        ghost = np.ascontiguousarray(ghost, dtype=np.int32)
        flux = np.ascontiguousarray(flux, dtype=np.int32)
        _lib.check(self.lib.khb_batch_set_mesh(self.h, ghost.ctypes.data_as(C.c_void_p), len(ghost), int(n_ghost_first),
                                               flux.ctypes.data_as(C.c_void_p), len(flux)), "khb_batch_set_mesh")

    def set_mesh_sync(self, conserved):
        """What the mesh's exchange moves: primitives (the simple and ImEx drivers), or conserved
        variables with the primitives as inversion seeds, the ghost zones then inverted (the kharma
        driver; kharma_driver.cpp:109-118)."""
        _lib.check(self.lib.khb_batch_set_mesh_sync(self.h, 1 if conserved else 0), "khb_batch_set_mesh_sync")

    def mesh_exchange(self):
        """Fill the ghost zones of every block's state from the mesh."""
        _lib.check(self.lib.khb_batch_mesh_exchange(self.h, self.stream), "khb_batch_mesh_exchange")

    def state(self):
        """Host copies of every block's (P, U, pflag, fflag)."""
        self.torch_stream.synchronize()
        return [(b.P.cpu().numpy(), b.U.cpu().numpy(), b.pflag.cpu().numpy(), b.fflag.cpu().numpy())
                for b in self.blocks]

"""Extended MHD and the implicit solve of one meshblock through libkhb.

Mirrors the calls the reference's EMHD and Implicit packages make per stage:
  * EMHD::AddSource (emhd/emhd.cpp:288-397)           -> ImplicitSolver.add_source
  * Implicit::Step (implicit/implicit.cpp:159-571)     -> ImplicitSolver.step
  * Implicit::FixSolve (implicit/fix_solve.cpp:44-130)  -> ImplicitSolver.fix_solve
  * Flux::MeshPtoU with EMHD + EMHD::BlockPtoU         -> ImplicitSolver.ptou
  * Flux::GetFlux with the EMHD variables               -> ImplicitSolver.get_flux
  * one ImEx stage / vl2 step (driver/imex_step.cpp)    -> ImplicitSolver.imex_stage / imex_step

State tensors are (10, n3, n2, n1) float64 CUDA tensors with slots rho, u, u1-u3, B1-B3, q~, dP~
(conserved: rho u^t, T^t_t + rho u^t, T^t_i, B^i gdet, q~ u^t gdet, dP~ u^t gdet); solve_norm and
solve_fail are (n3, n2, n1) float64 like the reference's fields.
"""
import ctypes as C

import numpy as np
import torch

from . import _lib
from .block import Block, Fields
from .spec import BlockSpec, EmhdSpec, ImplicitSpec

NSLOTS = 10


def build_connection(spec: BlockSpec):
    """Connection coefficients Gamma^a_bc at zone centres, (n2, n1, 4, 4, 4), via khb_build_connection."""
    lib = _lib.load()
    n3, n2, n1 = spec.shape
    conn = np.zeros((n2, n1, 4, 4, 4))
    _lib.check(lib.khb_build_connection(C.byref(spec.khb_coords()), C.byref(spec.khb_config()), spec.x1min,
                                        spec.x2min, spec.x3min, conn.ctypes.data_as(C.c_void_p)),
               "khb_build_connection")
    return conn


class ImplicitSolver:
    """EMHD sources and the per-zone implicit Newton solve on one block's context."""

    def __init__(self, block: Block, emhd: EmhdSpec, implicit: ImplicitSpec = None, conn=None):
        self.block = block
        self.lib = block.lib
        self.spec = block.spec
        self.emhd = emhd
        self.implicit = implicit or ImplicitSpec()
        self._e = emhd.to_struct()
        self._i = self.implicit.to_struct()
        # EMHD::eflag (emhd.cpp:162-165): the stability-limit bits of the last ImEx stage
        self.eflag = torch.zeros(self.spec.shape, dtype=torch.int32, device=block.device)
        conn = build_connection(self.spec) if conn is None else np.ascontiguousarray(conn, dtype=np.float64)
        _lib.check(self.lib.khb_set_connection(block.ctx, conn.ctypes.data_as(C.c_void_p)), "khb_set_connection")

    @property
    def nf(self):
        return self.emhd.nfvar

    def set_implicit(self, implicit: ImplicitSpec):
        self.implicit = implicit
        self._i = implicit.to_struct()

    def zeros(self):
        return torch.zeros((NSLOTS,) + self.spec.shape, dtype=torch.float64, device=self.block.device)

    def scalar_field(self):
        return torch.zeros(self.spec.shape, dtype=torch.float64, device=self.block.device)

    def ptou(self, P, U=None):
        U = self.zeros() if U is None else U
        _lib.check(self.lib.khb_emhd_ptou(self.block.ctx, C.byref(self._e), Fields(P).ref, Fields(U).ref,
                                          self.block.stream), "khb_emhd_ptou")
        return U

    def add_source(self, P, dUdt):
        _lib.check(self.lib.khb_emhd_add_source(self.block.ctx, C.byref(self._e), Fields(P).ref, Fields(dUdt).ref,
                                                self.block.stream), "khb_emhd_add_source")

    def step(self, P_full, U_full, P_sub, src, P_solver, solve_norm, solve_fail, dt):
        """Implicit::Step: P_solver (guess on entry) is updated in place; launches only."""
        _lib.check(self.lib.khb_implicit_step(self.block.ctx, C.byref(self._e), C.byref(self._i),
                                              Fields(P_full).ref, Fields(U_full).ref, Fields(P_sub).ref,
                                              Fields(src).ref, Fields(P_solver).ref,
                                              C.c_void_p(solve_norm.data_ptr()), C.c_void_p(solve_fail.data_ptr()),
                                              float(dt), self.block.stream), "khb_implicit_step")

    def stats(self):
        """(iterations, max solve_norm per iteration) of the last step (synchronizes)."""
        it = C.c_int32()
        mx = np.zeros(64)
        _lib.check(self.lib.khb_implicit_stats(self.block.ctx, C.byref(it), mx.ctypes.data_as(C.c_void_p),
                                               self.block.stream), "khb_implicit_stats")
        return it.value, mx[:it.value].copy()

    def jacobian(self, P_full, U_full, P_sub, src, P_solver, dt):
        """Residual (nf, ...) and Jacobian (nf*nf, ...) at P_solver."""
        nf = self.nf
        J = torch.zeros((nf * nf,) + self.spec.shape, dtype=torch.float64, device=self.block.device)
        r = torch.zeros((nf,) + self.spec.shape, dtype=torch.float64, device=self.block.device)
        _lib.check(self.lib.khb_implicit_jacobian(self.block.ctx, C.byref(self._e), C.byref(self._i),
                                                  Fields(P_full).ref, Fields(U_full).ref, Fields(P_sub).ref,
                                                  Fields(src).ref, Fields(P_solver).ref, float(dt),
                                                  C.c_void_p(J.data_ptr()), C.c_void_p(r.data_ptr()),
                                                  self.block.stream), "khb_implicit_jacobian")
        return J, r

    def get_flux(self, dir, P):
        """EMHD face fluxes along dir: (F (10, ...), ctop) as new device tensors."""
        _lib.check(self.lib.khb_get_flux_emhd(self.block.ctx, C.byref(self._e), dir, Fields(P).ref,
                                              self.block.stream), "khb_get_flux_emhd")
        F = self.zeros()
        ctop = self.scalar_field()
        _lib.check(self.lib.khb_copy_flux_emhd(self.block.ctx, dir, Fields(F).ref, C.c_void_p(ctop.data_ptr()),
                                               self.block.stream), "khb_copy_flux_emhd")
        return F, ctop

    def imex_stage(self, stage, dt, P_full, U_full, P_sub, U_sub, P_out, U_out, solve_norm, solve_fail,
                   fflag=None, eflag=None):
        """One ImEx stage (vl2): fluxes, flux fixes, sources, explicit B update, Newton solve, floors and
        EMHD limits, FixSolve, ghost zones, P -> U.  fflag/eflag (int32 fields) receive the floor and
        limit bits of the interior; the block's own fflag and this solver's eflag are used when the
        floors or the limits are on and none is given."""
        if fflag is None and self.block.spec.floors_on:
            fflag = self.block.fflag
        if eflag is None and self.emhd.stability_limits:
            eflag = self.eflag
        ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
        _lib.check(self.lib.khb_imex_stage_flags(self.block.ctx, C.byref(self._e), C.byref(self._i), stage,
                                                 float(dt), Fields(P_full).ref, Fields(U_full).ref,
                                                 Fields(P_sub).ref, Fields(U_sub).ref, Fields(P_out).ref,
                                                 Fields(U_out).ref, C.c_void_p(solve_norm.data_ptr()),
                                                 C.c_void_p(solve_fail.data_ptr()), ptr(fflag), ptr(eflag),
                                                 self.block.stream), "khb_imex_stage_flags")

    def imex_step(self, P, U, dt, solve_norm, solve_fail):
        """One vl2 ImEx step in place on (P, U) through an intermediate state."""
        P1, U1 = self.zeros(), self.zeros()
        P2, U2 = self.zeros(), self.zeros()
        self.imex_stage(1, dt, P, U, P, U, P1, U1, solve_norm, solve_fail)
        self.imex_stage(2, dt, P, U, P1, U1, P2, U2, solve_norm, solve_fail)
        P.copy_(P2)
        U.copy_(U2)

    def fix_solve(self, P, U, solve_fail):
        _lib.check(self.lib.khb_fix_solve(self.block.ctx, C.byref(self._e), Fields(P).ref, Fields(U).ref,
                                          C.c_void_p(solve_fail.data_ptr()), self.block.stream), "khb_fix_solve")

"""Checkpoint-and-recompute adjoint of a run of RK2 steps of one block (khb_adjoint_step).

A `Run` advances a Block over a fixed timestep sequence with khb_stage (stage 1 then stage 2, the
same launches as khb_step), keeping a copy of the state (P, U) every `checkpoint_every` steps and
evaluating the objective

    J = sum over steps n and stages s of (dt_n / 2) * sum_f weight[f] * F1[rho](P_{n,s})[f]
        + sum (Pw * P_N) + sum (Uw * U_N)

(the RK2-consistent mass through the x1 faces that `weight` selects, plus a linear functional of the
final state; each part optional).  `Run.adjoint` walks the segments between checkpoints backwards:
each segment is recomputed forward from its checkpoint with the states of its steps kept, then
khb_adjoint_step carries (Pbar, Ubar) back through its steps.  The result is the adjoint of the
initial (P_0, U_0); `Run.gradient_prims` adds (dU/dP)^T Ubar_0 for initial data given as primitives
with U_0 = U(P_0) (khb_adjoint_ptou).  Memory: one state per checkpoint plus one state per step of
the longest segment.

The timestep sequence is an input: the adjoint is that of the run at those dts (the CFL control
that chose them is not differentiated).  Zones whose inversion fails take their fixup (an average of
the neighbours) and are differentiated through it; `forward` counts them (`Run.failures`), since
the objective is not differentiable where a perturbation turns a failure into a success.
"""
import ctypes as C

import torch

from . import _lib
from .block import Block, Fields


class Run:
    def __init__(self, block: Block, dts, weight=None, Pw=None, Uw=None, checkpoint_every=20):
        self.b = block
        self.lib = block.lib
        self.dts = [float(x) for x in dts]
        self.K = max(1, int(checkpoint_every))
        self.weight = None if weight is None else torch.as_tensor(weight, dtype=torch.float64,
                                                                   device=block.device).contiguous()
        self.Pw, self.Uw = Pw, Uw
        self.Ps = torch.empty_like(block.P)
        self.Us = torch.empty_like(block.U)
        self.Psf, self.Usf = Fields(self.Ps), Fields(self.Us)
        self.checkpoints = []
        self.failures = 0

    # ------------------------------------------------------------- forward
    def _stage(self, stage, dt, Pin, Uin, U0, Pout, Uout):
        b = self.b
        _lib.check(self.lib.khb_stage(b.ctx, stage, dt, Pin.ref, Uin.ref, U0.ref, Pout.ref, Uout.ref,
                                      C.c_void_p(b.pflag.data_ptr()), C.c_void_p(b.fflag.data_ptr()), b.stream),
                   "khb_stage")

    def _mass_flux(self, J, scale):
        """J += scale * sum_f weight[f] * F1[rho][f] of the fluxes the last stage left in scratch."""
        if self.weight is not None and J is not None:
            _lib.check(self.lib.khb_flux_dot(self.b.ctx, 1, 0, C.c_void_p(self.weight.data_ptr()), float(scale),
                                             C.c_void_p(J.data_ptr()), self.b.stream), "khb_flux_dot")

    def _step(self, dt, fails=None, J=None):
        """One step in place on the block's (P, U), adding its objective contribution to J (a device
        double).  fails: a device counter that receives the number of failed inversions of both stages."""
        b = self.b
        self._stage(1, dt, b.Pf, b.Uf, b.Uf, self.Psf, self.Usf)
        if fails is not None:
            fails += (b.pflag != 0).sum()
        self._mass_flux(J, 0.5 * dt)
        self._stage(2, dt, self.Psf, self.Usf, b.Uf, b.Pf, b.Uf)
        if fails is not None:
            fails += (b.pflag != 0).sum()
        self._mass_flux(J, 0.5 * dt)

    def forward(self):
        """Run all steps from the block's current state; returns J (a Python float)."""
        b = self.b
        self.checkpoints = []
        fails = torch.zeros((), dtype=torch.int64, device=b.device)
        J = torch.zeros((), dtype=torch.float64, device=b.device)
        for n, dt in enumerate(self.dts):
            if n % self.K == 0:
                self.checkpoints.append((b.P.clone(), b.U.clone()))
            self._step(dt, fails, J)
        self.failures = int(fails.item())
        if self.Pw is not None:
            J = J + (self.Pw * b.P).sum()
        if self.Uw is not None:
            J = J + (self.Uw * b.U).sum()
        return float(J.item())

    # ------------------------------------------------------------- adjoint
    def adjoint(self):
        """(Pbar_0, Ubar_0): adjoint of the initial state (interior zones; ghosts zero)."""
        b = self.b
        Pbar = torch.zeros_like(b.P) if self.Pw is None else self.Pw.to(b.P).clone()
        Ubar = torch.zeros_like(b.U) if self.Uw is None else self.Uw.to(b.U).clone()
        Pbf, Ubf = Fields(Pbar), Fields(Ubar)
        wptr = C.c_void_p(self.weight.data_ptr()) if self.weight is not None else None
        nseg = len(self.checkpoints)
        for s in reversed(range(nseg)):
            n0 = s * self.K
            n1 = min(n0 + self.K, len(self.dts))
            # recompute the segment: states[m] is the state before step n0 + m, states[-1] after n1 - 1
            P0, U0 = self.checkpoints[s]
            b.P.copy_(P0)
            b.U.copy_(U0)
            states = [(P0.clone(), U0.clone())]
            for n in range(n0, n1):
                self._stage(1, self.dts[n], b.Pf, b.Uf, b.Uf, self.Psf, self.Usf)
                self._stage(2, self.dts[n], self.Psf, self.Usf, b.Uf, b.Pf, b.Uf)
                states.append((b.P.clone(), b.U.clone()))
            for n in reversed(range(n0, n1)):
                Pn, Un = states[n - n0]
                Pn1, _ = states[n - n0 + 1]
                Pnf, Unf, Pn1f = Fields(Pn), Fields(Un), Fields(Pn1)
                _lib.check(self.lib.khb_adjoint_step(b.ctx, self.dts[n], Pnf.ref, Unf.ref, Pn1f.ref, Pbf.ref,
                                                     Ubf.ref, wptr, 0.5 * self.dts[n], b.stream),
                           "khb_adjoint_step")
            del states
        # leave the block at the final state of the forward run
        if nseg:
            b.P.copy_(self.checkpoints[-1][0])
            b.U.copy_(self.checkpoints[-1][1])
            for n in range((nseg - 1) * self.K, len(self.dts)):
                self._step(self.dts[n])
        return Pbar, Ubar

    def gradient_prims(self, P0):
        """dJ/dP_0 for initial data P0 (device tensor) with U_0 = U(P_0): Pbar_0 + (dU/dP)^T Ubar_0."""
        Pbar, Ubar = self.adjoint()
        _lib.check(self.lib.khb_adjoint_ptou(self.b.ctx, Fields(P0).ref, Fields(Ubar).ref, Fields(Pbar).ref,
                                             self.b.stream), "khb_adjoint_ptou")
        return Pbar

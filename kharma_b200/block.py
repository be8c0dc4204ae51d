"""One meshblock on the GPU: device state, geometry, and the per-step calls through libkhb.

The state lives in torch CUDA tensors (torch is used only for device memory and streams):
P and U are (nvar, n3, n2, n1) float64, pflag and fflag (n3, n2, n1) int32.  Each variable
is handed to the C ABI as its own pointer, as Parthenon's per-variable allocations would be.
"""
import ctypes as C

import numpy as np
import torch

from . import _lib
from .spec import BlockSpec


def build_geometry(spec: BlockSpec):
    """GRCoordinates caches for the block (host numpy arrays), via khb_build_geometry."""
    lib = _lib.load()
    n3, n2, n1 = spec.shape
    G1, G2 = n1 + 1, n2 + 1
    geom = {
        "gcov": np.zeros((7, G2, G1, 4, 4)),
        "gcon": np.zeros((7, G2, G1, 4, 4)),
        "gdet": np.zeros((7, G2, G1)),
        "gdet_conn": np.zeros((n2, n1, 4, 4, 4)),
        "r_center": np.zeros((n2, n1)),
    }
    cfg = spec.khb_config()
    cs = spec.khb_coords()
    ptr = lambda a: a.ctypes.data_as(C.c_void_p)
    _lib.check(lib.khb_build_geometry(C.byref(cs), C.byref(cfg), spec.x1min, spec.x2min, spec.x3min,
                                      ptr(geom["gcov"]), ptr(geom["gcon"]), ptr(geom["gdet"]),
                                      ptr(geom["gdet_conn"]), ptr(geom["r_center"])), "khb_build_geometry")
    return geom


class Fields:
    """Per-variable device pointers of a (nvar, n3, n2, n1) float64 CUDA tensor."""

    def __init__(self, t):
        self.t = t
        self.s = _lib.KhbFields()
        for p in range(t.shape[0]):
            self.s.v[p] = t[p].data_ptr()

    @property
    def ref(self):
        return C.byref(self.s)


class Block:
    def __init__(self, spec: BlockSpec, geometry=None, device="cuda"):
        if not torch.cuda.is_available():
            raise RuntimeError("kharma_b200.Block needs a CUDA device")
        self.lib = _lib.load()
        self.spec = spec
        self.device = torch.device(device)
        cfg = spec.khb_config()
        ctx = C.c_void_p()
        _lib.check(self.lib.khb_create(C.byref(cfg), C.byref(ctx)), "khb_create")
        self.ctx = ctx
        self.geom = geometry if geometry is not None else build_geometry(spec)
        self._set_geometry(self.geom)
        shape = (spec.nvar,) + spec.shape
        self.P = torch.zeros(shape, dtype=torch.float64, device=self.device)
        self.U = torch.zeros(shape, dtype=torch.float64, device=self.device)
        self.pflag = torch.zeros(spec.shape, dtype=torch.int32, device=self.device)
        self.fflag = torch.zeros(spec.shape, dtype=torch.int32, device=self.device)
        self.Pf = Fields(self.P)
        self.Uf = Fields(self.U)
        # B_CT: the face-centred field sqrt(-g) B^d on the x_d faces, (3, n3, n2, n1)
        self.ct = spec.b_ct != "none"
        if self.ct:
            self.Bf = torch.zeros((3,) + spec.shape, dtype=torch.float64, device=self.device)
            self.Bff = Fields(self.Bf)

    def _set_geometry(self, g):
        arrs = [np.ascontiguousarray(g[k], dtype=np.float64) for k in ("gcov", "gcon", "gdet", "gdet_conn", "r_center")]
        ptrs = [a.ctypes.data_as(C.c_void_p) for a in arrs]
        _lib.check(self.lib.khb_set_geometry(self.ctx, *ptrs), "khb_set_geometry")

    def __del__(self):
        try:
            if getattr(self, "ctx", None):
                self.lib.khb_destroy(self.ctx)
                self.ctx = None
        except Exception:
            pass

    @property
    def stream(self):
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    # ------------------------------------------------------------- state
    def set_prims(self, P_host, faces=None):
        """Load primitives (interior at least), fill ghost zones and set U = U(P) everywhere.  A B_CT
        block also sets its face field: `faces` (3, n3, n2, n1) if given, else interpolated from the
        zone B (khb_ct_faces_from_prims); the zone B is then rebuilt from the faces."""
        self.P.copy_(torch.as_tensor(P_host, dtype=torch.float64))
        # ghost B_P is rebuilt from B_U by the boundary call: seed B_U = B_P sqrt(-g) first
        self.ptou()
        self.boundaries()
        if self.ct:
            if faces is None:
                _lib.check(self.lib.khb_ct_faces_from_prims(self.ctx, self.Pf.ref, self.Bff.ref, self.stream),
                           "khb_ct_faces_from_prims")
            else:
                self.Bf.copy_(torch.as_tensor(faces, dtype=torch.float64))
            _lib.check(self.lib.khb_ct_utop(self.ctx, self.Bff.ref, self.Pf.ref, self.Uf.ref, self.stream), "khb_ct_utop")
            _lib.check(self.lib.khb_ct_boundaries(self.ctx, self.Pf.ref, self.Uf.ref, self.Bff.ref, self.stream),
                       "khb_ct_boundaries")
        self.ptou()

    def ptou(self):
        _lib.check(self.lib.khb_ptou(self.ctx, self.Pf.ref, self.Uf.ref, self.stream), "khb_ptou")

    def boundaries(self):
        _lib.check(self.lib.khb_boundaries(self.ctx, self.Pf.ref, self.Uf.ref, self.stream), "khb_boundaries")

    # ------------------------------------------------------------- stepping
    def step(self, dt):
        """One RK2 step in place (launch only)."""
        if self.ct:
            _lib.check(self.lib.khb_ct_step(self.ctx, float(dt), self.Pf.ref, self.Uf.ref, self.Bff.ref,
                                            C.c_void_p(self.pflag.data_ptr()), C.c_void_p(self.fflag.data_ptr()),
                                            self.stream), "khb_ct_step")
            return
        _lib.check(self.lib.khb_step(self.ctx, float(dt), self.Pf.ref, self.Uf.ref,
                                     C.c_void_p(self.pflag.data_ptr()), C.c_void_p(self.fflag.data_ptr()),
                                     self.stream), "khb_step")

    def min_ndt(self):
        """Minimum zone timestep of the last step's second stage (synchronizes)."""
        out = C.c_double()
        _lib.check(self.lib.khb_get_min_ndt(self.ctx, C.byref(out), self.stream), "khb_get_min_ndt")
        return out.value

    def max_divb(self):
        out = C.c_double()
        if self.ct:
            _lib.check(self.lib.khb_ct_max_divb(self.ctx, self.Bff.ref, C.byref(out), self.stream), "khb_ct_max_divb")
            return out.value
        _lib.check(self.lib.khb_max_divb(self.ctx, self.Uf.ref, C.byref(out), self.stream), "khb_max_divb")
        return out.value

    def set_tuning(self, key, value):
        _lib.check(self.lib.khb_set_tuning(self.ctx, key.encode(), int(value)), "khb_set_tuning")

    def launch_count(self):
        return int(self.lib.khb_launch_count(self.ctx))

    # ------------------------------------------------------------- package-level calls
    def get_flux(self, dir, P=None):
        Pf = Fields(P) if P is not None else self.Pf
        _lib.check(self.lib.khb_get_flux(self.ctx, dir, Pf.ref, self.stream), "khb_get_flux")

    def fix_flux(self):
        _lib.check(self.lib.khb_fix_flux(self.ctx, self.stream), "khb_fix_flux")

    def flux_ct(self):
        _lib.check(self.lib.khb_flux_ct(self.ctx, self.stream), "khb_flux_ct")

    def copy_flux(self, dir):
        F = torch.zeros_like(self.U)
        ctop = torch.zeros(self.spec.shape, dtype=torch.float64, device=self.device)
        Ff = Fields(F)
        _lib.check(self.lib.khb_copy_flux(self.ctx, dir, Ff.ref, C.c_void_p(ctop.data_ptr()), self.stream),
                   "khb_copy_flux")
        return F, ctop

    def utop(self, U, P, pflag, fflag):
        _lib.check(self.lib.khb_utop(self.ctx, Fields(U).ref, Fields(P).ref, C.c_void_p(pflag.data_ptr()),
                                     C.c_void_p(fflag.data_ptr()), self.stream), "khb_utop")

    def apply_floors(self, P, U, pflag, fflag):
        _lib.check(self.lib.khb_apply_floors(self.ctx, Fields(P).ref, Fields(U).ref, C.c_void_p(pflag.data_ptr()),
                                             C.c_void_p(fflag.data_ptr()), self.stream), "khb_apply_floors")

    def fix_utop(self, P, U, pflag):
        _lib.check(self.lib.khb_fix_utop(self.ctx, Fields(P).ref, Fields(U).ref, C.c_void_p(pflag.data_ptr()),
                                         self.stream), "khb_fix_utop")


class Driver:
    """Step loop with the reference's timestep schedule.

    The first step uses dt_start (= dt_min by default, grmhd.cpp:283-288).  After each step
    GRMHD::EstimateTimestep gives clip(cfl * min_zone_dt, dt_min, max_dt_increase * dt) and
    KHARMADriver::SetGlobalTimeStep takes min(2 dt, that) (kharma_driver.cpp:439-460).
    """

    def __init__(self, block: Block, dt_start=None):
        self.block = block
        self.dt = block.spec.dt_min if dt_start is None else dt_start
        self.t = 0.0
        self.nstep = 0

    def next_dt(self, min_ndt, dt):
        s = self.block.spec
        ndt = min(max(min_ndt * s.cfl, s.dt_min), s.max_dt_increase * dt)
        return min(2.0 * dt, ndt)

    def step(self, dt=None):
        dt = self.dt if dt is None else dt
        self.block.step(dt)
        mn = self.block.min_ndt()
        self.t += dt
        self.nstep += 1
        self.dt = self.next_dt(mn, dt)
        return dt, mn


class DeviceDriver:
    """The reference's timestep schedule (as Driver) kept on the device: each step reads its dt from
    device memory and sets the next one there (khb_set_timestep / khb_step_device_dt), so a step
    needs no host synchronisation and can be replayed from a CUDA graph (khb_step_graph, on the
    block's current stream, which must not be the default stream)."""

    def __init__(self, block: Block, dt_start=None, graph=True):
        self.block = block
        s = block.spec
        dt0 = s.dt_min if dt_start is None else dt_start
        _lib.check(block.lib.khb_set_timestep(block.ctx, float(dt0), s.cfl, s.dt_min, s.max_dt_increase),
                   "khb_set_timestep")
        self.graph = graph
        self.nstep = 0

    def step(self):
        b = self.block
        fn = b.lib.khb_step_graph if self.graph else b.lib.khb_step_device_dt
        _lib.check(fn(b.ctx, b.Pf.ref, b.Uf.ref, C.c_void_p(b.pflag.data_ptr()), C.c_void_p(b.fflag.data_ptr()),
                      b.stream), "khb_step_graph" if self.graph else "khb_step_device_dt")
        self.nstep += 1

    def step_host(self, hP):
        """One step of the host-resident primitives hP ((nvar, n3, n2, n1) float64, pinned CPU tensor),
        in place (khb_step_host: P in, U = U(P), the graph step, P out).  Launches and copies only."""
        b = self.block
        ptrs = (C.c_void_p * b.spec.nvar)(*[hP[p].data_ptr() for p in range(b.spec.nvar)])
        _lib.check(b.lib.khb_step_host(b.ctx, ptrs, b.Pf.ref, b.Uf.ref, C.c_void_p(b.pflag.data_ptr()),
                                       C.c_void_p(b.fflag.data_ptr()), b.stream), "khb_step_host")
        self.nstep += 1

    def step_host_interior(self, hP):
        """step_host for host primitives holding the interior only ((nvar, nx3, nx2, nx1) float64,
        pinned, contiguous per variable): khb_step_host_interior rebuilds the ghost zones on the device."""
        b = self.block
        ptrs = (C.c_void_p * b.spec.nvar)(*[hP[p].data_ptr() for p in range(b.spec.nvar)])
        _lib.check(b.lib.khb_step_host_interior(b.ctx, ptrs, b.Pf.ref, b.Uf.ref, C.c_void_p(b.pflag.data_ptr()),
                                                C.c_void_p(b.fflag.data_ptr()), b.stream), "khb_step_host_interior")
        self.nstep += 1

    def timestep(self):
        """(next dt, time, dt of the last step); synchronizes."""
        dt, t, last = C.c_double(), C.c_double(), C.c_double()
        _lib.check(self.block.lib.khb_get_timestep(self.block.ctx, C.byref(dt), C.byref(t), C.byref(last),
                                                   self.block.stream), "khb_get_timestep")
        return dt.value, t.value, last.value

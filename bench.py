#!/usr/bin/env python
"""Zone-cycles/s of KHARMA's per-step GRMHD path on B200 (one 128^3 FM-torus meshblock per GPU).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl khb|reference]

One step = one full RK2 step (both stages: face fluxes in 3 directions, flux-CT, divergence,
geometric source, RK update, 1D_W inversion, floors, fixups, boundaries, CFL reduction) of the
plain FP64 path on a 128x128x128 funky-MKS torus (a = 0.9375, r_in = 6, r_max = 12, gamma 13/9,
SANE field at beta_min = 100, MC reconstruction, LLF, flux-CT, drift-frame floors).  One
zone-cycle is one interior zone advanced one RK2 step.  Synthetic data: the initial state is built
by kharma_b200.problems.fm_torus from a seeded RNG (u jitter +-4%).

For N > 1 (torchrun) the torus is n1 x n2 x (128 N) zones split into x3 slabs, one 128^3 slab per
rank (weak scaling): per stage the ranks exchange one plane of fluid primitives and pflag before
the inversion fixups and 4 planes of every primitive and conserved variable after the physical
boundaries (NCCL point-to-point), and reduce the timestep (allreduce MIN) every step; time = max
over ranks.

--impl reference times the reference algorithm on the host cores: the CPU oracle (a restatement of
KHARMA's hot path; kharma.host itself cannot be built here), on a bounded slab of the same torus.
"""
import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "zone-cycles/s at 128^3 torus: FP64 plain vs FP32-flux form; % of HBM roofline"
UNIT = "zone-cycles/s"
B_ALG_PER_ZC = 72 * 8          # algorithmic HBM bytes per zone-cycle, 72 * nvar (nvar = 8)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="khb", choices=["khb", "reference"])
    ap.add_argument("--size", default="128,128,128")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp32", action="store_true")
    ap.add_argument("--no-kernel-times", action="store_true")
    ap.add_argument("--no-emhd", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--form", default="fp64", choices=["fp64", "fp32_flux"],
                    help="arithmetic of the timed step (the FP32-flux form is also measured beside FP64 by default)")
    ap.add_argument("--slab-path", action="store_true",
                    help="at N = 1, step the block through the x3-slab path (one slab, local exchange)")
    ap.add_argument("--adjoint-only", action="store_true",
                    help="time the differentiation form (forward + checkpointed adjoint) and print only that")
    ap.add_argument("--adjoint-shape", default="192,200,20,64",
                    help="differentiation form: block size n (n^3), steps, checkpoint spacing, FD directions")
    ap.add_argument("--adjoint-workload", default="torus", choices=["torus", "bondi"],
                    help="differentiation form: the floored FMKS torus (default) or a smooth Bondi block")
    ap.add_argument("--emhd-only", action="store_true",
                    help="run only the implicit EMHD Newton measurement and print its JSON object")
    return ap.parse_args()


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def detail(name, obj):
    """A bulky secondary measurement on its own stdout line, ahead of the final JSON line."""
    print(f"detail {name}: " + json.dumps(obj), flush=True)


def compact(obj, digits=6):
    """obj with every float rounded to `digits` significant digits (keeps the final line short)."""
    if isinstance(obj, float):
        return float(f"{obj:.{digits}g}")
    if isinstance(obj, dict):
        return {k: compact(v, digits) for k, v in obj.items()}
    if isinstance(obj, (list, tuple)):
        return [compact(v, digits) for v in obj]
    return obj


def profile_traffic(kernel, size, form):
    """DRAM bytes per launch of `kernel` (dram__bytes_read.sum + dram__bytes_write.sum) from the
    committed ncu summary of this workload, which states it on a line
    `traffic_per_launch_bytes: <kernel> <form> <n1>x<n2>x<n3> <bytes>`; None when no summary covers it."""
    want = (kernel, form, "x".join(str(x) for x in size))
    pdir = os.path.join(ROOT, "profiles")
    try:
        names = sorted(os.listdir(pdir))
    except OSError:
        return None, None
    for name in names:
        if not name.endswith(".md"):
            continue
        with open(os.path.join(pdir, name)) as f:
            for ln in f:
                t = ln.strip().strip("`").split()
                if len(t) == 5 and t[0] == "traffic_per_launch_bytes:" and tuple(t[1:4]) == want:
                    return float(t[4]), "profiles/" + name
    return None, None


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_state(spec):
    from kharma_b200 import problems
    from kharma_b200.block import build_geometry
    geom = build_geometry(spec)
    P0 = problems.fm_torus(spec, geom, seed=1234)
    return geom, P0


# ----------------------------------------------------------------------------------- CPU side
def _oracle_block(n1, n2, n3):
    """The oracle (the CPU restatement of the reference hot path) on the benchmark block."""
    # the OpenMP runtime reads OMP_PROC_BIND when the oracle library is first loaded
    os.environ.setdefault("OMP_PROC_BIND", "close")
    from kharma_b200 import problems
    from kharma_b200.spec import torus_spec
    from oracle import orc
    spec = torus_spec(n1, n2, n3)
    o = orc.Oracle(spec)
    P, U = o.init_state(problems.fm_torus(spec, o.geometry(), seed=1234))
    return orc, o, spec, P, U


def _host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def cpu_baseline_block(n1, n2, n3, runs=5):
    """The oracle on the same n1 x n2 x n3 block as the GPU arm: one warm-up step, then `runs` RK2
    steps timed one by one on all host threads (median reported), then one step on one thread."""
    orc, o, spec, P, U = _oracle_block(n1, n2, n3)
    threads = orc.set_threads(0)
    dt = spec.dt_min
    _, _, dt, _ = o.step(P, U, dt)
    per = []
    for _ in range(runs):
        t0 = time.perf_counter()
        _, _, dt, _ = o.step(P, U, dt)
        per.append(time.perf_counter() - t0)
    zones = n1 * n2 * n3
    med = statistics.median(per)
    orc.set_threads(1)
    t0 = time.perf_counter()
    o.step(P, U, dt)
    one = time.perf_counter() - t0
    orc.set_threads(threads)
    return {"value": zones / med, "unit": UNIT, "cores": threads, "kind": "port",
            "single_thread_value": zones / one,
            "sample": f"oracle port, same {n1}x{n2}x{n3} block, {threads} threads ({_cpu_model()}): median of {runs} "
                      f"RK2 steps after 1 warm-up; 1 thread: {one:.2f} s/step"}


def reference_arm(args, rank, world):
    """The reference's algorithm on the host cores: the oracle port (kharma.host cannot be built), on
    the GPU arm's block and metric, all host threads, W warm-up steps then K timed RK2 steps."""
    if rank != 0:
        return
    n1, n2, n3 = [int(x) for x in args.size.split(",")]
    orc, o, spec, P, U = _oracle_block(n1, n2, n3)
    threads = orc.set_threads(0)
    dt = spec.dt_min
    for _ in range(args.warmup):
        _, _, dt, _ = o.step(P, U, dt)
    per = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _, _, dt, _ = o.step(P, U, dt)
        per.append(time.perf_counter() - t0)
    el = sum(per)
    zones = n1 * n2 * n3
    v = zones * args.steps / el
    sample = (f"oracle port of the reference hot path, {threads} OpenMP threads ({_cpu_model()}), the same "
              f"{n1}x{n2}x{n3} block, {args.steps} RK2 steps after {args.warmup} warm-up; median step "
              f"{statistics.median(per):.3f} s")
    out = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * el / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic", "config": {"workload": f"FM torus FMKS {n1}x{n2}x{n3} one meshblock",
                                            "recon": "linear_mc", "flux": "llf", "b_field": "flux_ct",
                                            "inverter": "onedw", "floors": "drift"},
           "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                            "median_step_value": zones / statistics.median(per)},
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


# ----------------------------------------------------------------------------------- GPU side
def kernel_times(block, spec, nsteps=3):
    """Per-kernel CUDA-event timing of the stage pieces on the launching stream."""
    import torch
    from kharma_b200 import _lib
    lib = block.lib
    st = block.stream
    cur = torch.cuda.current_stream()
    nv = spec.nvar
    Ps, Us = block.Pf, block.Uf
    P1 = torch.empty_like(block.P)
    U1 = torch.empty_like(block.U)
    from kharma_b200.block import Fields
    P1f, U1f = Fields(P1), Fields(U1)
    pf = C.c_void_p(block.pflag.data_ptr())
    ff = C.c_void_p(block.fflag.data_ptr())
    names = []
    times = {}

    def timed(name, fn):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(cur)
        _lib.check(fn(), name)
        e1.record(cur)
        names.append((name, e0, e1))

    dt = 1e-4
    for _ in range(nsteps):
        for stage, (Pin, Uin, Pout, Uout) in ((1, (Ps, Us, P1f, U1f)), (2, (P1f, U1f, Ps, Us))):
            for d in range(1, spec.ndim + 1):
                timed(f"k_flux_x{d}", lambda d=d, Pin=Pin: lib.khb_get_flux(block.ctx, d, Pin.ref, st))
            timed("k_fix_flux", lambda: lib.khb_fix_flux(block.ctx, st))
            timed("k_zone", lambda stage=stage, Pin=Pin, Uin=Uin, Pout=Pout, Uout=Uout:
                  lib.khb_zone_pass(block.ctx, stage, dt, Pin.ref, Uin.ref, Us.ref, Pout.ref, Uout.ref, pf, ff, st))
            timed("k_fixup", lambda Pout=Pout, Uout=Uout: lib.khb_fix_utop_list(block.ctx, Pout.ref, Uout.ref, pf, st))
            timed("k_boundaries", lambda Pout=Pout, Uout=Uout: lib.khb_boundaries(block.ctx, Pout.ref, Uout.ref, st))
    torch.cuda.synchronize()
    for name, e0, e1 in names:
        times.setdefault(name, []).append(e0.elapsed_time(e1))
    return {k: (float(np.mean(v)), len(v) // nsteps) for k, v in times.items()}


def emhd_newton(n=128, reps=3):
    """Per-zone implicit EMHD Newton solve (Implicit::Step) on the conducting atmosphere at n^3:
    forward-difference Jacobian (the reference's) vs the exact tangent Jacobian.  Each form solves
    the same system to a maximum residual of 1e-10 relative to max|U|/dt; reported are the Newton
    iterations the device-side stopping test took and the CUDA-event time of the whole solve."""
    import torch
    from kharma_b200 import problems
    from kharma_b200.block import Block, build_geometry
    from kharma_b200.emhd import ImplicitSolver
    from kharma_b200.spec import EmhdSpec, ImplicitSpec, atmosphere_spec
    spec = atmosphere_spec(n, n, n)
    emhd = EmhdSpec(closure_type="kappa_eta", higher_order_terms=True, tau=1.0, kappa=0.1, eta=0.1)
    prof = np.load(os.path.join(ROOT, "tests", "golden", "atmosphere_profiles.npz"))
    prof = {k: prof["%s_%d" % (k, n)] for k in ("rCoords", "rho", "u", "phi")}
    geom = build_geometry(spec)
    P = problems.conducting_atmosphere(spec, geom, emhd, prof, jitter=1e-3, seed=1234)
    b = Block(spec, geometry=geom)
    sol = ImplicitSolver(b, emhd)
    dt = 0.1
    Pd = torch.tensor(P, dtype=torch.float64, device="cuda")
    Ud = sol.ptou(Pd)
    Sd = torch.zeros_like(Pd)
    sol.add_source(Pd, Sd)
    # stand-in for the flux divergence of the perturbed atmosphere: seeded noise of 1e-3 |U|/dt
    g = torch.Generator(device="cuda").manual_seed(1234)
    Sd += (2 * torch.rand(Pd.shape, generator=g, device="cuda", dtype=torch.float64) - 1) * 1e-3 * Ud.abs() / dt
    k, j, i = spec.interior
    tol = 1e-10 * float(Ud[:, k, j, i].abs().max()) / dt
    out = {"workload": f"conducting atmosphere (KS a=0, MKS hslope 1, r 200-300) {n}^3, 10 primitives, "
                       f"kappa_eta closure tau=1 kappa=eta=0.1, higher-order terms; dt={dt}",
           "tolerance_abs": tol, "tolerance_rel": 1e-10, "zones": n ** 3}
    Psol = torch.empty_like(Pd)
    norm = sol.scalar_field()
    fail = sol.scalar_field()
    scale = float(Ud[:, k, j, i].abs().max()) / dt

    def solve(jac, rel, max_iter=16):
        sol.set_implicit(ImplicitSpec(min_nonlinear_iter=1, max_nonlinear_iter=max_iter, rootfind_tol=rel * scale,
                                      jacobian=jac))
        times = []
        for r in range(reps + 1):
            Psol.copy_(Pd)
            norm.zero_()
            fail.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            sol.step(Pd, Ud, Pd, Sd, Psol, norm, fail, dt)
            e1.record()
            torch.cuda.synchronize()
            if r:
                times.append(e0.elapsed_time(e1))
        it, mx = sol.stats()
        ms = float(np.median(times))
        return {"iterations": it, "ms_per_solve": ms, "ms_per_iteration": ms / max(it, 1),
                "zone_iterations_per_s": n ** 3 * it / (ms / 1000.0),
                "max_norm_per_iteration": [float(x) for x in mx],
                "failed_zones": int((fail[k, j, i] == 1).sum())}

    for jac in ("fd", "exact"):
        out[jac] = solve(jac, 1e-10)
    out["exact_vs_fd_wall_time"] = out["fd"]["ms_per_solve"] / out["exact"]["ms_per_solve"]
    # iterations and time to tolerance over a sweep of relative tolerances (max residual norm over
    # max|U|/dt), and at the reference's own convention: an absolute rootfind_tol of 1e-12 on the
    # zone's residual L2 norm (implicit.cpp:101, 502-554)
    sweep = {}
    for rel in (1e-8, 1e-9, 1e-10, 1e-11, 1e-12, 1e-13):
        sweep["%.0e" % rel] = {jac: solve(jac, rel) for jac in ("fd", "exact")}
    # the reference's defaults: at most 3 iterations to an absolute 1e-12, which lies below this state's
    # round-off floor of the residual, so both forms stop at 3: compared is the residual they reach
    sweep["abs_1e-12_max3"] = {jac: solve(jac, 1e-12 / scale, max_iter=3) for jac in ("fd", "exact")}
    out["sweep"] = {k: {jac: {"iterations": v[jac]["iterations"], "ms_per_solve": round(v[jac]["ms_per_solve"], 3),
                              "final_max_norm": v[jac]["max_norm_per_iteration"][-1],
                              "failed_zones": v[jac]["failed_zones"]} for jac in v} for k, v in sweep.items()}
    return out


def emhd_summary(e):
    """The implicit-solve figures the final line carries: iterations and ms per solve to 1e-10 (relative)
    and over the tolerance sweep, forward-difference vs exact Jacobian."""
    return {"tol_rel": 1e-10, "fd_iterations": e["fd"]["iterations"], "exact_iterations": e["exact"]["iterations"],
            "fd_ms": round(e["fd"]["ms_per_solve"], 3), "exact_ms": round(e["exact"]["ms_per_solve"], 3),
            "exact_vs_fd_wall_time": round(e["exact_vs_fd_wall_time"], 3),
            "sweep_iterations_fd_exact": {k: [v["fd"]["iterations"], v["exact"]["iterations"]]
                                          for k, v in e["sweep"].items()},
            "ref_defaults_final_norm_fd_exact": [e["sweep"]["abs_1e-12_max3"][j]["final_max_norm"] for j in ("fd", "exact")]}


def batching(steps=20, warm=3):
    """The batching form: the 184-block three-level Bondi mesh (8 x 64^3, 48 x 32^3, 128 x 16^3 zones,
    KS a = 0, MKS, WENO5, LLF, hydro) stepped through the plain per-block launch path (khb_step per
    block), the batched path (one launch per kernel per stage), and its CUDA-graph replay after the
    autotuner has chosen the tile shapes; FP64 and FP32-flux.  CUDA events on the batch's stream."""
    import torch
    from kharma_b200.batch import Batch, bondi_smr_layout

    def timed(fn, n):
        s = torch.cuda.current_stream()
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(n):
            fn()
        e1.record(s)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    out = {"workload": "Bondi (r_s = 8, mdot = 1, gamma 5/3) on a 3-level static-refined mesh of 184 blocks: "
                       "8 x 64^3, 48 x 32^3, 128 x 16^3 zones, KS a=0 MKS, WENO5, LLF, hydro; ghost zones "
                       "hold the analytic solution (blocks advance independently)"}
    dt = 1e-3
    for prec in ("fp64", "fp32_flux"):
        b = Batch(bondi_smr_layout(precision=prec))
        zones = b.zones
        r = {"zones": zones}
        with torch.cuda.stream(b.torch_stream):
            r["per_block_ms_per_step"] = timed(lambda: b.step_per_block(dt), max(3, steps // 4))
            r["batched_ms_per_step"] = timed(lambda: b.step(dt), steps)
            tune, pers = b.autotune(3)
            plan = b.plan()
            r["autotune"] = {"planes_per_cta": tune, "persistent": pers, "plan": plan}
            # both launch plans with the tuned tile shapes: one launch per kernel per stage, and three
            for p in (1 - plan, plan):
                b.set_plan(p)
                l0 = b.launch_count()
                r[f"graph_ms_per_step_plan{p}"] = timed(lambda: b.step_graph(dt), steps)
                r[f"launches_per_step_plan{p}"] = (b.launch_count() - l0) / (steps + warm)
            r["graph_ms_per_step"] = r[f"graph_ms_per_step_plan{plan}"]
            r["launches_per_step"] = r[f"launches_per_step_plan{plan}"]
        for k in ("per_block", "batched", "graph"):
            r[k + "_zone_cycles_per_s"] = zones / (r[k + "_ms_per_step"] / 1000.0)
        r["speedup_graph_vs_per_block"] = r["per_block_ms_per_step"] / r["graph_ms_per_step"]
        out[prec] = r
        del b
        torch.cuda.empty_cache()
    out["smr_mesh"] = batching_mesh(steps, warm)
    return out


def batching_mesh(steps=20, warm=3):
    """The batching form's problem on a conforming three-level SMR mesh with the ghost exchange and
    flux correction between blocks (Parthenon meshes have one block size): Bondi in spherical KS
    (a = 0, MKS), r in [3, 30], 4 x 4 x 2 root blocks of 32^3, the central 2 x 2 (x 2) roots refined
    and the 2 x 2 (x 4) level-1 blocks away from level 0 refined again (24 + 48 + 128 = 200 blocks),
    outflow x1, reflecting x2, periodic x3, WENO5, LLF, FP64, the kharma driver's exchange; the
    autotuned CUDA-graph step against the blocks stepped one after another with khb_step (no
    exchange, so a lower bound for a per-block path).  CUDA events on the batch's stream."""
    import numpy as np
    import torch
    from kharma_b200 import problems
    from kharma_b200.block import build_geometry
    from kharma_b200.mesh import SMRMesh, smr_batch
    from kharma_b200.spec import bondi_spec

    ks = bondi_spec(32, 32, 32, float(np.log(3.0)), float(np.log(30.0)), 0.0, 1.0, 0.0, 2 * np.pi,
                    bc=("outflow", "outflow", "reflecting", "reflecting", "periodic", "periodic"))
    refine = ([(i, j, k) for i in (1, 2) for j in (1, 2) for k in (0, 1)] +
              [(1, (i, j, k)) for i in (3, 4) for j in (3, 4) for k in range(4)])
    mesh = SMRMesh(ks, (4, 4, 2), (32, 32, 32), refine=refine)
    b = smr_batch(mesh, lambda sp: problems.bondi(sp, build_geometry(sp)))
    dt = 1e-3

    def timed(fn, n):
        with torch.cuda.stream(b.torch_stream):
            for _ in range(warm):
                fn()
            torch.cuda.synchronize()
            l0 = b.launch_count()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(b.torch_stream)
            for _ in range(n):
                fn()
            e1.record(b.torch_stream)
            torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n, (b.launch_count() - l0) / n

    per_block, _ = timed(lambda: b.step_per_block(dt), max(3, steps // 4))
    with torch.cuda.stream(b.torch_stream):
        tune, pers = b.autotune(3)
    ms, launches = timed(lambda: b.step_graph(dt), steps)
    out = {"workload": f"Bondi in spherical KS (a=0, MKS), r 3-30, 3-level SMR mesh of {len(mesh.blocks)} blocks of "
                       f"32^3 (24 + 48 + 128), {mesh.zones:,} zones, WENO5, LLF, FP64, outflow/reflecting/periodic "
                       f"faces, kharma driver exchange",
           "ghost_entries": int(len(mesh.tables()[0])),
           "graph_ms_per_step": ms, "zone_cycles_per_s": mesh.zones / (ms / 1000.0), "launches_per_step": launches,
           "autotune": {"planes_per_cta": tune, "persistent": pers, "plan": b.plan()},
           "per_block_no_exchange_ms_per_step": per_block,
           "speedup_graph_vs_per_block": per_block / ms}
    del b
    torch.cuda.empty_cache()
    return out


def smr_form(steps=20, warm=3):
    """Static mesh refinement through the batch: a 4 x 4 x 4 root grid of 32^3 hydro blocks on the
    periodic unit box with the central 2 x 2 x 2 roots refined (56 coarse + 64 fine blocks, 3.9M
    zones), entropy wave, linear MC, LLF, FP64, fixed dt; the CUDA-graph step with the ghost exchange
    and flux correction, against the same blocks stepped without the mesh tables (ghost zones then
    carry over unchanged).  CUDA events on the batch's stream."""
    import numpy as np
    import torch
    from kharma_b200 import problems
    from kharma_b200.mesh import SMRMesh, smr_batch
    from kharma_b200.spec import BlockSpec

    base = BlockSpec(nx1=32, nx2=32, nx3=32, x1min=0., x1max=1., x2min=0., x2max=1., x3min=0., x3max=1.,
                     gam=5. / 3., nvar=5, recon="linear_mc")
    refine = [(i, j, k) for i in (1, 2) for j in (1, 2) for k in (1, 2)]
    mesh = SMRMesh(base, (4, 4, 4), (32, 32, 32), refine=refine)
    b = smr_batch(mesh, lambda sp: problems.entropy_wave(sp, amp=0.1))
    dt = 0.3 * min(blk.spec.dx[0] for blk in mesh.blocks)
    ghost, n_first, flux = mesh.tables()

    def timed(n):
        with torch.cuda.stream(b.torch_stream):
            for _ in range(warm):
                b.step_graph(dt)
            torch.cuda.synchronize()
            l0 = b.launch_count()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(b.torch_stream)
            for _ in range(n):
                b.step_graph(dt)
            e1.record(b.torch_stream)
            torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n, (b.launch_count() - l0) / n

    ms, launches = timed(steps)
    b.set_plan(1)
    ms_f, launches_f = timed(steps)
    b.set_plan(0)
    out = {"workload": "periodic box, 4x4x4 root blocks of 32^3 with the central 2x2x2 refined: 56 coarse + 64 fine "
                       "blocks, 3,932,160 zones, hydro entropy wave, linear MC, LLF, FP64",
           "ghost_entries": int(len(ghost)), "flux_entries": int(len(flux)),
           "graph_ms_per_step": ms, "zone_cycles_per_s": mesh.zones / (ms / 1000.0), "launches_per_step": launches,
           "fused_plan": {"graph_ms_per_step": ms_f, "zone_cycles_per_s": mesh.zones / (ms_f / 1000.0),
                          "launches_per_step": launches_f}}
    empty = np.zeros((0, 6), dtype=np.int32)
    b.set_mesh(empty, 0, empty)
    ms0, _ = timed(steps)
    out["without_mesh_ms_per_step"] = ms0
    out["mesh_overhead"] = ms / ms0 - 1.0
    del b
    torch.cuda.empty_cache()
    # three levels: the central 2 x 2 x 2 of the refined blocks refined again
    refine3 = refine + [(1, (i, j, k)) for i in (3, 4) for j in (3, 4) for k in (3, 4)]
    mesh = SMRMesh(base, (4, 4, 4), (32, 32, 32), refine=refine3)
    b = smr_batch(mesh, lambda sp: problems.entropy_wave(sp, amp=0.1))
    dt = 0.3 * min(blk.spec.dx[0] for blk in mesh.blocks)
    ms3, launches3 = timed(steps)
    out["three_levels"] = {"workload": f"the same with the central 2x2x2 level-1 blocks refined again: 56 + 56 + 64 "
                                       f"blocks, {mesh.zones:,} zones",
                           "graph_ms_per_step": ms3, "zone_cycles_per_s": mesh.zones / (ms3 / 1000.0),
                           "launches_per_step": launches3}
    del b
    torch.cuda.empty_cache()
    # spherical-KS Bondi on the two-level layout: r in [3, 30] (MKS, outflow x1), reflecting x2,
    # periodic x3, WENO5; the kharma driver's exchange (conserved variables and seeds, ghost zones
    # inverted) and the primitive exchange
    from kharma_b200.block import build_geometry
    from kharma_b200.spec import bondi_spec
    ks = bondi_spec(32, 32, 32, float(np.log(3.0)), float(np.log(30.0)), 0.0, 1.0, 0.0, 2 * np.pi,
                    bc=("outflow", "outflow", "reflecting", "reflecting", "periodic", "periodic"))
    mesh = SMRMesh(ks, (4, 4, 4), (32, 32, 32), refine=refine)
    ks_out = {"workload": f"Bondi (r_s = 8) in spherical KS (a = 0, MKS), r in [3, 30], 4x4x4 root blocks of 32^3 "
                          f"with the central 2x2x2 refined: {len(mesh.blocks)} blocks, {mesh.zones:,} zones, "
                          f"WENO5, LLF, FP64, outflow/reflecting/periodic faces"}
    for conserved in (True, False):
        b = smr_batch(mesh, lambda sp: problems.bondi(sp, build_geometry(sp)), conserved=conserved)
        dt = 1e-3
        ms_k, launches_k = timed(steps)
        ks_out["kharma_driver_exchange" if conserved else "primitive_exchange"] = {
            "graph_ms_per_step": ms_k, "zone_cycles_per_s": mesh.zones / (ms_k / 1000.0),
            "launches_per_step": launches_k}
        del b
        torch.cuda.empty_cache()
    out["ks_bondi"] = ks_out
    out["b_ct_mhd"] = smr_b_ct_form()
    out["b_ct_torus"] = smr_b_ct_torus_form()
    return out


def smr_b_ct_torus_form(steps=5, warm=2):
    """The FM torus (FMKS, a = 0.9375, MC, LLF, drift-frame floors, outflow x1 with inflow checks,
    reflecting x2 with the polar flux fixes, periodic x3) on a two-level B_CT mesh: 4 x 4 x 2 root
    blocks of 32^3 with the central 2 x 2 x 2 refined (24 + 64 = 88 blocks), a weak field (the curl of
    a vector potential in native coordinates, no normal field at the poles), gs05_c EMFs, FP64, the
    kharma driver's exchange; the CUDA-graph step with the per-block work over 8 streams.  CUDA events
    on the current stream; max face divergence after the run."""
    import dataclasses
    import torch
    from kharma_b200 import ctmesh
    from kharma_b200.ctmesh import cut
    from kharma_b200.mesh import SMRMesh
    from kharma_b200.spec import torus_spec

    # the domain of the 128 x 128 x 64 torus: 5.5 level-0 zones inside the horizon
    base = dataclasses.replace(torus_spec(128, 128, 64), b_ct="gs05_c")
    refine = [(i, j, k) for i in (1, 2) for j in (1, 2) for k in (0, 1)]
    mesh = SMRMesh(base, (4, 4, 2), (32, 32, 32), refine=refine)
    m = ctmesh.CTMesh(mesh, ctmesh.torus_blocks(mesh), cut(mesh, ctmesh.potential_faces_levels(mesh, 1e-3, 5e-4)),
                      streams=8)
    dt = 1e-3
    for _ in range(warm):
        m.step_graph(dt)
    torch.cuda.synchronize()
    s = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(steps):
        m.step_graph(dt)
    e1.record(s)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    out = {"workload": f"FM torus (FMKS a=0.9375) on a two-level B_CT mesh: {len(mesh.blocks)} blocks of 32^3 "
                       f"(24 + 64), {mesh.zones:,} zones, MC, LLF, gs05_c, drift floors, FP64, kharma driver exchange",
           "graph_ms_per_step": ms, "zone_cycles_per_s": mesh.zones / (ms / 1000.0),
           "max_face_divb_dx_after": m.max_divb() * min(min(b.spec.dx) for b in mesh.blocks),
           "all_finite": bool(all(torch.isfinite(b.P).all() for b in m.blocks))}
    m._graph = None
    del m
    torch.cuda.empty_cache()
    return out


def smr_b_ct_form(steps=5, warm=2):
    """A multilevel mesh of B_CT MHD blocks (khb_ctmesh): the 4 x 4 x 4 root grid of 32^3 blocks with the
    central 2 x 2 x 2 refined (56 + 64 blocks, 3.9M zones), magnetized entropy wave (faces the curl of
    a vector potential), linear MC, LLF, gs05_c EMFs, FP64, fixed dt, kharma driver; each stage runs
    every block's khb_ct_stage_fluxes, the flux and EMF corrections, every block's update half, the
    exchange of the updated conserved state and seeds with every ghost zone inverted, and every
    block's inversion and fixups (khb_ct_stage_update_part, khb_ctmesh_exchange_cons), launched block
    by block from the host (eager) or replayed from a CUDA graph of the whole step, the per-block work
    spread over 8 streams; the simple/ImEx drivers' exchange of primitives (graph) beside it; against
    the same blocks stepped alone (khb_ct_step, eager, one stream).  CUDA events on the current
    stream; max face divergence after the run."""
    import torch
    from kharma_b200 import ctmesh
    from kharma_b200.ctmesh import curl_faces_levels, cut, fluid_levels
    from kharma_b200.mesh import SMRMesh
    from kharma_b200.spec import BlockSpec

    ct_base = BlockSpec(nx1=32, nx2=32, nx3=32, x1min=0., x1max=1., x2min=0., x2max=1., x3min=0., x3max=1.,
                        gam=4. / 3., nvar=8, recon="linear_mc", riemann="llf", b_ct="gs05_c", driver="kharma")
    refine = [(i, j, k) for i in (1, 2) for j in (1, 2) for k in (1, 2)]
    mesh = SMRMesh(ct_base, (4, 4, 4), (32, 32, 32), refine=refine)
    m = ctmesh.CTMesh(mesh, cut(mesh, fluid_levels(mesh)), cut(mesh, curl_faces_levels(mesh)), streams=8)
    dt = 0.3 * min(blk.spec.dx[0] for blk in mesh.blocks)

    def timed(step):
        for _ in range(warm):
            step()
        torch.cuda.synchronize()
        s = torch.cuda.current_stream()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(steps):
            step()
        e1.record(s)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    ms_eager = timed(lambda: m.step(dt))
    ms = timed(lambda: m.step_graph(dt))
    divb = m.max_divb() * min(mesh.blocks[0].spec.dx)
    ms_alone = timed(lambda: [b.step(dt) for b in m.blocks])
    n_face, n_emf = int(len(m.tables["face"])), int(len(m.tables["emf"]))
    m._graph = None
    del m
    torch.cuda.empty_cache()
    mp = ctmesh.CTMesh(mesh, cut(mesh, fluid_levels(mesh)), cut(mesh, curl_faces_levels(mesh)), streams=8,
                       conserved=False)
    ms_prims = timed(lambda: mp.step_graph(dt))
    mp._graph = None
    del mp
    out = {"workload": f"B_CT MHD mesh: 4x4x4 root blocks of 32^3, central 2x2x2 refined: {len(mesh.blocks)} blocks, "
                       f"{mesh.zones:,} zones, magnetized entropy wave, linear MC, LLF, gs05_c, FP64",
           "graph_ms_per_step": ms, "zone_cycles_per_s": mesh.zones / (ms / 1000.0), "eager_ms_per_step": ms_eager,
           "prims_exchange_graph_ms_per_step": ms_prims,
           "blocks_alone_eager_one_stream_ms_per_step": ms_alone,
           "max_face_divb_dx_after": divb,
           "face_entries": n_face, "emf_entries": n_emf}
    torch.cuda.empty_cache()
    return out


def b_ct_form(n=128, steps=20, warm=3):
    """B_CT (face-centred field, gs05_c EMFs) against the flux-CT path on the same n^3 periodic MHD
    fast mode (Minkowski, linear MC, LLF, 1D_W) and on the n^3 FM torus, fixed dt, steps launched back
    to back on one stream; CUDA events."""
    import dataclasses
    import torch
    from kharma_b200 import problems
    from kharma_b200.block import Block
    from kharma_b200.spec import mhdmodes_spec

    out = {"workload": f"MHD fast mode {n}^3 periodic, Minkowski, linear MC, LLF, FP64"}
    base = mhdmodes_spec(n, n, n, recon="linear_mc")
    P0 = problems.mhdmodes(base, 3, amp=1e-2)
    for name, spec in (("flux_ct", base), ("b_ct_gs05_c", dataclasses.replace(base, b_ct="gs05_c"))):
        b = Block(spec)
        b.set_prims(P0)
        b.step(spec.dt_min)
        dt = 0.5 * spec.cfl * b.min_ndt()
        for _ in range(warm):
            b.step(dt)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            b.step(dt)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        out[name] = {"ms_per_step": ms, "zone_cycles_per_s": n ** 3 / (ms / 1000.0), "max_divb": b.max_divb()}
        del b
        torch.cuda.empty_cache()
    out["b_ct_over_flux_ct_time"] = out["b_ct_gs05_c"]["ms_per_step"] / out["flux_ct"]["ms_per_step"]
    # the FM torus workload with B_CT (outflow X1, reflecting X2 faces: zero_EMF, the face field's
    # ghost layers and their divergence cleaning each stage) beside the same torus with flux-CT
    from kharma_b200.block import build_geometry
    from kharma_b200.spec import torus_spec
    tspec = torus_spec(n, n, n)
    geom = build_geometry(tspec)
    P0t, Bf0 = problems.fm_torus(tspec, geom, faces=True)
    torus = {"workload": f"FM torus FMKS {n}^3 (outflow X1, reflecting X2, periodic X3, drift floors), MC, LLF, FP64"}
    for name, spec in (("flux_ct", tspec), ("b_ct_gs05_c", dataclasses.replace(tspec, b_ct="gs05_c"))):
        b = Block(spec, geometry=geom)
        b.set_prims(P0t, faces=Bf0 if spec.b_ct != "none" else None)
        dt = 1e-3
        for _ in range(warm):
            b.step(dt)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            b.step(dt)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        torus[name] = {"ms_per_step": ms, "zone_cycles_per_s": n ** 3 / (ms / 1000.0), "max_divb": b.max_divb()}
        del b
        torch.cuda.empty_cache()
    torus["b_ct_over_flux_ct_time"] = torus["b_ct_gs05_c"]["ms_per_step"] / torus["flux_ct"]["ms_per_step"]
    out["torus"] = torus
    return out


def adjoint_form(n=192, steps=200, every=20, ndir=64, workload="torus"):
    """The differentiation form.  workload "torus" (the adjoint workload itself): the n^3 FMKS torus
    block of the benchmark (a = 0.9375, SANE field, u jittered +-4% from a seed, linear MC, LLF,
    flux-CT, 1D_W, drift-frame floors and ceilings, outflow X1 faces with inflow checks, reflecting X2
    faces with the polar flux fixes, periodic X3); the gradient is taken with respect to the initial
    internal energy, and the FD directions perturb u only (u0 (1 + eps xi), xi seeded normal).
    workload "bondi": an n^3 Bondi block (KS a = 0, MKS, r in [3, 30], x2 in [0.1, 0.9], all x3;
    linear MC, LLF, hydro) with exchange faces holding the analytic solution and smooth seeded ramps
    on every variable; FD directions in every variable.  Objective: the time integral over `steps`
    steps of the mass flux through the x1 face layer nearest r = 5; checkpoints every `every` steps.
    The FP32-flux form's forward run and adjoint are timed with CUDA events (the adjoint includes the
    recompute of each segment); its gradient is compared with the FP64 adjoint, and the FP64 adjoint
    with central differences of the FP64 forward run on `ndir` seeded random directions (step size
    1e-7, retried with 1e-6 and 1e-8 when the relative difference exceeds 1e-4; the best is kept)."""
    import dataclasses
    import math
    import numpy as np
    import torch
    from kharma_b200 import problems
    from kharma_b200.adjoint import Run
    from kharma_b200.block import Block, build_geometry
    from kharma_b200.spec import bondi_spec, torus_spec

    if workload == "torus":
        spec64 = torus_spec(n, n, n)
        geom, P0 = make_state(spec64)
        P0 = torch.as_tensor(P0, device="cuda")
        spec32 = dataclasses.replace(spec64, precision="fp32_flux")
        desc = (f"FM torus {n}^3 FMKS (a=0.9375, SANE, u +-4% seeded, linear MC, LLF, flux-CT, 1D_W, drift floors "
                f"and ceilings, outflow/reflecting/periodic faces); gradient w.r.t. the initial internal energy; ")
    else:
        spec64 = bondi_spec(n, n, n, math.log(3.0), math.log(30.0), 0.1, 0.9, 0.0, 2 * math.pi, recon="linear_mc")
        geom = build_geometry(spec64)
        P0 = torch.as_tensor(problems.add_ramps(spec64, problems.bondi(spec64, geom)), device="cuda")
        spec32 = bondi_spec(n, n, n, math.log(3.0), math.log(30.0), 0.1, 0.9, 0.0, 2 * math.pi,
                            recon="linear_mc", precision="fp32_flux")
        desc = (f"Bondi {n}^3 block (KS a=0 MKS, r 3-30, linear MC, LLF, hydro, exchange faces) + seeded "
                f"ramps; ")
    i_f = spec64.ng + int(round((math.log(5.0) - spec64.x1min) / spec64.dx[0]))
    w = np.zeros(spec64.shape)
    w[spec64.interior[0], spec64.interior[1], i_f] = spec64.dx[1] * spec64.dx[2]
    w = torch.as_tensor(w.reshape(-1), device="cuda")
    b64 = Block(spec64, geometry=geom)
    b64.set_prims(P0)
    b64.step(spec64.dt_min)
    dt = 0.5 * spec64.cfl * b64.min_ndt()
    dts = [dt] * steps

    def timed(fn):
        s = torch.cuda.current_stream()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        r = fn()
        e1.record(s)
        torch.cuda.synchronize()
        return r, e0.elapsed_time(e1)

    def gradient(block):
        block.set_prims(P0)
        P0_full = block.P.clone()
        run = Run(block, dts, weight=w, checkpoint_every=every)
        J, ms_f = timed(run.forward)
        torch.cuda.reset_peak_memory_stats()
        g, ms_a = timed(lambda: run.gradient_prims(P0_full))
        return J, g, ms_f, ms_a, torch.cuda.max_memory_allocated(), run.failures

    b32 = Block(spec32, geometry=geom)
    gradient(b32)                      # warm-up (allocations, first launches)
    gradient(b64)
    J32, g32, f32, a32, mem32, _ = gradient(b32)
    J64, g64, f64, a64, mem64, fails64 = gradient(b64)
    if workload == "torus":
        # the gradient with respect to the initial internal-energy perturbation field, which acts where
        # rho is above the floor (outside, the exactly axisymmetric atmosphere puts the x3 MC slopes at
        # the limiter's non-smooth point, where the objective has no derivative)
        jittered = (P0[0] > spec64.floors.rho_min_geom)
        g32 = torch.where(jittered, g32[1], torch.zeros_like(g32[1]))[None]
        g64 = torch.where(jittered, g64[1], torch.zeros_like(g64[1]))[None]
    zones = n ** 3
    out = {"workload": desc + f"objective: integral of the mass flux through r=5 over {steps} steps; "
                              f"checkpoints every {every} steps",
           "dt": dt,
           "fp32_flux": {"forward_ms_per_step": f32 / steps, "adjoint_ms_per_step": a32 / steps,
                         "adjoint_over_forward": a32 / f32, "peak_bytes_during_adjoint": mem32,
                         "adjoint_zone_cycles_per_s": zones * steps / (a32 / 1000.0)},
           "fp64": {"forward_ms_per_step": f64 / steps, "adjoint_ms_per_step": a64 / steps,
                    "adjoint_over_forward": a64 / f64, "peak_bytes_during_adjoint": mem64},
           "objective_fp32_vs_fp64_rel": abs(J32 - J64) / abs(J64),
           "gradient_fp32_vs_fp64_rel_l2": float((g32 - g64).norm() / g64.norm())}
    del b32
    torch.cuda.empty_cache()

    # FP64 adjoint against central differences of the FP64 run
    def objective(P):
        b64.set_prims(P)
        return Run(b64, dts, weight=w, checkpoint_every=steps).forward()
    rng = np.random.Generator(np.random.PCG64(1))
    sl = (slice(None),) + spec64.interior
    scale = P0[sl].pow(2).mean(dim=(1, 2, 3)).sqrt().cpu().numpy() + 1e-6
    rels = []
    for _ in range(ndir):
        v = torch.zeros_like(P0)
        xi = torch.as_tensor(rng.standard_normal(tuple(v[sl].shape)), device="cuda")
        if workload == "torus":
            v[1][spec64.interior] = xi[1] * P0[1][spec64.interior]
            v[1] = torch.where(jittered, v[1], torch.zeros_like(v[1]))
        else:
            v[sl] = xi * torch.as_tensor(scale[:, None, None, None], device="cuda")
        ad = float((g64 * v[1:2]).sum()) if workload == "torus" else float((g64 * v).sum())
        best = math.inf
        for e in ((1e-5, 1e-6, 1e-7) if workload == "torus" else (1e-7, 1e-6, 1e-8)):
            fd = (objective(P0 + e * v) - objective(P0 - e * v)) / (2 * e)
            best = min(best, abs(fd - ad) / max(abs(fd), abs(ad), 1e-300))
            if best < 1e-4:
                break
        rels.append(best)
    if rels:
        out["fd_check_fp64"] = {"directions": ndir, "median_rel": float(np.median(rels)),
                                "worst_rel": float(max(rels)), "below_1e-4": int(sum(r < 1e-4 for r in rels)),
                                "below_1e-3": int(sum(r < 1e-3 for r in rels))}
    out["failed_inversions_fp64_forward"] = fails64
    return out


def gpu_arm(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from kharma_b200 import problems
    from kharma_b200.block import Block, Driver
    from kharma_b200.spec import torus_spec

    torch.cuda.set_device(local_rank)
    n1, n2, n3 = [int(x) for x in args.size.split(",")]
    spec = torus_spec(n1, n2, n3)
    geom, P0 = make_state(spec)
    zones = n1 * n2 * n3

    def make(precision):
        """N = 1: the whole block, khb_step per step.  N > 1: this rank's 128^3 slab of a
        n1 x n2 x (n3 N) torus (x3 decomposition, NCCL halo exchange, global dt reduction)."""
        if world == 1 and not args.slab_path:
            b = Block(torus_spec(n1, n2, n3, precision=precision), geometry=geom)
            b.set_prims(P0)
            return b, Driver(b)
        from kharma_b200 import slabs as sl
        local = world == 1
        gspec = torus_spec(n1, n2, n3 * world, precision=precision)
        ex = sl.LocalExchange() if local else sl.DistExchange()
        sb = sl.SlabBlock(gspec, world, rank, ex, geometry=geom)
        Ploc = P0 if local else problems.fm_torus(sb.spec, geom, seed=1234 + rank)
        sl.set_prims([sb], ex, [Ploc], local=local)
        # across ranks the halo exchange of each stage overlaps the next stage's inner faces
        return sb.block, sl.SlabDriver([sb], ex, local=local, overlap=not local)

    def run(precision, steps, warmup, sampler=None, graph=None):
        """Time `steps` RK2 steps.  graph (N = 1): the step replayed from a CUDA graph with the
        timestep kept on the device (khb_step_graph), else the host-driven step (khb_step plus the
        timestep read-back each step)."""
        graph = (world == 1 and not args.slab_path) if graph is None else graph
        b, drv = make(precision)
        if graph:
            from kharma_b200.block import DeviceDriver
            drv = DeviceDriver(b, graph=True)
        for _ in range(warmup):
            drv.step()
        if hasattr(drv, "sync"):
            drv.sync()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        l0 = b.launch_count()
        if sampler:
            sampler.start()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            drv.step()
        if hasattr(drv, "sync"):
            drv.sync()                      # the last step's exchange inside the timed region
        e1.record()
        torch.cuda.synchronize()
        clocks = sampler.stop() if sampler else None
        if world > 1:
            dist.barrier()
        ms = e0.elapsed_time(e1)
        launches = b.launch_count() - l0
        return b, drv, ms, launches, clocks

    sampler = ClockSampler(torch.cuda.current_device())
    bench_stream = torch.cuda.Stream()
    torch.cuda.set_stream(bench_stream)          # graph capture needs a non-default stream
    b, drv, ms, launches, clocks = run(args.form, args.steps, args.warmup, sampler)
    graph_ok = world == 1 and not args.slab_path
    host_driven = None
    if world == 1 and not args.slab_path:
        _, _, ms_h, _, _ = run(args.form, max(3, args.steps // 4), args.warmup, graph=False)
        host_driven = {"ms_per_step": ms_h / max(3, args.steps // 4),
                       "value": zones / (ms_h / max(3, args.steps // 4) / 1000.0)}
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    ms_step = ms_max / args.steps
    value = world * zones / (ms_step / 1000.0)

    # FP32-flux form on the same workload
    fp32 = None
    if not args.no_fp32 and world == 1:
        b32, _, ms32, _, _ = run("fp32_flux", args.steps, args.warmup)
        t32 = torch.tensor([ms32], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(t32, op=dist.ReduceOp.MAX)
        v32 = world * zones / (float(t32.item()) / args.steps / 1000.0)
        fp32 = {"value": v32, "unit": UNIT, "ms_per_step": float(t32.item()) / args.steps,
                "speedup_vs_fp64": v32 / value}
        if not args.no_kernel_times:
            kt32 = kernel_times(b32, b32.spec)
            fp32["kernel_ms_per_launch"] = {k: round(v[0], 4) for k, v in kt32.items()}
        del b32
        # accuracy: 100 steps of each form from the same state with the FP64 run's dt sequence
        ref = Block(torus_spec(n1, n2, n3), geometry=geom)
        ref.set_prims(P0)
        dref = Driver(ref)
        dts = [dref.step()[0] for _ in range(100)]
        f32 = Block(torus_spec(n1, n2, n3, precision="fp32_flux"), geometry=geom)
        f32.set_prims(P0)
        for dt in dts:
            f32.step(dt)
        torch.cuda.synchronize()
        sl = spec.interior
        r64, r32 = ref.P[0][sl], f32.P[0][sl]
        fp32["rel_l1_rho_after_100_steps"] = float((r32 - r64).abs().sum() / r64.abs().sum())
        del ref, f32

    # end-to-end through the C ABI with a host-resident state: khb_step_host_interior copies the
    # interior primitives in (pinned host memory), rebuilds U = U(P) and the ghost zones on the device
    # (the state's own: the lock-step P -> U and the boundaries leave both as functions of the
    # interior after every step), replays the graph step and copies the interior primitives back
    e2e = None
    if not args.no_e2e:
        isl = (slice(None),) + spec.interior
        hP = torch.empty(b.P.shape if not graph_ok else b.P[isl].shape, dtype=torch.float64, pin_memory=True)
        hP.copy_(b.P if not graph_ok else b.P[isl])
        torch.cuda.synchronize()
        ke = max(3, args.steps // 2)
        if world > 1:
            dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        if graph_ok:
            for _ in range(ke):
                drv.step_host_interior(hP)
        else:
            for _ in range(ke):
                b.P.copy_(hP, non_blocking=True)
                b.ptou()
                drv.step()
                if hasattr(drv, "sync"):
                    drv.sync()              # the state complete before it is read back
                hP.copy_(b.P, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        te = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
        if world > 1:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        ms_e = float(te.item()) / ke
        nbytes = hP.numel() * 8
        e2e = {"value": world * zones / (ms_e / 1000.0), "unit": UNIT, "h2d_bytes_per_step": nbytes,
               "d2h_bytes_per_step": nbytes if world == 1 else nbytes + 8, "ms_per_step": ms_e,
               "path": "khb_step_host_interior" if graph_ok else "P in, khb_ptou, host-driven step, P out"}

    # roofline of the dominant kernel, timed live with CUDA events
    peak, peak_kind = measured_peaks()
    roofline = None
    ktimes = None
    if not args.no_kernel_times and world == 1:
        ktimes = kernel_times(b, spec)
        tot = {k: v[0] * v[1] for k, v in ktimes.items()}
        dom = max(tot, key=tot.get)
        ms_launch = ktimes[dom][0]
        nv = spec.nvar
        # algorithmic bytes per launch: the zone pass moves the stage's state arrays
        # (stage 1: read P0,U0 write P1,U1; stage 2: read P1,U1,U0 write P2,U2 -> 4.5 nv doubles
        # per zone per launch on average); a flux pass reads P once (nv doubles per zone).
        per_zone = {"k_zone": 4.5 * nv * 8}.get(dom, nv * 8)
        ach = per_zone * zones / (ms_launch / 1000.0) / 1e9
        traffic, tsrc = profile_traffic(dom, (n1, n2, n3), args.form)
        roofline = {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "unit": "GB/s",
                    "frac": ach / peak, "peak_kind": peak_kind, "traffic": traffic, "traffic_source": tsrc,
                    "alg_bytes_per_zone_per_launch": per_zone,
                    "step_frac": B_ALG_PER_ZC * zones / (ms_step / 1000.0) / 1e9 / peak}
        detail("kernel_ms_per_launch", {k: round(v[0], 4) for k, v in ktimes.items()})

    emhd = None
    if rank == 0 and world == 1 and not args.no_emhd:
        emhd = emhd_newton()
        detail("emhd_newton", emhd)

    if rank == 0 and world == 1 and not args.no_batch:
        detail("b_ct", b_ct_form())
        detail("smr", smr_form())
        del b, drv
        torch.cuda.empty_cache()
        detail("batching", batching())

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_block(n1, n2, n3)

    if rank == 0:
        if host_driven:
            detail("host_driven_step", host_driven)
        if fp32 and "kernel_ms_per_launch" in fp32:
            detail("fp32_flux_kernel_ms_per_launch", fp32.pop("kernel_ms_per_launch"))
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
               "config": {"workload": (f"FM torus FMKS {n1}x{n2}x{n3} one meshblock per GPU" if world == 1 else
                                       f"FM torus FMKS {n1}x{n2}x{n3 * world}, one {n1}x{n2}x{n3} x3 slab per GPU"),
                          "recon": "linear_mc", "flux": "llf", "b_field": "flux_ct", "inverter": "onedw",
                          "floors": "drift", "form": args.form,
                          "parallelism": "single block" if world == 1 else f"x3 slabs x{world} (NCCL halo exchange)",
                          "l2": (f"state {2 * spec.nvar * spec.shape[0] * spec.shape[1] * spec.shape[2] * 8 / 1e6:.0f} MB "
                                 f"{'>' if 2 * spec.nvar * np.prod(spec.shape) * 8 > 126e6 else '<'} L2 (126 MB), no flush")},
               "gpu_launches": launches, "clocks": clocks, "roofline": roofline,
               "fp32_flux": fp32, "e2e": e2e, "cpu_baseline": cpu,
               "emhd_newton": emhd_summary(emhd) if emhd else None}
        print(json.dumps(compact(out)), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    import torch
    if args.emhd_only:
        if rank == 0:
            e = emhd_newton()
            detail("emhd_newton", e)
            print(json.dumps({"emhd_newton": emhd_summary(e)}), flush=True)
        return
    if args.adjoint_only:
        if rank == 0:
            n, steps, every, ndir = [int(x) for x in args.adjoint_shape.split(",")]
            print(json.dumps({"adjoint": adjoint_form(n, steps, every, ndir, args.adjoint_workload)}), flush=True)
        return
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    try:
        gpu_arm(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()

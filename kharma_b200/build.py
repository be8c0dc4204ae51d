"""Build libkhb.so in-tree for sm_100a with nvcc.

    python -m kharma_b200.build              (lib/libkhb.so)
    python -m kharma_b200.build --checked    (lib/libkhb_checked.so, KHB_BOUNDS_CHECK=1)

Translation units and their arithmetic flags:
  khb_fp64.cu      FP64 path (fluxes, zone pass, ghost zones)      -fmad=false
  khb_fp32.cu      FP32-flux form (fluxes, EMFs in FP32)           FMA contraction, fast FP32
                                                                   divide and square root, FTZ
  khb_api.cu       host side and C ABI
  khb_batch.cu     batches of meshblocks: tile tables, CUDA graph, autotuner
  khb_noalloc.cu   khb_max_divb_noalloc (static device scratch)   -fmad=false
  khb_emhd.cu      EMHD sources and the implicit Newton solve      -fmad=false
  khb_adjoint.cu   discrete adjoint of the step (FP64 faces)      -fmad=false
  khb_adjoint_fp32.cu  adjoint of the FP32-flux form's faces      as khb_fp32.cu
  khb_ct.cu        B_CT (face-centred field, EMFs, face update)   -fmad=false
  khb_ctmesh.cu    SMR meshes of B_CT blocks (corrections, exchange)  -fmad=false
  khb_geometry.cpp host construction of the geometry tables
The library is a plain shared object; the Python layer binds it with ctypes.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "lib", "libkhb.so")
OBJ = os.path.join(HERE, "lib", "obj")
UNITS = {
    "khb_fp64.cu": ["-fmad=false"],
    "khb_fp32.cu": ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"],
    "khb_api.cu": [],
    "khb_batch.cu": [],
    "khb_noalloc.cu": ["-fmad=false"],
    "khb_emhd.cu": ["-fmad=false"],
    "khb_adjoint.cu": ["-fmad=false"],
    "khb_adjoint_fp32.cu": ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"],
    "khb_ct.cu": ["-fmad=false"],
    "khb_ctmesh.cu": ["-fmad=false"],
    "khb_geometry.cpp": [],
}
HEADERS = ["khb_device.cuh", "khb_kernels.cuh", "khb_types.cuh", "khb_internal.hpp", "khb_dual.cuh", "khb_adjoint_flux.cuh", os.path.join("..", "..", "include", "khb.h")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]


def _deps_mtime():
    paths = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.abspath(__file__)]
    return max(os.path.getmtime(p) for p in paths)


CHECKED_OUT = os.path.join(HERE, "lib", "libkhb_checked.so")
CHECKED_OBJ = os.path.join(HERE, "lib", "obj_checked")


def build_checked(force=False, verbose=False):
    """The bounds-checked build (KHB_BOUNDS_CHECK=1, khb_bounds_status in include/khb.h)."""
    return build(force=force, extra_flags=["-DKHB_BOUNDS_CHECK=1"], out=CHECKED_OUT, obj=CHECKED_OBJ,
                 verbose=verbose)


def build(force=False, extra=(), out=OUT, verbose=False, jobs=4, extra_flags=(), obj=None):
    """Compile the units whose sources or headers changed and link out.  extra: flags that also force
    a full rebuild; extra_flags: flags of a build variant kept in its own object directory obj."""
    OBJ_DIR = obj or OBJ
    os.makedirs(OBJ_DIR, exist_ok=True)
    hdr_t = _deps_mtime()
    procs = []
    objs = []
    for src, flags in UNITS.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ_DIR, src + ".o")
        objs.append(o)
        stale = force or extra or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr_t)
        if not stale:
            continue
        cmd = ["nvcc", *ARCH, *COMMON, *flags, *extra, *extra_flags, "-c", s, "-o", o]
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = []
    for src, p in procs:
        log, _ = p.communicate()
        if p.returncode != 0:
            failed.append(src)
            sys.stderr.write(log)
        elif verbose and log.strip():
            print(log)
    if failed:
        raise RuntimeError(f"nvcc failed on {failed}")
    if procs or not os.path.exists(out):
        cmd = ["nvcc", *ARCH, "-shared", "-o", out, *objs]
        if verbose:
            print(" ".join(cmd))
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError("nvcc link failed")
    return out


if __name__ == "__main__":
    if "--checked" in sys.argv[1:]:
        print(build_checked(force=True, verbose=True))
    else:
        extra = [a for a in sys.argv[1:] if a.startswith("-")]
        print(build(force=True, extra=extra, verbose=True))

"""Build libkhb.so in-tree for sm_100a with nvcc.

    python -m kharma_b200.build [--fmad=false]

The library is a plain shared object (no torch extension); the Python layer binds it with ctypes.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "lib", "libkhb.so")
SOURCES = ["khb_api.cu", "khb_geometry.cpp"]
HEADERS = ["khb_device.cuh", "khb_kernels.cuh", os.path.join("..", "..", "include", "khb.h")]


def nvcc_command(out=OUT, extra=()):
    return ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
            "-Xcompiler", "-fPIC", "-shared", *extra, "-o", out] + [os.path.join(CSRC, s) for s in SOURCES]


def up_to_date(out=OUT):
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    deps = SOURCES + HEADERS + ["build.py"]
    return all(os.path.getmtime(os.path.join(CSRC if d != "build.py" else HERE, d)) <= t for d in deps)


def build(force=False, extra=(), out=OUT, verbose=False):
    os.makedirs(os.path.dirname(out), exist_ok=True)
    if not force and not extra and up_to_date(out):
        return out
    cmd = nvcc_command(out, extra)
    if verbose:
        print(" ".join(cmd))
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed building libkhb")
    return out


if __name__ == "__main__":
    extra = [a for a in sys.argv[1:] if a.startswith("-")]
    print(build(force=True, extra=extra, verbose=True))

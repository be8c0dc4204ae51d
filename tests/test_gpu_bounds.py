"""The bounds-checked build (kharma_b200/lib/libkhb_checked.so, KHB_BOUNDS_CHECK=1): the stand-in for
a memory checker.  The same workloads run through it and through the regular library, each in a
process of its own (the library is chosen at load time by KHB_LIB_PATH): every checked index stays
inside its array (status word 0 after each workload) and the results are bitwise those of the
regular build, whose checks compile away."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r'''
import ctypes as C, dataclasses, hashlib, json, sys
sys.path.insert(0, ROOT)
import torch
from kharma_b200 import _lib, problems
from kharma_b200.block import Block
from kharma_b200.spec import mhdmodes_spec, torus_spec
lib = _lib.load()
out = {"checked": int(lib.khb_bounds_checked())}
cases = {
    "torus_fofc": dataclasses.replace(torus_spec(32, 24, 8), fofc=True),
    "torus_kastaun": torus_spec(32, 24, 8, inverter="kastaun"),
    "modes_weno5": mhdmodes_spec(16, 16, 16, recon="weno5"),
    "modes_x3_faces": dataclasses.replace(mhdmodes_spec(12, 12, 12, recon="ppm"),
                                          bc=("outflow", "outflow", "periodic", "periodic", "reflecting", "outflow")),
    "torus_bct": dataclasses.replace(torus_spec(24, 16, 8), b_ct="gs05_c"),
}
for name, spec in cases.items():
    b = Block(spec)
    if name.startswith("torus"):
        if spec.b_ct != "none":
            P0, Bf0 = problems.fm_torus(spec, b.geom, seed=7, faces=True)
            b.set_prims(P0, faces=Bf0)
        else:
            b.set_prims(problems.fm_torus(spec, b.geom, seed=7))
    else:
        b.set_prims(problems.add_ramps(spec, problems.mhdmodes(spec, 3, amp=1e-2)))
    for _ in range(3):
        b.step(spec.dt_min)
    st = C.c_uint64()
    _lib.check(lib.khb_bounds_status(b.ctx, C.byref(st), b.stream), "khb_bounds_status")
    torch.cuda.synchronize()
    h = hashlib.sha1(b.P.cpu().numpy().tobytes() + b.U.cpu().numpy().tobytes()).hexdigest()
    out[name] = {"status": int(st.value), "hash": h}
print("RESULT " + json.dumps(out))
'''


def run(lib):
    env = dict(os.environ, KHB_LIB_PATH=lib)
    res = subprocess.run([sys.executable, "-c", CHILD.replace("ROOT", repr(ROOT))], env=env, capture_output=True,
                         text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-3000:]
    line = [ln for ln in res.stdout.splitlines() if ln.startswith("RESULT ")][-1]
    return json.loads(line[len("RESULT "):])


def test_checked_build_finds_no_out_of_range_index_and_changes_nothing():
    checked_lib = os.path.join(ROOT, "kharma_b200", "lib", "libkhb_checked.so")
    assert os.path.exists(checked_lib), "build the checked library: python -m kharma_b200.build --checked"
    chk = run(checked_lib)
    reg = run(os.path.join(ROOT, "kharma_b200", "lib", "libkhb.so"))
    assert chk["checked"] == 1 and reg["checked"] == 0
    for name in chk:
        if name == "checked":
            continue
        assert chk[name]["status"] == 0, (name, hex(chk[name]["status"]))
        assert reg[name]["status"] == 0
        assert chk[name]["hash"] == reg[name]["hash"], name

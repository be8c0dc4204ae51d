"""Copy the conducting-atmosphere ODE profiles that KHARMA's own test reads into an .npz fixture.

The reference problem generator (kharma/prob/emhd/conducting_atmosphere.cpp:52-240) loads the
files atmosphere_soln_{rCoords,rho,u,phi}.txt, one row per radial zone including the ghost
zones, and checks rCoords against its grid to 1e-10.  Its test harness keeps one set per
resolution under tests/conducting_atmosphere/conducting_atmosphere_<n1>_default/.

Run from the repository root with the path of a KHARMA checkout, as an argument or in the
environment variable KHARMA_REF:
    python tests/golden/make_atmosphere_profiles.py <path to kharma>
"""
import os
import sys

import numpy as np

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("KHARMA_REF")
if not REF:
    sys.exit("usage: make_atmosphere_profiles.py <path to a KHARMA checkout> (or set KHARMA_REF)")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "atmosphere_profiles.npz")

arrays = {}
for n1 in (64, 128):
    d = os.path.join(REF, "tests", "conducting_atmosphere", "conducting_atmosphere_%d_default" % n1)
    for name in ("rCoords", "rho", "u", "phi"):
        arrays["%s_%d" % (name, n1)] = np.loadtxt(os.path.join(d, "atmosphere_soln_%s.txt" % name))
np.savez(OUT, **arrays)
print("wrote", OUT, {k: v.shape for k, v in arrays.items()})

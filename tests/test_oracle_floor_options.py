"""The floor options the GPU parity tests cover change the oracle's result (they are exercised): the
mixed injection frames and radius-dependent floors against the default drift frame on the torus."""
import dataclasses

import numpy as np
import pytest

from kharma_b200 import problems
from kharma_b200.spec import torus_spec


def run(oracle_mod, spec, steps=2):
    o = oracle_mod.Oracle(spec)
    P, U = o.init_state(problems.fm_torus(spec, o.geometry(), seed=7))
    dt = spec.dt_min
    for _ in range(steps):
        _, _, dt, _ = o.step(P, U, dt)
    return P


@pytest.mark.parametrize("option", ["mixed_fluid_normal", "mixed_normal_drift", "radius_dependent"])
def test_option_changes_the_result(oracle_mod, option):
    base = torus_spec(24, 16, 1)
    if option == "radius_dependent":
        spec = dataclasses.replace(base, floors=dataclasses.replace(base.floors, radius_dependent_floors=True,
                                                                    floors_switch_r=20.0),
                                   floors_inner=dataclasses.replace(base.floors, rho_min_geom=1e-5, u_min_geom=1e-7))
    else:
        spec = dataclasses.replace(base, floor_frame=option, frame_switch_r=10.0, frame_switch_beta=10.0)
    assert not np.array_equal(run(oracle_mod, base), run(oracle_mod, spec))

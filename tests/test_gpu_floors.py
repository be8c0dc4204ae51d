"""Floor options against the oracle on the FM torus (3 steps, 1e-12, identical flags): the mixed
injection frames (floors/floors_impl.hpp:84-106: normal inside frame_switch_r and fluid outside; or
drift where min(rho, u)/b^2 < frame_switch_beta and normal elsewhere) and radius-dependent floors
with an inner prescription (floors.hpp:155-167, floors_functions.hpp:56-57, 89-90)."""
import dataclasses

import numpy as np
import pytest

from kharma_b200 import problems
from kharma_b200.spec import torus_spec

from test_gpu_parity import RTOL, make_pair, run_steps

pytestmark = pytest.mark.gpu


def with_floors(**kw):
    base = torus_spec(32, 24, 8)
    if "floors_inner" in kw:
        kw["floors"] = dataclasses.replace(base.floors, radius_dependent_floors=True, floors_switch_r=20.0)
    return dataclasses.replace(base, **kw)


CASES = {
    "mixed_fluid_normal": lambda: with_floors(floor_frame="mixed_fluid_normal", frame_switch_r=10.0),
    "mixed_normal_drift": lambda: with_floors(floor_frame="mixed_normal_drift", frame_switch_beta=10.0),
    "radius_dependent": lambda: with_floors(floors_inner=dataclasses.replace(torus_spec(8, 8, 1).floors,
                                                                            rho_min_geom=1e-5, u_min_geom=1e-7,
                                                                            bsq_over_rho_max=50.0)),
    "radius_dependent_kastaun": lambda: dataclasses.replace(
        with_floors(floors_inner=dataclasses.replace(torus_spec(8, 8, 1).floors, rho_min_geom=1e-5, u_min_geom=1e-7)),
        inverter="kastaun", iter_max=25, err_tol=1e-12, fix_average_neighbors=False),
}


@pytest.mark.parametrize("name", list(CASES))
def test_floor_options(oracle_mod, name):
    spec = CASES[name]()
    o, b, Po, Uo = make_pair(oracle_mod, spec, problems.fm_torus(spec, oracle_mod.Oracle(spec).geometry(), seed=7))
    worst, flags_equal = run_steps(o, b, Po, Uo, 3, spec)
    print(name, "worst per-variable relative error:", worst)
    assert np.all(worst <= RTOL), worst
    assert flags_equal

"""Shared inputs of the EMHD / implicit-solve tests: the conducting atmosphere on a small block.

The radial profile is the reference's own ODE solution (tests/golden/atmosphere_profiles.npz, made
by tests/golden/make_atmosphere_profiles.py); the explicit dU/dt handed to the implicit solve is
the EMHD explicit source plus seeded noise on every variable, so that the Newton iterations have
work to do.
"""
import os

import numpy as np

from kharma_b200 import problems
from kharma_b200.spec import EmhdSpec, ImplicitSpec, atmosphere_spec

HERE = os.path.dirname(os.path.abspath(__file__))


def profile(n1):
    z = np.load(os.path.join(HERE, "golden", "atmosphere_profiles.npz"))
    return {k: z["%s_%d" % (k, n1)] for k in ("rCoords", "rho", "u", "phi")}


EMHD_VARIANTS = {
    # the conducting-atmosphere deck's closure (conducting_atmosphere.par:68-80) with viscosity on
    "kappa_eta_ho": EmhdSpec(closure_type="kappa_eta", higher_order_terms=True, tau=1.0, kappa=0.1, eta=0.1),
    "constant": EmhdSpec(closure_type="constant", higher_order_terms=False, tau=1.0, conduction_alpha=0.1,
                         viscosity_alpha=0.1),
    "soundspeed_q_only": EmhdSpec(closure_type="soundspeed", higher_order_terms=True, viscosity=False, tau=1.0,
                                  conduction_alpha=0.1),
    "dp_only": EmhdSpec(closure_type="kappa_eta", higher_order_terms=True, conduction=False, tau=1.0, eta=0.1),
    "grmhd_only": EmhdSpec(closure_type="constant", conduction=False, viscosity=False),
    "torus": EmhdSpec(closure_type="torus", higher_order_terms=True, tau=1.0, conduction_alpha=0.1,
                      viscosity_alpha=0.1),
}


def atmosphere_case(n1=64, n2=8, n3=1, emhd=None, seed=7, noise=1e-2, dt=0.5):
    """(spec, emhd, P, dt, src_noise) with P the 10-slot initial state over the whole block."""
    spec = atmosphere_spec(n1, n2, n3)
    emhd = emhd or EMHD_VARIANTS["kappa_eta_ho"]
    from kharma_b200.block import build_geometry
    geom = build_geometry(spec)
    P = problems.conducting_atmosphere(spec, geom, emhd, profile(n1), jitter=1e-3, seed=seed)
    if not emhd.conduction:
        P[8] = 0.
    rng = np.random.Generator(np.random.PCG64(seed + 1))
    xi = rng.uniform(-1.0, 1.0, size=P.shape)
    return spec, emhd, P, dt, xi * noise


def source(U, S_emhd, xi, dt):
    """dU/dt for the implicit solve: the explicit EMHD sources plus noise of relative size |xi| per step."""
    S = S_emhd.copy()
    S[:8] += xi[:8] * np.abs(U[:8]) / dt
    S[8:] += xi[8:] * (np.abs(U[8:]) + 1e-3 * np.abs(U[0:1])) / dt
    return S


def implicit(jacobian="fd", **kw):
    base = dict(min_nonlinear_iter=1, max_nonlinear_iter=8, rootfind_tol=1e-10, jacobian=jacobian)
    base.update(kw)
    return ImplicitSpec(**base)


# A block with every ImEx boundary and limit step in play: the atmosphere's own faces (outflow X1
# with inflow checks, reflecting X2 with the polar flux fixes and the corner fix, periodic X3),
# geometric density floors that bind in the inner part of the block, the EMHD stability limits on,
# a monopole field strong enough for the anisotropy bounds to matter, and q~ / dP~ raised in seeded
# zones so that the limit bits are hit.
LIMITS_CASES = {
    # closure, B10, q~ factor, dP~ amplitude (in units of u)
    "constant": ("constant", 5e5, 5000.0, 2.0),
    "kappa_eta_ho": ("kappa_eta_ho", 2e6, 5000.0, 30.0),
}


def atmosphere_limits_case(name, n1=64, n2=6, n3=1, seed=3):
    """(spec, emhd, P) for LIMITS_CASES[name] on an n1 x n2 x n3 atmosphere block."""
    import dataclasses
    from kharma_b200.block import build_geometry
    from kharma_b200.spec import FloorSpec
    variant, B10, qfac, dpamp = LIMITS_CASES[name]
    emhd = dataclasses.replace(EMHD_VARIANTS[variant], stability_limits=True)
    spec = dataclasses.replace(atmosphere_spec(n1, n2, n3), floors_on=True, floor_frame="drift",
                               floors=FloorSpec(rho_min_geom=8000.0, u_min_geom=1e-8),
                               check_inflow_inner_x1=True, check_inflow_outer_x1=True,
                               zero_polar_flux=True, fix_polar_flux=True, fix_corner_inner=True)
    P = problems.conducting_atmosphere(spec, build_geometry(spec), emhd, profile(n1), jitter=1e-3, seed=seed,
                                       B10=B10)
    m = np.random.Generator(np.random.PCG64(seed + 8)).uniform(size=P.shape[1:])
    P[8] *= np.where(m < 0.2, qfac, 1.0)
    P[9] = np.where(m > 0.85, dpamp, np.where(m > 0.7, -dpamp, 0.0)) * P[1]
    return spec, emhd, P

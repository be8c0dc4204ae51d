"""The Kastaun inverter of the oracle (inverter/kastaun.hpp:83-406), CPU only.

No golden vectors exist for it in the reference, so it is pinned by its defining property and by the
other inverter: for magnetized states in the FM-torus geometry (spherical KS, a = 0.9375, FMKS),
P -> U -> Kastaun recovers P to 1e-9 relative (its tolerance is 1e-12 on mu = 1/(h W)); it agrees
with 1D_W on the same conserved states to 1e-6; and it reports its inverter floors with the
reference's FFlag bits (INVERTER_RHO = 16384, INVERTER_U = 32768, INVERTER_GAMMA = 65536).
"""
import numpy as np

from kharma_b200.spec import torus_spec

RHO_FLAG, U_FLAG, GAMMA_FLAG = 16384, 32768, 65536


def random_state(spec, seed):
    """Moderate magnetized states: u/rho below the torus floors' u_over_rho_max (2), and velocity and
    field components of order 0.1 in units of the local metric scale 1/sqrt(g_ii)."""
    from kharma_b200.block import build_geometry
    g = np.asarray(build_geometry(spec)["gcov"])[3, :spec.shape[1], :spec.shape[2]]
    rng = np.random.Generator(np.random.PCG64(seed))
    shape = (spec.nvar,) + spec.shape
    P = np.zeros(shape)
    P[0] = rng.uniform(0.3, 1.0, spec.shape)
    P[1] = rng.uniform(0.01, 0.5, spec.shape)
    for a in range(3):
        scale = 1.0 / np.sqrt(g[..., a + 1, a + 1])[None]
        P[2 + a] = rng.uniform(-0.1, 0.1, spec.shape) * scale
        P[5 + a] = rng.uniform(-0.1, 0.1, spec.shape) * scale
    return P


def outside(spec, oracle_mod, r_min=4.0):
    """Interior zones at r >= r_min (away from the horizon, where random states are unphysical)."""
    r = oracle_mod.Oracle(spec).geometry()["r_center"]
    return np.broadcast_to(r[None], spec.shape)[spec.interior] >= r_min


def invert(oracle_mod, spec, P, guess_scale=1.0, seed=3):
    o = oracle_mod.Oracle(spec)
    U = o.ptou(P)
    rng = np.random.Generator(np.random.PCG64(seed))
    Pg = P.copy()
    Pg[:5] *= 1.0 + (guess_scale - 1.0) * rng.uniform(-1, 1, Pg[:5].shape)
    pflag, fflag = o.utop(U, Pg)
    return Pg, pflag, fflag


def test_kastaun_round_trip(oracle_mod):
    spec = torus_spec(24, 24, 1, inverter="kastaun")
    P = random_state(spec, 1)
    Pk, pflag, fflag = invert(oracle_mod, spec, P, guess_scale=1.05)
    sl = spec.interior
    m = outside(spec, oracle_mod)
    assert m.mean() > 0.5
    assert not (pflag[sl][m] > 0).any()
    assert not fflag[sl][m].any()
    for v in range(5):
        rel = np.max(np.abs(Pk[v][sl][m] - P[v][sl][m]) / (np.abs(P[v][sl][m]) + 1e-3))
        assert rel < 1e-9, (v, rel)


def test_kastaun_agrees_with_onedw(oracle_mod):
    sk = torus_spec(24, 24, 1, inverter="kastaun")
    so = torus_spec(24, 24, 1, inverter="onedw")
    P = random_state(sk, 2)
    Pk, pk, _ = invert(oracle_mod, sk, P, guess_scale=1.02)
    Po, po, _ = invert(oracle_mod, so, P, guess_scale=1.02)
    sl = sk.interior
    ok = (pk[sl] == 0) & (po[sl] == 0) & outside(sk, oracle_mod)
    assert ok.sum() > 0.5 * ok.size
    for v in range(5):
        d = np.abs(Pk[v][sl] - Po[v][sl])[ok] / (np.abs(P[v][sl])[ok] + 1e-3)
        assert d.max() < 1e-6, (v, d.max())


def test_kastaun_inverter_floors(oracle_mod):
    spec = torus_spec(16, 16, 1, inverter="kastaun")
    spec.floors.rho_min_const = 1e-3
    spec.floors.u_min_const = 1e-4
    P = random_state(spec, 4)
    sl = spec.interior
    P[0][sl][:, :, :4] = 1e-5           # below rho_min_const
    P[1][sl][:, :4, :] = 1e-7           # below the energy floor
    P[0][sl][:, :4, :] = 0.5
    Pk, pflag, fflag = invert(oracle_mod, spec, P)
    f = fflag[sl].astype(int)
    assert (f[:, :, :4][:, 4:, :] & RHO_FLAG).all()
    assert (f[:, :4, 4:] & U_FLAG).all()
    assert (Pk[0][sl] >= 1e-3 * (1 - 1e-12)).all()

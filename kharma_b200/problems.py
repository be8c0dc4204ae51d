"""Synthetic initial states for the benchmark and test workloads (host-side, numpy).

These restate the reference's problem generators closely enough to produce the named workloads;
they are inputs, not part of the per-step path:
  * mhdmodes: linear MHD modes on a periodic box (prob/mhdmodes.hpp:60-242, seed_B.hpp:160-169)
  * fm_torus: Fishbone-Moncrief torus with a SANE field (prob/fm_torus.cpp:41-197,
    prob/fm_torus.hpp, prob/seed_B.cpp:215-534), internal energy jittered from a seeded RNG
    (prob/utils/perturbation.hpp:49-114)

Every function returns primitives P of shape (nvar, n3, n2, n1) with the interior set; ghost zones
are filled afterwards by the boundary conditions of the step (khb_boundaries) and U = U(P).
"""
import math

import numpy as np

# 2D-plane linear modes, prob/mhdmodes.hpp:140-190 (nmode: 0 entropy, 1 slow, 2 alfven, 3 fast),
# wave in the X1/X2 plane (dir = 3), background rho = u = 1, B = (1, 0, 0)
MODES_DIR3 = {
    0: dict(omega=0.0, drho=1.0, du=0.0, du1=0.0, du2=0.0, du3=0.0, dB1=0.0, dB2=0.0, dB3=0.0),
    1: dict(omega=2.41024185339, drho=0.558104461559, du=0.744139282078, du1=-0.277124827421,
            du2=0.0630348927707, du3=0.0, dB1=-0.164323721928, dB2=0.164323721928, dB3=0.0),
    2: dict(omega=3.44144232573, drho=0.0, du=0.0, du1=0.0, du2=0.0, du3=0.480384461415,
            dB1=0.0, dB2=0.0, dB3=0.877058019307),
    3: dict(omega=5.53726217331, drho=0.476395427447, du=0.635193903263, du1=-0.102965815319,
            du2=-0.316873207561, du3=0.0, dB1=0.359559114174, dB2=-0.359559114174, dB3=0.0),
}


def cell_centers(spec):
    """Native coordinates of the zone centres along each direction (entire block)."""
    n3, n2, n1 = spec.shape
    dx1, dx2, dx3 = spec.dx
    g2 = spec.ng if spec.nx2 > 1 else 0
    g3 = spec.ng if spec.nx3 > 1 else 0
    x1 = (spec.x1min - spec.ng * dx1) + (np.arange(n1) + 0.5) * dx1
    x2 = (spec.x2min - g2 * dx2) + (np.arange(n2) + 0.5) * dx2
    x3 = (spec.x3min - g3 * dx3) + (np.arange(n3) + 0.5) * dx3
    return x1, x2, x3


def mhdmodes(spec, nmode=3, amp=1e-4):
    """Linear mode with k = (2 pi, 2 pi, 0) on the periodic unit box (mhdmodes dir = 3)."""
    m = MODES_DIR3[nmode]
    n3, n2, n1 = spec.shape
    x1, x2, x3 = cell_centers(spec)
    X1, X2 = np.meshgrid(x1, x2, indexing="xy")          # (n2, n1)
    phase = 2 * np.pi * X1 + 2 * np.pi * X2
    mode = amp * np.cos(phase)
    cmode = np.cos(phase)
    P = np.zeros((spec.nvar, n3, n2, n1))
    P[0] = 1.0 + m["drho"] * mode
    P[1] = 1.0 + m["du"] * mode
    P[2] = 0.0 + m["du1"] * mode
    P[3] = 0.0 + m["du2"] * mode
    P[4] = 0.0 + m["du3"] * mode
    if spec.nvar > 5:
        P[5] = 1.0 + (amp * m["dB1"]) * cmode
        P[6] = 0.0 + (amp * m["dB2"]) * cmode
        P[7] = 0.0 + (amp * m["dB3"]) * cmode
    return P


# The 2D EMHD wave of prob/emhd/emhdmodes.hpp:56-160: mean state rho 1, u 2, B (0.1, 0.3, 0), wavevector
# (2 pi, 4 pi, 0), conduction and viscosity with the sound-speed closure; eigenvector coefficients of
# cos(phi) and sin(phi) per primitive (rho, u, u1, u2, u3, B1, B2, B3, q, dP) and the complex
# frequency (decay rate omega_real, angular frequency omega_imag) as the problem defines them
# (the B coefficients come through the "wave" field seed, prob/seed_B.hpp:160-169).
EMHD_MODE = {
    "mean": (1.0, 2.0, 0.0, 0.0, 0.0, 0.1, 0.3, 0.0, 0.0, 0.0),
    "cos": (-0.518522524082246, 0.5516170736393813, 0.008463122479547856, -0.16175466371870734, 0.0,
            -0.05973794979640743, 0.02986897489820372, 0.0, 0.5233486841539436, 0.2909106062057657),
    "sin": (0.1792647678001878, 0.0, -0.011862022608466367, 0.034828080823603294, 0.0,
            0.03351707506150924, -0.016758537530754618, 0.0, -0.04767672501939603, -0.02159452055336572),
    "omega_real": -0.5533585207638141, "omega_imag": -3.6262571286888425, "k1": 2 * np.pi, "k2": 4 * np.pi,
}


def emhdmodes(spec, amp=1e-8, t=0.0):
    """The EMHD wave on the periodic unit square (emhdmodes.hpp:129-157 without higher-order terms):
    10-slot primitives over the whole block at time t (t = 0: the initial state; later times: the
    analytic solution tests/emhdmodes/check.py compares with, phase advanced by omega_imag t and
    amplitude scaled by exp(omega_real t))."""
    m = EMHD_MODE
    n3, n2, n1 = spec.shape
    x1, x2, _ = cell_centers(spec)
    X1, X2 = np.meshgrid(x1, x2, indexing="xy")          # (n2, n1)
    phi = m["k1"] * X1 + m["k2"] * X2 + m["omega_imag"] * t
    c, s = np.cos(phi), np.sin(phi)
    decay = np.exp(m["omega_real"] * t)
    P = np.zeros((10, n3, n2, n1))
    for v in range(10):
        if v in (5, 6, 7):
            # the wave seed adds amp_B cos + amp2_B sin with amp_B = amp * coefficient
            P[v] = m["mean"][v] + ((amp * m["cos"][v]) * c + (amp * m["sin"][v]) * s) * decay
        else:
            P[v] = m["mean"][v] + (amp * (m["cos"][v] * c + m["sin"][v] * s)) * decay
    return P


def mhdmodes_period(nmode=3):
    return 2 * np.pi / MODES_DIR3[nmode]["omega"]


def mhdmodes_analytic(spec, nmode=3, amp=1e-4):
    """Exact linear solution after a whole number of periods: the initial mode itself."""
    return mhdmodes(spec, nmode, amp)


# ------------------------------------------------------------------------ FM torus
def _fmks(spec, X1, X2):
    """FunkyTransform (coordinate_systems.hpp:586-667): embedding r, th and dxdX entries."""
    h, ms, xt, pa, x0 = spec.hslope, spec.mks_smooth, spec.poly_xt, spec.poly_alpha, spec.startx1
    poly_norm = 0.5 * math.pi / (1. + 1. / (pa + 1.) * 1. / xt ** pa)
    r = np.exp(X1)
    thG = math.pi * X2 + ((1. - h) / 2.) * np.sin(2. * math.pi * X2)
    y = 2 * X2 - 1.
    thJ = poly_norm * y * (1. + (y / xt) ** pa / (pa + 1.)) + 0.5 * math.pi
    th = thG + np.exp(ms * (x0 - X1)) * (thJ - thG)
    d11 = np.exp(X1)
    d21 = -np.exp(ms * (x0 - X1)) * ms * (math.pi / 2. - math.pi * X2 + poly_norm * (2. * X2 - 1.)
                                           * (1 + ((-1. + 2 * X2) / xt) ** pa / (1 + pa))
                                           - 0.5 * (1. - h) * np.sin(2. * math.pi * X2))
    d22 = (math.pi + (1. - h) * math.pi * np.cos(2. * math.pi * X2)
           + np.exp(ms * (x0 - X1)) * (-math.pi + 2. * poly_norm * (1. + ((2. * X2 - 1.) / xt) ** pa / (pa + 1.))
                                       + (2. * pa * poly_norm * (2. * X2 - 1.) * ((2. * X2 - 1.) / xt) ** (pa - 1.))
                                       / ((1. + pa) * xt)
                                       - (1. - h) * math.pi * np.cos(2. * math.pi * X2)))
    return r, th, d11, d21, d22


def _lfish(a, r):
    """fm_torus.hpp:73-83: specific angular momentum of the FM solution in the midplane."""
    sqtr = math.sqrt(r)
    return ((a * a - 2. * a * sqtr + r * r) *
            ((-2. * a * r * (a * a - 2. * a * sqtr + r * r)) / math.sqrt(2. * a * sqtr + (-3. + r) * r) +
             ((a + (-2. + r) * sqtr) * (r ** 3 + a * a * (2. + r))) /
             math.sqrt(1 + (2. * a) / r ** 1.5 - 3. / r))) / \
        (r ** 3 * math.sqrt(2. * a * sqtr + (-3. + r) * r) * (a * a + (-2. + r) * r))


def _lnh(a, l, rin, r, th):
    """fm_torus.hpp:34-60: log enthalpy of the FM solution (valid for r >= rin)."""
    sth, cth = np.sin(th), np.cos(th)
    r2, a2 = r * r, a * a
    DD = r2 - 2. * r + a2
    AA = (r2 + a2) ** 2 - DD * a2 * sth * sth
    SS = r2 + a2 * cth * cth
    thin = math.pi / 2.
    sthin, cthin = math.sin(thin), math.cos(thin)
    rin2 = rin * rin
    DDin = rin2 - 2. * rin + a2
    AAin = (rin2 + a2) ** 2 - DDin * a2 * sthin * sthin
    SSin = rin2 + a2 * cthin * cthin
    val = (0.5 * np.log((1. + np.sqrt(1. + 4. * (l * l * SS * SS) * DD / (AA * AA * sth * sth))) / (SS * DD / AA))
           - 0.5 * np.sqrt(1. + 4. * (l * l * SS * SS) * DD / (AA * AA * sth * sth)) - 2. * a * r * l / AA
           - (0.5 * math.log((1. + math.sqrt(1. + 4. * (l * l * SSin * SSin) * DDin / (AAin * AAin * sthin * sthin)))
                             / (SSin * DDin / AAin))
              - 0.5 * math.sqrt(1. + 4. * (l * l * SSin * SSin) * DDin / (AAin * AAin * sthin * sthin))
              - 2. * a * rin * l / AAin))
    return np.where(r >= rin, val, 1.0)


def _torus_rho(a, rin, rmax, gam, kappa, r, th):
    l = _lfish(a, rmax)
    with np.errstate(all="ignore"):
        lnh = _lnh(a, l, rin, r, th)
        hm1 = np.exp(lnh) - 1.
        rho = np.power(np.maximum(hm1, 0.0) * (gam - 1.) / (kappa * gam), 1. / (gam - 1.))
    return np.where((lnh >= 0.) & (r >= rin), rho, 0.0)


def fm_torus(spec, geom, rin=6.0, rmax=12.0, kappa=1e-3, beta_min=100.0, u_jitter=0.08, seed=1234, faces=False,
             rho_max=None):
    """Fishbone-Moncrief torus + SANE field, on a spherical-KS FMKS block.

    geom: dict with the centre tables 'gcov', 'gcon' (arrays [7][n2+1][n1+1][4][4]) and 'gdet'
    from khb_build_geometry.  The field is A_phi = max(rho/rho_max - 0.2, 0) at zone corners,
    curled with the flux-CT averaged curl and normalised so max(p_gas)/max(p_B) = beta_min.
    faces=True also returns the B_CT face field sqrt(-g) B^d (3, n3, n2, n1): the face curl of the
    same A_phi with the same normalisation (B_CT's seeding, divergence-free to rounding).
    rho_max: the density normalisation (default: the midplane maximum over this block's x1 range,
    as the reference takes it over the mesh's; a block of a mesh passes the mesh's).
    """
    gam, a = spec.gam, spec.a
    n3, n2, n1 = spec.shape
    x1, x2, x3 = cell_centers(spec)
    X1, X2 = np.meshgrid(x1, x2, indexing="xy")              # (n2, n1)
    r, th, d11, d21, d22 = _fmks(spec, X1, X2)
    sth, cth = np.sin(th), np.cos(th)
    l = _lfish(a, rmax)
    with np.errstate(all="ignore"):
        lnh = _lnh(a, l, rin, r, th)
    inside = (lnh >= 0.) & (r >= rin)
    r2, a2 = r * r, a * a
    DD = r2 - 2. * r + a2
    AA = (r2 + a2) ** 2 - DD * a2 * sth * sth
    SS = r2 + a2 * cth * cth
    with np.errstate(all="ignore"):
        hm1 = np.exp(lnh) - 1.
        rho_l = np.power(np.maximum(hm1, 0) * (gam - 1.) / (kappa * gam), 1. / (gam - 1.))
        u_l = kappa * np.power(rho_l, gam) / (gam - 1.)
        expm2chi = SS * SS * DD / (AA * AA * sth * sth)
        up1 = np.sqrt((-1. + np.sqrt(1. + 4. * l * l * expm2chi)) / 2.)
        up = 2. * a * r * np.sqrt(1. + up1 * up1) / np.sqrt(AA * SS * DD) + np.sqrt(SS / AA) * up1 / sth
    # u^t from the BL metric (coordinate_utils.hpp:170-187), then BL -> KS (coordinate_systems.hpp:152-163)
    mmu = 1. + a2 * cth * cth / r2
    g00 = -(1. - 2. / (r * mmu))
    g03 = -2. * a * sth * sth / (r * mmu)
    g33 = sth * sth * (r2 + a2 + 2. * a2 * sth * sth / (r * mmu))
    AAq, BBq, CCq = g00, 2. * g03 * up, 1. + g33 * up * up
    with np.errstate(all="ignore"):
        ut_bl = (-BBq - np.sqrt(BBq * BBq - 4. * AAq * CCq)) / (2. * AAq)
    # KS: u^t += 2r/(r^2-2r+a^2) u^r (u^r = 0 here), u^phi += a/(...) u^r -> unchanged
    ucon_ks = [ut_bl, np.zeros_like(r), np.zeros_like(r), up]
    # KS -> native: dXdx = inverse of dxdX (only the (1,2) block is non-trivial)
    det = d11 * d22
    u1n = ucon_ks[1] / d11
    u2n = (-d21 * ucon_ks[1] + d11 * ucon_ks[2]) / det
    ucon_n = [ucon_ks[0], u1n, u2n, ucon_ks[3]]
    gcon = np.asarray(geom["gcon"])[3, :n2, :n1]             # centre, (n2, n1, 4, 4)
    alpha2 = -1.0 / gcon[..., 0, 0]
    uprim = [ucon_n[1 + v] + ucon_n[0] * alpha2 * gcon[..., 0, 1 + v] for v in range(3)]
    # rho_max along the midplane (fm_torus.cpp:145-169)
    if rho_max is None:
        xs = spec.x1min + np.arange(int((spec.x1max - spec.x1min) / 0.001) + 1) * 0.001
        rho_max = float(np.max(_torus_rho(a, rin, rmax, gam, kappa, np.exp(xs), np.full_like(xs, math.pi / 2))))
    P = np.zeros((spec.nvar, n3, n2, n1))
    for plane, val in ((0, rho_l / rho_max), (1, u_l / rho_max), (2, uprim[0]), (3, uprim[1]), (4, uprim[2])):
        P[plane] = np.where(inside, val, 0.0)[None, :, :]
    # initial fluid-frame floors over the whole block (floors.cpp:132-210; B = 0 at this point)
    fl = spec.floors
    rhoscal = 1. / np.sqrt(r * r * r)
    rhoflr = np.maximum(fl.rho_min_geom * rhoscal, fl.rho_min_const)
    uflr = np.maximum(fl.u_min_geom * rhoscal ** gam, fl.u_min_const)
    P[1] = np.maximum(P[1], uflr[None])
    rhoflr_temp = np.maximum(P[1], uflr[None]) / fl.u_over_rho_max
    P[0] = np.maximum(P[0], np.maximum(rhoflr[None], rhoflr_temp))
    # u jitter where rho is above the floor (perturbation.hpp:81-110)
    rng = np.random.Generator(np.random.PCG64(seed))
    jit = rng.uniform(-u_jitter / 2, u_jitter / 2, size=P[1].shape)
    P[1] = np.where(P[0] > fl.rho_min_geom, P[1] * (1. + jit), P[1])
    Bf = None
    if spec.nvar > 5:
        Bf = _seed_sane(spec, geom, P, a, rin, rmax, gam, kappa, rho_max, beta_min)
    return (P, Bf) if faces else P


def _seed_sane(spec, geom, P, a, rin, rmax, gam, kappa, rho_norm, beta_min):
    """A_phi at corners, averaged curl (b_flux_ct_functions.hpp:109-166), legacy beta normalisation
    (seed_B.cpp:464-534)."""
    n3, n2, n1 = spec.shape
    dx1, dx2, _ = spec.dx
    g2 = spec.ng if spec.nx2 > 1 else 0
    x1f = (spec.x1min - spec.ng * dx1) + np.arange(n1 + 1) * dx1
    x2f = (spec.x2min - g2 * dx2) + np.arange(n2 + 1) * dx2
    X1, X2 = np.meshgrid(x1f, x2f, indexing="xy")            # corners (n2+1, n1+1)
    r, th, _, _, _ = _fmks(spec, X1, X2)
    A = np.maximum(_torus_rho(a, rin, rmax, gam, kappa, r, th) / rho_norm - 0.2, 0.)
    # x3-independent A: the 3D average over k and k+1 equals the 2D average
    A3c2f = (A[1:, :-1] + A[1:, 1:]) / 2
    A3c2b = (A[:-1, :-1] + A[:-1, 1:]) / 2
    A3c1f = (A[:-1, 1:] + A[1:, 1:]) / 2
    A3c1b = (A[:-1, :-1] + A[1:, :-1]) / 2
    BU1 = (A3c2f - A3c2b) / dx2
    BU2 = -(A3c1f - A3c1b) / dx1
    gdet = np.asarray(geom["gdet"])[3, :n2, :n1]
    P[5] = (BU1 / gdet)[None]
    P[6] = (BU2 / gdet)[None]
    P[7] = 0.0
    # legacy normalisation: beta_min = max(p_gas) / (0.5 max(b^2)) over the interior
    gcov = np.asarray(geom["gcov"])[3, :n2, :n1]
    gcon = np.asarray(geom["gcon"])[3, :n2, :n1]
    sl = spec.interior
    bsq = _bsq(P[:, sl[0], sl[1], sl[2]], gcov[sl[1], sl[2]], gcon[sl[1], sl[2]])
    bsq_max = float(np.max(bsq))
    p_max = float(np.max((gam - 1.) * P[1][sl]))
    beta_now = p_max / (0.5 * bsq_max)
    norm = math.sqrt(beta_now / beta_min)
    P[5:8] *= norm
    # the face curl (A_3 at the corners of face i's lower edge): sqrt(-g) B^1 on x1 faces, B^2 on x2
    Bf = np.zeros((3,) + spec.shape)
    Bf[0] = (norm * (A[1:, :-1] - A[:-1, :-1]) / dx2)[None]
    Bf[1] = (-norm * (A[:-1, 1:] - A[:-1, :-1]) / dx1)[None]
    return Bf


def _bsq(P, gcov, gcon):
    """b^2 at zone centres from primitives (grmhd_functions.hpp:165-246)."""
    u1, u2, u3 = P[2], P[3], P[4]
    g = gcov
    qsq = (g[..., 1, 1] * u1 * u1 + g[..., 2, 2] * u2 * u2 + g[..., 3, 3] * u3 * u3 +
           2. * (g[..., 1, 2] * u1 * u2 + g[..., 1, 3] * u1 * u3 + g[..., 2, 3] * u2 * u3))
    gamma = np.sqrt(1. + qsq)
    alpha = 1. / np.sqrt(-gcon[..., 0, 0])
    ucon = np.stack([gamma / alpha] + [P[2 + v] - gamma * alpha * gcon[..., 0, 1 + v] for v in range(3)])
    ucov = np.einsum("...mn,n...->m...", g, ucon)
    b0 = sum(P[5 + v] * ucov[1 + v] for v in range(3))
    bcon = np.stack([b0] + [(P[5 + v] + b0 * ucon[1 + v]) / ucon[0] for v in range(3)])
    bcov = np.einsum("...mn,n...->m...", g, bcon)
    return np.sum(bcon * bcov, axis=0)


def conducting_atmosphere(spec, geom, emhd, profile, jitter=1e-3, seed=1234, B10=1.0):
    """Hydrostatic conducting atmosphere in Schwarzschild/MKS (prob/emhd/conducting_atmosphere.cpp:52-240).

    profile: dict with the radial ODE solution arrays 'rCoords', 'rho', 'u', 'phi', one entry per
    radial zone including ghosts (the reference reads them from atmosphere_soln_*.txt).  The fluid
    is at rest with respect to the normal observer (u^mu = (1/sqrt(-g_00), 0, 0, 0)), q = phi
    converted to q~ by the higher-order-terms scaling, dP~ = 0, and a monopole field
    B^1 = B10 / r^3 (prob/seed_B.hpp:155-158).  rho, u and q~ are then multiplied by
    (1 + jitter * U(-1, 1)) from a seeded PCG64 stream.  Returns P with 10 slots
    (rho, u, u1-u3, B1-B3, q~, dP~) over the entire block.
    """
    n3, n2, n1 = spec.shape
    gam = spec.gam
    rc = np.asarray(geom["r_center"])[:, :n1]                    # (n2, n1)
    if len(profile["rCoords"]) != n1 or np.max(np.abs(rc - profile["rCoords"][None, :])) > 1e-10:
        raise ValueError("atmosphere profile does not match the grid radii")
    gcov = np.asarray(geom["gcov"])[3, :n2, :n1]
    gcon = np.asarray(geom["gcon"])[3, :n2, :n1]
    rho = np.broadcast_to(profile["rho"][None, :], (n2, n1))
    u = np.broadcast_to(profile["u"][None, :], (n2, n1))
    q = np.broadcast_to(profile["phi"][None, :], (n2, n1)).copy()
    ucon0 = 1.0 / np.sqrt(-gcov[..., 0, 0])
    alpha2 = -1.0 / gcon[..., 0, 0]
    uprim = [ucon0 * alpha2 * gcon[..., 0, 1 + v] for v in range(3)]
    if emhd.higher_order_terms:
        Theta = (gam - 1.) * u / rho
        # EMHD::set_parameters with q = dP = bsq = 0 (emhd.hpp:179-261)
        cs2 = gam * (gam - 1.) * u / (rho + gam * u)
        if emhd.closure_type == "kappa_eta":
            tau, chi = emhd.tau, emhd.kappa / np.maximum(rho, 1e-20)
        elif emhd.closure_type == "constant":
            tau, chi = emhd.tau, np.full_like(rho, emhd.conduction_alpha)
        elif emhd.closure_type in ("soundspeed", "sound_speed"):
            tau = emhd.tau
            chi = emhd.conduction_alpha * cs2 * tau
        else:
            tau = np.sqrt(rc ** 3)
            cs2 = np.maximum(cs2, 1e-20)
            max_alpha = (1 - cs2) / (2 * cs2 + 1.e-12)
            chi = np.minimum(max_alpha, emhd.conduction_alpha) * cs2 * tau
        q = q * np.where(chi != 0, np.sqrt(tau / (chi * rho * Theta * Theta)), 0.0)
    P = np.zeros((10, n3, n2, n1))
    P[0], P[1], P[8] = rho[None], u[None], q[None]
    for v in range(3):
        P[2 + v] = uprim[v][None]
    P[5] = (B10 / rc ** 3)[None]
    if jitter:
        rng = np.random.Generator(np.random.PCG64(seed))
        for plane in (0, 1, 8):
            P[plane] *= 1.0 + jitter * rng.uniform(-1.0, 1.0, size=P[plane].shape)
    return P


# ------------------------------------------------------------------------ Bondi accretion
def _bondi_T(r, C1, C2, n, rs):
    """bondi.hpp get_T: bisection for the temperature on the inflowing branch, vectorised with a
    per-zone stopping mask (rtol 1e-12, ftol 1e-14 as in the reference)."""
    rtol, ftol = 1.e-12, 1.e-14

    def tfunc(T):
        A = 1. + (1. + n) * T
        B = C1 / (r * r * np.power(T, n))
        return A * A * (1. - 2. / r + B * B) - C2

    Tinf = (math.sqrt(C2) - 1.) / (n + 1)
    Tnear = np.power(C1 * np.sqrt(2. / (r * r * r)), 1. / n)
    Tmin = np.where(r < rs, Tinf, np.maximum(Tnear, Tinf))
    Tmax = np.where(r < rs, Tnear, 1.0)
    T0, T1 = Tmin.copy(), Tmax.copy()
    f0, f1 = tfunc(T0), tfunc(T1)
    bad = f0 * f1 > 0
    Th = (T0 + T1) / 2.
    fh = tfunc(Th)
    epsT = rtol * (Tmin + Tmax)
    for _ in range(200):
        go = (np.abs(Th - T0) > epsT) & (np.abs(Th - T1) > epsT) & (np.abs(fh) > ftol)
        if not go.any():
            break
        up = go & (fh * f0 > 0.)
        dn = go & ~(fh * f0 > 0.)
        T0 = np.where(up, Th, T0)
        f0 = np.where(up, fh, f0)
        T1 = np.where(dn, Th, T1)
        f1 = np.where(dn, fh, f1)
        Th = np.where(go, (T0 + T1) / 2., Th)
        fh = np.where(go, tfunc(Th), fh)
    return np.where(bad, -1., Th)


def bondi_solution(r, rs=8.0, mdot=1.0, gam=5.0 / 3.0):
    """bondi.hpp get_bondi_soln: rho, u and the Boyer-Lindquist u^r of the steady Bondi inflow."""
    n = 1. / (gam - 1.)
    uc = math.sqrt(1. / (2. * rs))
    Vc = math.sqrt(uc * uc / (1. - 3. * uc * uc))
    Tc = -n * Vc * Vc / ((n + 1.) * (n * Vc * Vc - 1.))
    C1 = uc * rs * rs * Tc ** n
    A = 1. + (1. + n) * Tc
    C2 = A * A * (1. - 2. / rs + uc * uc)
    K = (4 * math.pi * C1 / mdot) ** (1 / n)
    Kn = K ** n
    T = _bondi_T(r, C1, C2, n, rs)
    Tn = np.power(T, n)
    rho = Tn / Kn
    u = rho * T * n
    ur = -C1 / (Tn * r * r)
    return rho, u, ur


def bondi(spec, geom, rs=8.0, mdot=1.0):
    """Bondi inflow on a spherical-KS (a = 0) MKS block, every zone including the ghosts set to the
    analytic solution (prob/bondi.hpp get_prim_bondi with ur_frac = 1, uphi = 0, no diffinit):
    u^r in Boyer-Lindquist, u^t from the BL metric (set_ut, coordinate_utils.hpp:170-187), BL -> KS
    (coordinate_systems.hpp:154-164), KS -> native through dX/dx of MKS, then the primitive
    velocity (fourvel_to_prim, coordinate_utils.hpp:195-202)."""
    assert spec.base == "spherical_ks" and spec.transform == "mks" and spec.a == 0.0
    n3, n2, n1 = spec.shape
    x1, x2, _ = cell_centers(spec)
    X1, _ = np.meshgrid(x1, x2, indexing="xy")              # (n2, n1)
    r = np.exp(X1)
    rho, u, ur = bondi_solution(r, rs, mdot, spec.gam)
    # BL metric at a = 0: g_tt = -(1 - 2/r), g_rr = 1/(1 - 2/r); u^t from the normalisation
    AA = -(1. - 2. / r)
    CC = 1. + (1. / (1. - 2. / r)) * ur * ur
    ut_bl = (-0. - np.sqrt(0. - 4. * AA * CC)) / (2. * AA)
    ut_ks = ut_bl + (2. * r / (r * r - 2. * r)) * ur
    # MKS: r = exp(X1), dr/dX1 = r; theta depends on X2 only, u^theta = 0
    ucon = [ut_ks, ur / r, np.zeros_like(r), np.zeros_like(r)]
    gcon = np.asarray(geom["gcon"])[3, :n2, :n1]
    alpha2 = -1.0 / gcon[..., 0, 0]
    uprim = [ucon[1 + v] + ucon[0] * alpha2 * gcon[..., 0, 1 + v] for v in range(3)]
    P = np.zeros((spec.nvar, n3, n2, n1))
    for p, val in enumerate((rho, u, uprim[0], uprim[1], uprim[2])):
        P[p] = val[None, :, :]
    return P


# ------------------------------------------------------------------------ derivative-check states
def add_ramps(spec, P, frac=0.05, seed=9):
    """P_q + amp_q (a x1' + b x2' + c x3'), x' the native coordinates normalised to [-1/2, 1/2] over the
    interior, seeded a, b, c in [1/2, 3/2], amp_q = frac times the variable's mean magnitude (1e-3 for
    a variable that is zero).  A state with no flat neighbourhood in any variable or direction: at a
    flat neighbourhood the MC-limited slope is not differentiable, so derivative checks start here."""
    rng = np.random.Generator(np.random.PCG64(seed))
    x1, x2, x3 = cell_centers(spec)
    nrm = lambda x, lo, hi: (x - 0.5 * (lo + hi)) / (hi - lo)
    X3, X2, X1 = np.meshgrid(nrm(x3, spec.x3min, spec.x3max), nrm(x2, spec.x2min, spec.x2max),
                             nrm(x1, spec.x1min, spec.x1max), indexing="ij")
    sc = np.abs(P).mean(axis=(1, 2, 3))
    amp = np.where(sc > 1e-12, frac * sc, 1e-3)
    P = P.copy()
    for q in range(P.shape[0]):
        a, b, c = rng.uniform(0.5, 1.5, 3)
        P[q] += amp[q] * (a * X1 + (b * X2 if spec.nx2 > 1 else 0) + (c * X3 if spec.nx3 > 1 else 0))
    return P


# ------------------------------------------------------------------------ B_CT face fields
def ct_curl_faces(spec, B0=(1.0, 0.0, 0.0), amp=0.05):
    """A face field sqrt(-g) B^d (3, n3, n2, n1) on a Cartesian Minkowski block (sqrt(-g) = 1): the
    uniform B0 plus the discrete curl of A_3 = amp sin(2 pi x1) cos(2 pi x2) sampled at the zone
    corners, so that the face divergence vanishes to rounding.  Face i of direction d is the lower
    x_d face of zone i."""
    assert spec.cart_minkowski
    n3, n2, n1 = spec.shape
    dx1, dx2, _ = spec.dx
    g2 = spec.ng if spec.nx2 > 1 else 0
    xf = spec.x1min + (np.arange(n1 + 1) - spec.ng) * dx1          # corner x1 of zone i (lower)
    yf = spec.x2min + (np.arange(n2 + 1) - g2) * dx2
    Y, X = np.meshgrid(yf, xf, indexing="ij")                     # (n2+1, n1+1)
    A = amp * np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y)
    Bf = np.zeros((3,) + spec.shape)
    Bf[0] = B0[0] + ((A[1:, :-1] - A[:-1, :-1]) / dx2)[None]       # (A(i, j+1) - A(i, j)) / dx2
    Bf[1] = B0[1] - ((A[:-1, 1:] - A[:-1, :-1]) / dx1)[None]       # -(A(i+1, j) - A(i, j)) / dx1
    Bf[2] = B0[2]
    return Bf



# ------------------------------------------------------------------------ hydro entropy wave
def entropy_wave(spec, amp=0.1, v=(0.3, 0.2, 0.1), t=0.0, gam=None):
    """Hydro (5-variable) entropy wave on a periodic unit box in Minkowski space: rho = 1 + amp
    sin(2 pi (x1 + x2 + x3 - (v1 + v2 + v3) t)) over the active directions, uniform pressure (u = 1)
    and uniform 3-velocity v (primitive u^i = W v^i).  An exact solution, advected at v."""
    n3, n2, n1 = spec.shape
    x1, x2, x3 = cell_centers(spec)
    X3, X2, X1 = np.meshgrid(x3, x2, x1, indexing="ij")
    ph = X1 - v[0] * t
    vv = [v[0], 0.0, 0.0]
    if spec.nx2 > 1:
        ph = ph + X2 - v[1] * t
        vv[1] = v[1]
    if spec.nx3 > 1:
        ph = ph + X3 - v[2] * t
        vv[2] = v[2]
    W = 1.0 / math.sqrt(1.0 - sum(c * c for c in vv))
    P = np.zeros((5, n3, n2, n1))
    P[0] = 1.0 + amp * np.sin(2 * np.pi * ph)
    P[1] = 1.0
    for d in range(3):
        P[2 + d] = W * vv[d]
    return P

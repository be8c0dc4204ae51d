"""Block and package options, mirroring the KHARMA parameter blocks the hot path reads.

A BlockSpec carries what the Flux, B_FluxCT, Inverter, Floors, Boundaries and GRMHD packages
put in their Params for one meshblock, and converts it to the khb_config / khb_coords structs
of the C ABI.  Defaults follow the reference's GetOrAdd* defaults (cited per field group).
"""
from typing import Optional
from dataclasses import dataclass, field
import math

from . import _lib


@dataclass
class FloorSpec:
    """Floors::Prescription (floors/floors.hpp:100-167).  Defaults are the spherical ones."""
    rho_min_const: float = 1e-20
    u_min_const: float = 1e-20
    rho_min_geom: float = 1e-6
    u_min_geom: float = 1e-8
    r_char: float = 10.0
    bsq_over_rho_max: float = 1e20
    bsq_over_u_max: float = 1e20
    u_over_rho_max: float = 1e20
    ktot_max: float = 1e20
    gamma_max: float = 50.0
    use_r_char: bool = False
    temp_adjust_u: bool = False
    adjust_k: bool = True
    radius_dependent_floors: bool = False
    floors_switch_r: float = 50.0

    def to_struct(self):
        s = _lib.KhbFloors()
        for name, _ in _lib.KhbFloors._fields_:
            setattr(s, name, type(getattr(s, name))(getattr(self, name)))
        return s


@dataclass
class BlockSpec:
    # parthenon/meshblock and parthenon/mesh
    nx1: int
    nx2: int
    nx3: int
    x1min: float
    x1max: float
    x2min: float
    x2max: float
    x3min: float
    x3max: float
    ng: int = 4                         # driver/nghost (kharma.cpp:151)
    # GRMHD
    gam: float = 4.0 / 3.0
    nvar: int = 8                       # 8: GRMHD + flux-CT B field; 5: GRHD
    cfl: float = 0.9                    # GRMHD/cfl (grmhd.cpp:83)
    dt_min: float = 1e-5                # parthenon/time/dt_min (grmhd.cpp:88)
    max_dt_increase: float = 2.0        # parthenon/time/max_dt_increase (grmhd.cpp:93)
    # Flux (flux.cpp:52-242)
    recon: str = "weno5"
    riemann: str = "llf"
    precision: str = "fp64"
    recon_floors: bool = False
    low_order_edges: bool = False       # flux/low_order_edges (weno5 only)
    low_order_poles: bool = False       # flux/low_order_poles (weno5 only)
    recon_fallback: bool = False        # flux/reconstruction_fallback
    # coordinates (coordinate_embedding.hpp:119-210)
    base: str = "cartesian_minkowski"
    transform: str = "null"
    a: float = 0.0
    hslope: float = 0.3
    mks_smooth: float = 0.5
    poly_xt: float = 0.82
    poly_alpha: float = 14.0
    startx1: float = 0.0
    # boundaries (boundaries.cpp:57-368, kharma.cpp:238-253)
    bc: tuple = ("periodic",) * 6
    check_inflow_inner_x1: bool = False
    check_inflow_outer_x1: bool = False
    zero_polar_flux: bool = False
    fix_polar_flux: bool = False
    fix_corner_inner: bool = False
    # floors (floors.cpp:40-130)
    floors_on: bool = False
    floor_frame: str = "drift"
    floors: FloorSpec = field(default_factory=FloorSpec)
    # floors_inner block (used inside floors.floors_switch_r when floors.radius_dependent_floors; None:
    # the same as floors) and the switch points of the mixed injection frames
    floors_inner: Optional[FloorSpec] = None
    frame_switch_r: float = 50.0
    frame_switch_beta: float = 10.0
    # inverter (inverter.cpp:46-115): 1D_W (8 iterations, 1e-8) or Kastaun (25, 1e-12)
    inverter: str = "onedw"
    iter_max: int = 8
    err_tol: float = 1e-8
    fix_average_neighbors: bool = True
    fix_atmosphere: bool = True
    # first-order flux correction (flux.cpp:175-221)
    fofc: bool = False
    fofc_polar_cells: int = 0
    fofc_eh_buffer: float = 0.1
    fofc_use_glf: bool = False               # fofc/use_glf: speed-of-light LF speeds on replaced faces
    fofc_use_source_term: bool = False       # fofc/use_source_term: the guess takes the geometric source
    # magnetic field transport (b_field/solver, b_field/ct_scheme): "none" = B_FluxCT (cell-centred B);
    # "bs99", "gs05_0", "gs05_c" ("sg07") = B_CT with a face-centred field
    b_ct: str = "none"
    # driver
    driver: str = "simple"

    @property
    def ndim(self):
        return 1 + (self.nx2 > 1) + (self.nx3 > 1)

    @property
    def dx(self):
        return ((self.x1max - self.x1min) / self.nx1, (self.x2max - self.x2min) / self.nx2,
                (self.x3max - self.x3min) / self.nx3)

    @property
    def shape(self):
        """Entire-block shape (n3, n2, n1) including ghosts."""
        n1 = self.nx1 + 2 * self.ng
        n2 = self.nx2 + 2 * self.ng if self.nx2 > 1 else 1
        n3 = self.nx3 + 2 * self.ng if self.nx3 > 1 else 1
        return (n3, n2, n1)

    @property
    def interior(self):
        """Slices (k, j, i) of the interior zones."""
        ng = self.ng
        sk = slice(ng, ng + self.nx3) if self.nx3 > 1 else slice(0, 1)
        sj = slice(ng, ng + self.nx2) if self.nx2 > 1 else slice(0, 1)
        return (sk, sj, slice(ng, ng + self.nx1))

    @property
    def spherical(self):
        return self.base != "cartesian_minkowski"

    @property
    def cart_minkowski(self):
        return self.base == "cartesian_minkowski" and self.transform == "null"

    def khb_config(self):
        c = _lib.KhbConfig()
        c.nx1, c.nx2, c.nx3, c.ng = self.nx1, self.nx2, self.nx3, self.ng
        c.dx1, c.dx2, c.dx3 = self.dx
        c.gam = self.gam
        c.nvar = self.nvar
        c.recon = _lib.RECON[self.recon]
        c.riemann = _lib.FLUX[self.riemann]
        c.precision = _lib.PREC[self.precision]
        for x in range(6):
            c.bc[x] = _lib.BC[self.bc[x]]
        c.check_inflow_inner_x1 = int(self.check_inflow_inner_x1)
        c.check_inflow_outer_x1 = int(self.check_inflow_outer_x1)
        c.zero_polar_flux = int(self.zero_polar_flux)
        c.fix_polar_flux = int(self.fix_polar_flux)
        c.fix_corner_inner = int(self.fix_corner_inner)
        c.spherical = int(self.spherical)
        c.cart_minkowski = int(self.cart_minkowski)
        c.floors_on = int(self.floors_on)
        c.floor_frame = _lib.FRAME[self.floor_frame]
        c.recon_floors = int(self.recon_floors)
        c.iter_max = self.iter_max
        c.err_tol = self.err_tol
        c.fix_average_neighbors = int(self.fix_average_neighbors)
        c.fix_atmosphere = int(self.fix_atmosphere)
        c.floors = self.floors.to_struct()
        c.floors_inner = (self.floors_inner or self.floors).to_struct()
        c.frame_switch_r, c.frame_switch_beta = self.frame_switch_r, self.frame_switch_beta
        c.inverter = _lib.INVERTER[self.inverter]
        c.fofc, c.fofc_polar_cells, c.fofc_eh_buffer = int(self.fofc), self.fofc_polar_cells, self.fofc_eh_buffer
        c.fofc_use_glf, c.fofc_use_source_term = int(self.fofc_use_glf), int(self.fofc_use_source_term)
        c.r_horizon = self.r_horizon
        c.ct_scheme = _lib.CT_SCHEME[self.b_ct]
        c.recon_lower = 1 if self.low_order_edges else (2 if self.low_order_poles else 0)
        c.recon_fallback = int(self.recon_fallback)
        return c

    @property
    def r_horizon(self):
        """Event-horizon radius of the coordinates (coordinate_embedding.hpp:247-258)."""
        if self.base in ("spherical_ks", "spherical_bl"):
            return 1.0 + math.sqrt(1.0 - self.a * self.a)
        return 0.0

    def khb_coords(self):
        s = _lib.KhbCoords()
        s.base = _lib.BASE[self.base]
        s.transform = _lib.TRANSFORM[self.transform]
        s.a, s.hslope, s.mks_smooth = self.a, self.hslope, self.mks_smooth
        s.poly_xt, s.poly_alpha, s.startx1 = self.poly_xt, self.poly_alpha, self.startx1
        return s


def mhdmodes_spec(n1, n2, n3, recon="weno5", riemann="llf", precision="fp64", driver="simple"):
    """pars/tests/mhdmodes.par: periodic [0,1]^3 Minkowski box, gamma 4/3, CFL 0.9, dt_min 1e-4,
    floors off, 1D_W inverter (set explicitly: the reference default is Kastaun)."""
    return BlockSpec(nx1=n1, nx2=n2, nx3=n3, x1min=0.0, x1max=1.0, x2min=0.0, x2max=1.0,
                     x3min=0.0, x3max=1.0, gam=4.0 / 3.0, nvar=8, cfl=0.9, dt_min=1e-4,
                     recon=recon, riemann=riemann, precision=precision, driver=driver,
                     floors=FloorSpec(rho_min_const=1e-8, u_min_const=1e-10, rho_min_geom=0., u_min_geom=0.))


def torus_spec(n1, n2, n3, r_out=1000.0, a=0.9375, recon="linear_mc", precision="fp64", gam=13.0 / 9.0,
               driver="kharma", inverter="onedw", fofc=False):
    """FM torus in funky-MKS coordinates (kharma.cpp:144-316 domain logic; pars/benchmark decks).

    x1 spans [x1min, log(r_out)] with x1min chosen to put 5.5 zones inside the horizon, x2 in [0,1],
    x3 in [0, 2 pi].  Boundaries: outflow X1 with inflow checks, reflecting X2 with polar flux
    fixes and the corner fix, periodic X3.  Floors in the drift frame (floors.cpp:68) with the
    benchmark deck's magnetization/temperature ceilings.
    """
    rhor = 1.0 + math.sqrt(1.0 - a * a)
    x1max = math.log(r_out)
    x1hor = math.log(rhor)
    x1min = (n1 * x1hor / 5.5 - x1max) / (-1.0 + n1 / 5.5)
    return BlockSpec(nx1=n1, nx2=n2, nx3=n3, x1min=x1min, x1max=x1max, x2min=0.0, x2max=1.0,
                     x3min=0.0, x3max=2 * math.pi, gam=gam, nvar=8, cfl=0.9, dt_min=1e-5,
                     recon=recon, riemann="llf", precision=precision,
                     base="spherical_ks", transform="fmks", a=a, hslope=0.3, mks_smooth=0.5,
                     poly_xt=0.82, poly_alpha=14.0, startx1=x1min,
                     bc=("outflow", "outflow", "reflecting", "reflecting", "periodic", "periodic"),
                     check_inflow_inner_x1=True, check_inflow_outer_x1=True,
                     zero_polar_flux=True, fix_polar_flux=True, fix_corner_inner=True,
                     floors_on=True, floor_frame="drift",
                     floors=FloorSpec(rho_min_geom=1e-6, u_min_geom=1e-8, bsq_over_rho_max=100.0,
                                      u_over_rho_max=2.0),
                     driver=driver, inverter=inverter,
                     # inverter.cpp:66-92: Kastaun defaults to 25 iterations to 1e-12 and to the
                     # atmosphere fixup without neighbour averaging
                     iter_max=25 if inverter == "kastaun" else 8,
                     err_tol=1e-12 if inverter == "kastaun" else 1e-8,
                     fix_average_neighbors=inverter != "kastaun",
                     fofc=fofc)


def bondi_spec(nx1, nx2, nx3, x1min, x1max, x2min=0.0, x2max=1.0, x3min=0.0, x3max=2 * math.pi,
               precision="fp64", recon="weno5", bc=("exchange",) * 6):
    """One meshblock of the Bondi problem (pars/bondi/bondi.par): spherical KS at a = 0 in MKS
    coordinates (hslope 0.3), gamma 5/3, WENO5, LLF, hydro only (b_field none: 5 variables),
    floors off.  The block covers the given native-coordinate ranges; by default every face is an
    exchange face whose ghost zones the caller fills (here: with the analytic solution)."""
    return BlockSpec(nx1=nx1, nx2=nx2, nx3=nx3, x1min=x1min, x1max=x1max, x2min=x2min, x2max=x2max,
                     x3min=x3min, x3max=x3max, gam=5.0 / 3.0, nvar=5, cfl=0.9, dt_min=1e-5,
                     recon=recon, riemann="llf", precision=precision,
                     base="spherical_ks", transform="mks", a=0.0, hslope=0.3,
                     bc=tuple(bc), floors_on=False, driver="kharma")


@dataclass
class EmhdSpec:
    """EMHD package options (emhd/emhd.cpp:60-130).  Defaults are the reference's GetOrAdd defaults."""
    closure_type: str = "torus"
    higher_order_terms: bool = False
    feedback: bool = True
    conduction: bool = True
    viscosity: bool = True
    tau: float = 1.0
    conduction_alpha: float = 1.0
    viscosity_alpha: float = 1.0
    kappa: float = 1.0
    eta: float = 1.0
    # emhd/stability_limits (emhd.cpp:118-125): limit q and dP to the instability bounds after the solve
    stability_limits: bool = False

    @property
    def nfvar(self):
        """Implicitly evolved variables: rho, u, u1-u3, then q and dP when present."""
        return 5 + int(self.conduction) + int(self.viscosity)

    def to_struct(self):
        s = _lib.KhbEmhdParams()
        s.closure = _lib.CLOSURE[self.closure_type]
        s.higher_order_terms, s.feedback = int(self.higher_order_terms), int(self.feedback)
        s.conduction, s.viscosity = int(self.conduction), int(self.viscosity)
        s.stability_limits = int(self.stability_limits)
        s.tau, s.conduction_alpha, s.viscosity_alpha = self.tau, self.conduction_alpha, self.viscosity_alpha
        s.kappa, s.eta = self.kappa, self.eta
        return s


@dataclass
class ImplicitSpec:
    """Implicit package options (implicit/implicit.cpp:99-119); jacobian selects the reference's
    forward-difference Jacobian ("fd") or the exact tangent Jacobian ("exact")."""
    min_nonlinear_iter: int = 1
    max_nonlinear_iter: int = 3
    jacobian_delta: float = 4e-8
    rootfind_tol: float = 1e-12
    use_qr: bool = True
    linesearch: bool = True
    max_linesearch_iter: int = 3
    linesearch_eps: float = 1e-4
    linesearch_lambda: float = 1.0
    jacobian: str = "fd"

    def to_struct(self):
        s = _lib.KhbImplicitParams()
        s.min_nonlinear_iter, s.max_nonlinear_iter = self.min_nonlinear_iter, self.max_nonlinear_iter
        s.use_qr, s.linesearch, s.max_linesearch_iter = int(self.use_qr), int(self.linesearch), self.max_linesearch_iter
        s.jacobian = _lib.JACOBIAN[self.jacobian]
        s.jacobian_delta, s.rootfind_tol = self.jacobian_delta, self.rootfind_tol
        s.linesearch_eps, s.linesearch_lambda = self.linesearch_eps, self.linesearch_lambda
        return s


def atmosphere_spec(n1, n2, n3, r_in=200.0, r_out=300.0):
    """Conducting-atmosphere geometry (tests/conducting_atmosphere/conducting_atmosphere.par):
    Schwarzschild (KS, a = 0) in MKS with hslope = 1, r in [r_in, r_out], gamma 4/3, WENO5/LLF.
    Boundaries are not part of the implicit operator; outflow/reflecting/periodic are set."""
    return BlockSpec(nx1=n1, nx2=n2, nx3=n3, x1min=math.log(r_in), x1max=math.log(r_out),
                     x2min=0.0, x2max=1.0, x3min=0.0, x3max=2 * math.pi, gam=4.0 / 3.0, nvar=8,
                     recon="weno5", riemann="llf", base="spherical_ks", transform="mks", a=0.0, hslope=1.0,
                     bc=("outflow", "outflow", "reflecting", "reflecting", "periodic", "periodic"),
                     floors_on=False, driver="kharma")

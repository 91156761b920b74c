"""Mesh-block options for the hydro step, read from snapy's YAML files.

``HydroConfig`` is the ctypes mirror of ``snapb_hydro_config`` in
``include/snapb.h``.  ``from_yaml`` reads the keys that the reference's
``MeshBlockOptionsImpl::from_yaml`` and the module ``*OptionsImpl::from_yaml``
functions read for this path, with the same defaults:

* geometry.{type,bounds,cells}             src/coord/coordinate.cpp:58-166
* dynamics.equation-of-state.*             src/eos/equation_of_state.cpp:26-80
* dynamics.reconstruct.{vertical,horizontal}.{type,scale,shock}
                                           src/recon/reconstruct.cpp:13-35
* dynamics.riemann-solver.type             src/riemann/riemann_solver.cpp:10-28
* dynamics.disable-flux-x{1,2,3}           src/hydro/hydro_options.cpp:42-49
* integration.{type,cfl,implicit-scheme,nlim,tlim}
                                           src/implicit/implicit_hydro.cpp:20-32
* forcing.const-gravity.*                  src/forcing/const_gravity.cpp:10-24
* forcing.diffusion.{nu_iso,kappa_iso}     src/forcing/diffusion.cpp:115-128
* boundary-condition.external.*            src/mesh/meshblock_options.cpp:86-170
* scalar.{nvar,names,reconstruct}          src/scalar/scalar_options.cpp:9-60

Unsupported options raise ``ValueError`` instead of being ignored.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

RECON = {"dc": 0, "plm": 1, "cp3": 2, "cp5": 3, "weno3": 4, "weno5": 5}
RIEMANN = {"roe": 0, "lmars": 1, "hllc": 2, "upwind": 3}
BC = {"custom": 0, "reflecting": 1, "periodic": 2, "outflow": 3}
PRIMITIVE, CONSERVED, SCALAR = 0, 1, 2

# kintera's universal gas constant, J/(mol K); R = RGAS / weight
RGAS = 8.31446261815324


class HydroConfig(ctypes.Structure):
    _fields_ = [
        ("nx1", ctypes.c_int32), ("nx2", ctypes.c_int32), ("nx3", ctypes.c_int32),
        ("nghost", ctypes.c_int32), ("nvar", ctypes.c_int32), ("nscalar", ctypes.c_int32),
        ("x1min", ctypes.c_double), ("x1max", ctypes.c_double),
        ("x2min", ctypes.c_double), ("x2max", ctypes.c_double),
        ("x3min", ctypes.c_double), ("x3max", ctypes.c_double),
        ("gammad", ctypes.c_double), ("rgas", ctypes.c_double),
        ("recon1_type", ctypes.c_int32), ("recon1_shock", ctypes.c_int32),
        ("recon1_scale", ctypes.c_int32),
        ("recon23_type", ctypes.c_int32), ("recon23_shock", ctypes.c_int32),
        ("recon23_scale", ctypes.c_int32),
        ("scalar_recon_type", ctypes.c_int32), ("scalar_recon_scale", ctypes.c_int32),
        ("riemann", ctypes.c_int32), ("implicit_scheme", ctypes.c_int32),
        ("grav1", ctypes.c_double), ("grav2", ctypes.c_double), ("grav3", ctypes.c_double),
        ("non_hydrostatic", ctypes.c_double),
        ("nu_iso", ctypes.c_double), ("kappa_iso", ctypes.c_double),
        ("bc", ctypes.c_int32 * 6), ("disable_flux", ctypes.c_int32 * 3),
        ("reserved", ctypes.c_int32),
    ]

    # -- convenience ------------------------------------------------------
    @property
    def nc1(self):
        return self.nx1 + 2 * self.nghost if self.nx1 > 1 else 1

    @property
    def nc2(self):
        return self.nx2 + 2 * self.nghost if self.nx2 > 1 else 1

    @property
    def nc3(self):
        return self.nx3 + 2 * self.nghost if self.nx3 > 1 else 1

    @property
    def shape(self):
        return (self.nvar, self.nc3, self.nc2, self.nc1)

    @property
    def scalar_shape(self):
        return (self.nscalar, self.nc3, self.nc2, self.nc1)

    def interior(self):
        """Index tuple of the interior cells (without the variable axis)."""
        g = self.nghost
        sl = []
        for nx in (self.nx3, self.nx2, self.nx1):
            sl.append(slice(g, g + nx) if nx > 1 else slice(0, 1))
        return tuple(sl)

    def copy(self):
        c = HydroConfig()
        ctypes.memmove(ctypes.byref(c), ctypes.byref(self), ctypes.sizeof(HydroConfig))
        return c


def make_config(nx1=1, nx2=1, nx3=1, nghost=3, x1=(0.0, 1.0), x2=(0.0, 1.0), x3=(0.0, 1.0),
                gammad=1.4, rgas=None, weight=29.0e-3, recon1="weno5", recon23="weno5",
                shock1=False, shock23=False, scale1=False, scale23=False, riemann="hllc",
                implicit_scheme=0, grav=(0.0, 0.0, 0.0), non_hydrostatic=1.0, nu_iso=0.0,
                kappa_iso=0.0, bc=("reflecting",) * 6, nscalar=0, scalar_recon="dc",
                scalar_scale=False, disable_flux=(False, False, False)) -> HydroConfig:
    """Build a HydroConfig from keyword arguments (names follow the YAML keys)."""
    c = HydroConfig()
    c.nx1, c.nx2, c.nx3, c.nghost = nx1, nx2, nx3, nghost
    c.nvar, c.nscalar = 5, nscalar
    c.x1min, c.x1max = x1
    c.x2min, c.x2max = x2
    c.x3min, c.x3max = x3
    c.gammad = gammad
    c.rgas = rgas if rgas is not None else RGAS / weight
    c.recon1_type, c.recon1_shock, c.recon1_scale = RECON[recon1], int(shock1), int(scale1)
    c.recon23_type, c.recon23_shock, c.recon23_scale = RECON[recon23], int(shock23), int(scale23)
    c.scalar_recon_type, c.scalar_recon_scale = RECON[scalar_recon], int(scalar_scale)
    if riemann not in ("roe", "lmars", "hllc"):
        raise ValueError(f"unsupported hydro riemann solver {riemann!r}")
    c.riemann = RIEMANN[riemann]
    if implicit_scheme not in (0, 1, 9):
        raise ValueError(f"unsupported implicit scheme {implicit_scheme}")
    c.implicit_scheme = implicit_scheme
    c.grav1, c.grav2, c.grav3 = grav
    c.non_hydrostatic = non_hydrostatic
    c.nu_iso, c.kappa_iso = nu_iso, kappa_iso
    for i, b in enumerate(bc):
        c.bc[i] = BC[b]
    for i, d in enumerate(disable_flux):
        c.disable_flux[i] = int(d)
    validate(c)
    return c


def validate(c: HydroConfig):
    for nx in (c.nx1, c.nx2, c.nx3):
        if nx > 1 and nx < c.nghost:
            raise ValueError("number of grids must be greater than the ghost zone size")
    need = {0: 1, 1: 2, 2: 2, 3: 3, 4: 2, 5: 3}
    for t in (c.recon1_type, c.recon23_type):
        if need[t] > c.nghost:
            raise ValueError("reconstruction stencil wider than the ghost zone")
    if c.implicit_scheme and c.nx1 <= 1:
        raise ValueError("the implicit scheme needs an active x1 axis")
    if c.implicit_scheme and c.grav1 == 0.0 and c.grav2 == 0.0 and c.grav3 == 0.0 \
            and c.non_hydrostatic == 1.0:
        # the reference requires a const-gravity section for the implicit solve
        pass
    if c.nu_iso < 0 or c.kappa_iso < 0:
        raise ValueError("diffusion coefficients must be non-negative")
    if not (0.0 <= c.non_hydrostatic <= 1.0):
        raise ValueError("non-hydrostatic must lie in [0, 1]")


@dataclass
class Integration:
    """integration.* keys (harp's Integrator options)."""
    type: str = "rk3"
    cfl: float = 0.9
    nlim: int = -1
    tlim: float = 1.0e9
    max_redo: int = 5


@dataclass
class LayoutOptions:
    """distribute.* keys (LayoutOptionsImpl::from_yaml,
    src/layout/layout.cpp:165-185); the periodic flags follow the external
    boundary types of x2 / x3 (src/mesh/meshblock_options.cpp:132-146)."""
    type: str = "slab"
    px: int = 1  # nb2
    py: int = 1  # nb3
    pz: int = 1  # nb1
    periodic_x: bool = False
    periodic_y: bool = False


@dataclass
class MeshBlockOptions:
    hydro: HydroConfig
    integration: Integration = field(default_factory=Integration)
    scalar_names: list = field(default_factory=list)
    layout: LayoutOptions = field(default_factory=LayoutOptions)

    @staticmethod
    def from_yaml(path_or_dict) -> "MeshBlockOptions":
        import yaml

        if isinstance(path_or_dict, dict):
            cfg = path_or_dict
        else:
            with open(path_or_dict) as f:
                cfg = yaml.safe_load(f)
        return _from_dict(cfg)


def _get(d, *keys, default=None):
    for k in keys:
        if not isinstance(d, dict) or k not in d or d[k] is None:
            return default
        d = d[k]
    return d


def config_dict(c) -> dict:
    """A HydroConfig as the plain dict the C++ host module's constructors take
    (every field of snapb_hydro_config; bc and disable_flux as lists)."""
    d = {f: getattr(c, f) for f, _ in c._fields_ if f not in ("bc", "disable_flux", "reserved")}
    d["bc"] = list(c.bc)
    d["disable_flux"] = list(c.disable_flux)
    return d


def _from_dict(cfg: dict) -> MeshBlockOptions:
    geo = cfg.get("geometry", {}) or {}
    if geo.get("type", "cartesian") != "cartesian":
        raise ValueError("only cartesian geometry is on this path")
    b = geo.get("bounds", {}) or {}
    cells = geo.get("cells", {}) or {}
    dyn = cfg.get("dynamics", {}) or {}
    eos = dyn.get("equation-of-state", {}) or {}
    etype = eos.get("type", "moist-mixture")
    if etype != "ideal-gas":
        raise ValueError(f"equation of state {etype!r} is not on this path (ideal-gas only)")
    if eos.get("limiter", False):
        raise ValueError("the EOS limiter is not supported on this path")
    rec = dyn.get("reconstruct", {}) or {}
    vert = rec.get("vertical") or {}
    hor = rec.get("horizontal") or {}
    rs = _get(dyn, "riemann-solver", "type", default="roe")
    integ = cfg.get("integration", {}) or {}
    forcing = cfg.get("forcing", {}) or {}
    grav = forcing.get("const-gravity")
    diff = forcing.get("diffusion") or {}
    ext = _get(cfg, "boundary-condition", "external", default={}) or {}
    nx1 = int(cells.get("nx1", 1))
    nx2 = int(cells.get("nx2", 1))
    nx3 = int(cells.get("nx3", 1))
    bcs = []
    for ax, nx in ((1, nx1), (2, nx2), (3, nx3)):
        for side in ("inner", "outer"):
            bcs.append(ext.get(f"x{ax}-{side}", "reflecting") if nx > 1 else "reflecting")
    sc = cfg.get("scalar", {}) or {}
    names = list(sc.get("names", []) or [])
    nscalar = len(names) if names else int(sc.get("nvar", 0))
    srec = sc.get("reconstruct") or {}
    disable = [bool(dyn.get(f"disable-flux-x{i}", False)) for i in (1, 2, 3)]
    g = [0.0, 0.0, 0.0]
    nh = 1.0
    if grav is not None:
        g = [float(grav.get("grav1", 0.0)), float(grav.get("grav2", 0.0)),
             float(grav.get("grav3", 0.0))]
        nh = float(grav.get("non-hydrostatic", 1.0))
        for i in range(3):
            if disable[i]:
                g[i] = 0.0
    scheme = int(integ.get("implicit-scheme", 0) or 0)
    if scheme and grav is None:
        raise ValueError("[ImplicitHydro] forcing does not have const-gravity")
    for k in forcing:
        if k not in ("const-gravity", "diffusion"):
            raise ValueError(f"forcing {k!r} is not on this path")
    hc = make_config(
        nx1=nx1, nx2=nx2, nx3=nx3, nghost=int(cells.get("nghost", 1)),
        x1=(float(b.get("x1min", 0.0)), float(b.get("x1max", 1.0))),
        x2=(float(b.get("x2min", 0.0)), float(b.get("x2max", 1.0))),
        x3=(float(b.get("x3min", 0.0)), float(b.get("x3max", 1.0))),
        gammad=float(eos.get("gammad", 1.4)), weight=float(eos.get("weight", 29.0e-3)),
        recon1=vert.get("type", "dc"), recon23=hor.get("type", "dc"),
        shock1=bool(vert.get("shock", False)), shock23=bool(hor.get("shock", False)),
        scale1=bool(vert.get("scale", False)), scale23=bool(hor.get("scale", False)),
        riemann=rs, implicit_scheme=scheme, grav=tuple(g), non_hydrostatic=nh,
        nu_iso=float(diff.get("nu_iso", 0.0)), kappa_iso=float(diff.get("kappa_iso", 0.0)),
        bc=tuple(bcs), nscalar=nscalar, scalar_recon=srec.get("type", "dc"),
        scalar_scale=bool(srec.get("scale", False)), disable_flux=tuple(disable))
    it = Integration(type=integ.get("type", "rk3"), cfl=float(integ.get("cfl", 0.9)),
                     nlim=int(integ.get("nlim", -1)), tlim=float(integ.get("tlim", 1.0e9)))
    if it.type != "rk3":
        raise ValueError(f"integrator {it.type!r} is not on this path (rk3 only)")
    dist = cfg.get("distribute", {}) or {}
    lay = LayoutOptions(type=str(dist.get("layout", "slab")), px=int(dist.get("nb2", 1)),
                        py=int(dist.get("nb3", 1)), pz=int(dist.get("nb1", 1)),
                        periodic_x="periodic" in bcs[2:4], periodic_y="periodic" in bcs[4:6])
    return MeshBlockOptions(hydro=hc, integration=it, scalar_names=names, layout=lay)

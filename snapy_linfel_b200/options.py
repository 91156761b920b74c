"""The snapy options classes of the hydro path, with the reference's chained
accessors: ``op.name()`` reads an option and ``op.name(value)`` sets it and
returns the options object, so settings chain
(``ReconstructOptions().shock(True).interp(InterpOptions("weno5"))``).

Mirrors the pybind surface of the reference (``ADD_OPTION`` in
python/csrc/pyoptions.hpp) for the classes on this path, with the reference's
defaults and YAML readers:

* InterpOptions            python/csrc/pyrecon.cpp:12-26, src/recon/interpolation.hpp:30-31
* ReconstructOptions       python/csrc/pyrecon.cpp:28-41, src/recon/reconstruct.cpp:13-35
* RiemannSolverOptions     python/csrc/pyriemann.cpp:12-24, src/riemann/riemann_solver.hpp:33-36
* ImplicitOptions          python/csrc/pyimplicit.cpp:16-33, src/implicit/implicit_hydro.cpp:20-48
* EquationOfStateOptions   python/csrc/pyeos.cpp:18-40, src/eos/equation_of_state.hpp:41-53
* ConstGravityOptions, DiffusionOptions
                           src/forcing/forcing.hpp:46-49, 174-175
* CoordinateOptions        src/coord/coordinate.cpp:58-166 (geometry.* keys)
* HydroOptions             python/csrc/pyhydro.cpp:16-46, src/hydro/hydro_options.cpp:14-80

``HydroOptions.config(coord, ...)`` turns the options and a geometry into the
``snapb_hydro_config`` that the C ABI and the module classes
(snapy_linfel_b200.modules) take.  Options this path does not implement
(moist thermodynamics, Coriolis and the other forcings, the EOS limiter) can
be read but raise ValueError when a configuration is built from them.
"""
from __future__ import annotations

import copy

_UNSET = object()


class _Options:
    """Base of the option classes: subclasses list (name, default) pairs in
    _FIELDS; each becomes a chained accessor method."""

    _FIELDS: tuple = ()
    _NAME = "Options"

    def __init__(self, **kw):
        for name, default in self._FIELDS:
            setattr(self, "_" + name, copy.deepcopy(default))
        for k, v in kw.items():
            getattr(self, k)(v)

    def __init_subclass__(cls, **kw):
        super().__init_subclass__(**kw)
        for name, _ in cls._FIELDS:
            if name in cls.__dict__:
                continue

            def accessor(self, value=_UNSET, _n=name):
                if value is _UNSET:
                    return getattr(self, "_" + _n)
                setattr(self, "_" + _n, value)
                return self

            accessor.__name__ = name
            accessor.__doc__ = f"get {name}() / set {name}(value) -> self"
            setattr(cls, name, accessor)

    def report(self) -> str:
        lines = []
        for name, _ in self._FIELDS:
            v = getattr(self, "_" + name)
            if isinstance(v, _Options):
                v = "\n  ".join(v.report().splitlines())
                lines.append(f"* {name} =\n  {v}")
            else:
                lines.append(f"* {name} = {v!r}")
        return "\n".join(lines)

    def __repr__(self):
        return f"{self._NAME}(\n{self.report()})"

    def __eq__(self, other):
        return type(self) is type(other) and all(
            getattr(self, "_" + n) == getattr(other, "_" + n) for n, _ in self._FIELDS)


def _load(filename):
    import yaml

    if isinstance(filename, dict):
        return filename
    with open(filename) as f:
        return yaml.safe_load(f) or {}


class InterpOptions(_Options):
    _NAME = "InterpOptions"
    _FIELDS = (("type", "dc"), ("scale", False))

    def __init__(self, type=None, **kw):
        super().__init__(**kw)
        if type is not None:
            self._type = type


class ReconstructOptions(_Options):
    _NAME = "ReconstructOptions"
    _FIELDS = (("shock", True), ("interp", None))

    @staticmethod
    def from_yaml(filename, section: str) -> "ReconstructOptions":
        """dynamics.reconstruct.<section> (section: 'vertical' or 'horizontal')"""
        cfg = _load(filename)
        op = ReconstructOptions()
        node = ((cfg.get("dynamics") or {}).get("reconstruct") or {}).get(section)
        if not node:
            return op
        op.shock(bool(node.get("shock", False)))
        op.interp(InterpOptions(str(node.get("type", "dc"))).scale(bool(node.get("scale", False))))
        return op


class RiemannSolverOptions(_Options):
    _NAME = "RiemannSolverOptions"
    _FIELDS = (("type", "hllc"), ("dir", "omni"))

    @staticmethod
    def from_yaml(filename, section: str = "dynamics") -> "RiemannSolverOptions":
        cfg = _load(filename)
        op = RiemannSolverOptions()
        node = (cfg.get(section) or {}).get("riemann-solver") or {}
        op.type(str(node.get("type", "roe")))
        return op


class ImplicitOptions(_Options):
    _NAME = "ImplicitOptions"
    _FIELDS = (("scheme", 0),)
    _TYPES = {0: "none", 1: "vic-partial", 9: "vic-full"}

    def type(self) -> str:
        """'none' (0), 'vic-partial' (1: the 3x3 blocks of rho, v1, p) or
        'vic-full' (9: 5x5 blocks)"""
        if self._scheme not in self._TYPES:
            raise ValueError("Unsupported implicit scheme")
        return self._TYPES[self._scheme]

    @staticmethod
    def from_yaml(filename, verbose: bool = False):
        """integration.implicit-scheme; None when the key is absent"""
        cfg = _load(filename)
        node = cfg.get("integration") or {}
        if "implicit-scheme" not in node or node["implicit-scheme"] is None:
            return None
        return ImplicitOptions().scheme(int(node["implicit-scheme"]))


class EquationOfStateOptions(_Options):
    _NAME = "EquationOfStateOptions"
    _FIELDS = (("type", "moist-mixture"), ("gammad", 1.4), ("weight", 29.0e-3),
               ("density_floor", 1.0e-10), ("pressure_floor", 1.0e-10),
               ("temperature_floor", 20.0), ("limiter", False), ("eos_file", ""),
               ("verbose", False))

    @staticmethod
    def from_yaml(filename, verbose: bool = False) -> "EquationOfStateOptions":
        cfg = _load(filename)
        node = (cfg.get("dynamics") or {}).get("equation-of-state") or {}
        op = EquationOfStateOptions()
        op.type(str(node.get("type", "moist-mixture")))
        for key, name in (("gammad", "gammad"), ("weight", "weight"),
                          ("density-floor", "density_floor"),
                          ("pressure-floor", "pressure_floor"),
                          ("temperature-floor", "temperature_floor")):
            if key in node:
                getattr(op, name)(float(node[key]))
        op.limiter(bool(node.get("limiter", False)))
        op.eos_file(str(node.get("eos-file", "")))
        op.verbose(bool(verbose))
        return op


class ConstGravityOptions(_Options):
    _NAME = "ConstGravityOptions"
    _FIELDS = (("grav1", 0.0), ("grav2", 0.0), ("grav3", 0.0), ("non_hydrostatic", 1.0))

    @staticmethod
    def from_yaml(forcing: dict):
        node = (forcing or {}).get("const-gravity")
        if node is None:
            return None
        return ConstGravityOptions(
            grav1=float(node.get("grav1", 0.0)), grav2=float(node.get("grav2", 0.0)),
            grav3=float(node.get("grav3", 0.0)),
            non_hydrostatic=float(node.get("non-hydrostatic", 1.0)))


class DiffusionOptions(_Options):
    _NAME = "DiffusionOptions"
    _FIELDS = (("nu_iso", 0.0), ("kappa_iso", 0.0))

    @staticmethod
    def from_yaml(forcing: dict):
        node = (forcing or {}).get("diffusion")
        if node is None:
            return None
        return DiffusionOptions(nu_iso=float(node.get("nu_iso", 0.0)),
                                kappa_iso=float(node.get("kappa_iso", 0.0)))


class CoordinateOptions(_Options):
    """geometry.{type, bounds, cells} of the mesh block"""
    _NAME = "CoordinateOptions"
    _FIELDS = (("type", "cartesian"), ("x1min", 0.0), ("x1max", 1.0), ("x2min", 0.0),
               ("x2max", 1.0), ("x3min", 0.0), ("x3max", 1.0), ("nx1", 1), ("nx2", 1),
               ("nx3", 1), ("nghost", 1))

    @staticmethod
    def from_yaml(filename) -> "CoordinateOptions":
        cfg = _load(filename)
        geo = cfg.get("geometry") or {}
        b = geo.get("bounds") or {}
        cells = geo.get("cells") or {}
        op = CoordinateOptions().type(str(geo.get("type", "cartesian")))
        for k in ("x1min", "x1max", "x2min", "x2max", "x3min", "x3max"):
            if k in b:
                getattr(op, k)(float(b[k]))
        for k in ("nx1", "nx2", "nx3", "nghost"):
            if k in cells:
                getattr(op, k)(int(cells[k]))
        return op


class HydroOptions(_Options):
    _NAME = "HydroOptions"
    _FIELDS = (("verbose", False), ("disable_flux_x1", False), ("disable_flux_x2", False),
               ("disable_flux_x3", False), ("grav", None), ("coriolis", None),
               ("diffusion", None), ("eos", None), ("recon1", None), ("recon23", None),
               ("riemann", None), ("icorr", None))

    @staticmethod
    def from_yaml(filename, verbose: bool = False) -> "HydroOptions":
        """the reference's HydroOptionsImpl::from_yaml: EOS, the vertical and
        horizontal reconstructions, the Riemann solver, the implicit
        correction, disable-flux flags, and the const-gravity / diffusion
        forcings (gravity zeroed along disabled axes)"""
        cfg = _load(filename)
        op = HydroOptions()
        op.eos(EquationOfStateOptions.from_yaml(cfg, verbose))
        op.recon1(ReconstructOptions.from_yaml(cfg, "vertical"))
        op.recon23(ReconstructOptions.from_yaml(cfg, "horizontal"))
        op.riemann(RiemannSolverOptions.from_yaml(cfg, "dynamics"))
        op.icorr(ImplicitOptions.from_yaml(cfg))
        dyn = cfg.get("dynamics")
        if dyn:
            op.verbose(bool(dyn.get("verbose", verbose)))
            for i in (1, 2, 3):
                getattr(op, f"disable_flux_x{i}")(bool(dyn.get(f"disable-flux-x{i}", False)))
        forcing = cfg.get("forcing")
        if not forcing:
            return op
        grav = ConstGravityOptions.from_yaml(forcing)
        if grav is not None:
            for i in (1, 2, 3):
                if getattr(op, f"disable_flux_x{i}")():
                    getattr(grav, f"grav{i}")(0.0)
        op.grav(grav)
        if forcing.get("coriolis") is not None:
            op.coriolis(dict(forcing["coriolis"]))
        op.diffusion(DiffusionOptions.from_yaml(forcing))
        return op

    def config(self, coord: CoordinateOptions, bc=("reflecting",) * 6, nscalar: int = 0,
               scalar_recon: InterpOptions | None = None):
        """the snapb_hydro_config of these options on a geometry"""
        from .config import RGAS, make_config

        if coord.type() != "cartesian":
            raise ValueError("only cartesian geometry is on this path")
        eos = self.eos() or EquationOfStateOptions()
        if eos.type() != "ideal-gas":
            raise ValueError(f"equation of state {eos.type()!r} is not on this path "
                             "(ideal-gas only)")
        if eos.limiter():
            raise ValueError("the EOS limiter is not supported on this path")
        if self.coriolis() is not None:
            raise ValueError("forcing 'coriolis' is not on this path")
        r1 = self.recon1() or ReconstructOptions()
        r23 = self.recon23() or ReconstructOptions()
        i1 = r1.interp() or InterpOptions()
        i23 = r23.interp() or InterpOptions()
        g = self.grav()
        d = self.diffusion()
        ic = self.icorr()
        scheme = ic.scheme() if ic is not None else 0
        if scheme and g is None:
            raise ValueError("[ImplicitHydro] forcing does not have const-gravity")
        sr = scalar_recon or InterpOptions()
        return make_config(
            nx1=coord.nx1(), nx2=coord.nx2(), nx3=coord.nx3(), nghost=coord.nghost(),
            x1=(coord.x1min(), coord.x1max()), x2=(coord.x2min(), coord.x2max()),
            x3=(coord.x3min(), coord.x3max()), gammad=eos.gammad(),
            rgas=RGAS / eos.weight(), recon1=i1.type(), recon23=i23.type(),
            shock1=r1.shock(), shock23=r23.shock(), scale1=i1.scale(), scale23=i23.scale(),
            riemann=(self.riemann() or RiemannSolverOptions()).type(), implicit_scheme=scheme,
            grav=(g.grav1(), g.grav2(), g.grav3()) if g is not None else (0.0, 0.0, 0.0),
            non_hydrostatic=g.non_hydrostatic() if g is not None else 1.0,
            nu_iso=d.nu_iso() if d is not None else 0.0,
            kappa_iso=d.kappa_iso() if d is not None else 0.0, bc=tuple(bc), nscalar=nscalar,
            scalar_recon=sr.type(), scalar_scale=sr.scale(),
            disable_flux=(self.disable_flux_x1(), self.disable_flux_x2(),
                          self.disable_flux_x3()))


__all__ = ["InterpOptions", "ReconstructOptions", "RiemannSolverOptions", "ImplicitOptions",
           "EquationOfStateOptions", "ConstGravityOptions", "DiffusionOptions",
           "CoordinateOptions", "HydroOptions"]

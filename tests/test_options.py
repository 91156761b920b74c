"""The snapy options classes with chained accessors (python/csrc/pyhydro.cpp,
pyrecon.cpp, pyriemann.cpp, pyimplicit.cpp, pyeos.cpp): defaults, chaining,
from_yaml, and the configuration they build against the YAML loader."""
import pytest

from snapy_linfel_b200.config import RECON, RIEMANN, MeshBlockOptions
from snapy_linfel_b200.options import (ConstGravityOptions, CoordinateOptions,
                                       DiffusionOptions, EquationOfStateOptions,
                                       HydroOptions, ImplicitOptions, InterpOptions,
                                       ReconstructOptions, RiemannSolverOptions)

STRAKA_LIKE = """
geometry:
  type: cartesian
  bounds: {x1min: 0., x1max: 6400., x2min: 0., x2max: 25600., x3min: -0.5, x3max: 0.5}
  cells: {nx1: 32, nx2: 128, nx3: 1, nghost: 3}
dynamics:
  equation-of-state: {type: ideal-gas, gammad: 1.4, weight: 0.02896}
  reconstruct:
    vertical: {type: weno5, scale: false, shock: false}
    horizontal: {type: weno5, scale: false, shock: false}
  riemann-solver: {type: lmars}
boundary-condition:
  external: {x1-inner: reflecting, x1-outer: reflecting, x2-inner: reflecting,
             x2-outer: reflecting}
forcing:
  const-gravity: {grav1: -9.8}
  diffusion: {nu_iso: 75., kappa_iso: 75.}
integration: {type: rk3, cfl: 0.9, implicit-scheme: 1, tlim: 900}
"""


def test_defaults_match_the_reference():
    assert InterpOptions().type() == "dc" and InterpOptions().scale() is False
    assert ReconstructOptions().shock() is True and ReconstructOptions().interp() is None
    assert RiemannSolverOptions().type() == "hllc" and RiemannSolverOptions().dir() == "omni"
    assert ImplicitOptions().scheme() == 0 and ImplicitOptions().type() == "none"
    e = EquationOfStateOptions()
    assert (e.type(), e.gammad(), e.weight(), e.density_floor(), e.temperature_floor(),
            e.limiter()) == ("moist-mixture", 1.4, 29.0e-3, 1.0e-10, 20.0, False)
    g = ConstGravityOptions()
    assert (g.grav1(), g.grav2(), g.grav3(), g.non_hydrostatic()) == (0.0, 0.0, 0.0, 1.0)
    h = HydroOptions()
    assert h.verbose() is False and h.grav() is None and h.icorr() is None


def test_setters_chain_and_return_the_object():
    r = ReconstructOptions().shock(False).interp(InterpOptions("weno5").scale(True))
    assert isinstance(r, ReconstructOptions)
    assert (r.shock(), r.interp().type(), r.interp().scale()) == (False, "weno5", True)
    assert ImplicitOptions().scheme(9).type() == "vic-full"
    with pytest.raises(ValueError):
        ImplicitOptions().scheme(3).type()
    h = HydroOptions().disable_flux_x2(True).riemann(RiemannSolverOptions().type("roe"))
    assert h.disable_flux_x2() is True and h.riemann().type() == "roe"
    assert "riemann" in repr(h) and "HydroOptions(" in repr(h)


def test_from_yaml_and_config_match_the_loader(tmp_path):
    p = tmp_path / "straka_like.yaml"
    p.write_text(STRAKA_LIKE)
    h = HydroOptions.from_yaml(str(p))
    assert h.eos().type() == "ideal-gas" and h.eos().weight() == pytest.approx(0.02896)
    assert h.recon1().interp().type() == "weno5" and h.recon1().shock() is False
    assert h.riemann().type() == "lmars" and h.icorr().scheme() == 1
    assert h.grav().grav1() == -9.8 and h.diffusion().nu_iso() == 75.0
    coord = CoordinateOptions.from_yaml(str(p))
    assert (coord.nx1(), coord.nx2(), coord.nghost(), coord.x2max()) == (32, 128, 3, 25600.0)
    c = h.config(coord)
    want = MeshBlockOptions.from_yaml(str(p)).hydro
    for f, _ in type(c)._fields_:
        if f in ("bc", "disable_flux"):
            assert list(getattr(c, f)) == list(getattr(want, f)), f
        else:
            assert getattr(c, f) == getattr(want, f), f
    assert c.recon1_type == RECON["weno5"] and c.riemann == RIEMANN["lmars"]


def test_disabled_axis_zeroes_gravity_and_unsupported_options_raise(tmp_path):
    text = STRAKA_LIKE.replace("riemann-solver: {type: lmars}",
                               "riemann-solver: {type: lmars}\n  disable-flux-x1: true")
    p = tmp_path / "d.yaml"
    p.write_text(text)
    h = HydroOptions.from_yaml(str(p))
    assert h.disable_flux_x1() is True and h.grav().grav1() == 0.0
    with pytest.raises(ValueError):
        HydroOptions().eos(EquationOfStateOptions()).config(CoordinateOptions(nx1=8, nghost=3))
    with pytest.raises(ValueError):
        (HydroOptions().eos(EquationOfStateOptions().type("ideal-gas").limiter(True))
         .config(CoordinateOptions(nx1=8, nghost=3)))
    assert DiffusionOptions.from_yaml({}) is None


def test_modules_take_options_with_a_parent_block():
    from snapy_linfel_b200 import modules
    from snapy_linfel_b200.config import make_config

    try:
        modules._lib.lib()
    except modules._lib.SnapbError:
        pytest.skip("libsnapb.so not built")
    blk = make_config(nx1=12, nx2=8, recon1="plm", recon23="plm", riemann="hllc")
    rec = modules.Reconstruct(ReconstructOptions().shock(True).interp(InterpOptions("weno5")),
                              blk)
    assert rec.cfg.recon1_type == RECON["weno5"] and rec.cfg.recon23_shock == 1
    assert rec.cfg.nx1 == 12
    rs = modules.RiemannSolver(RiemannSolverOptions().type("roe"), blk)
    assert rs.solver == RIEMANN["roe"]
    with pytest.raises(TypeError):
        modules.Reconstruct(ReconstructOptions())
    h = (HydroOptions().eos(EquationOfStateOptions().type("ideal-gas"))
         .recon1(ReconstructOptions().interp(InterpOptions("weno5")))
         .recon23(ReconstructOptions().interp(InterpOptions("weno5")))
         .riemann(RiemannSolverOptions().type("lmars")))
    hyd = modules.Hydro(h, blk)
    assert hyd.cfg.riemann == RIEMANN["lmars"] and hyd.cfg.nx2 == 8

"""CPU checks of the drop-in boundary: the C-ABI library loads and exports
every entry point include/snapb.h declares; the ctypes config struct has the
C layout; host-side argument validation rejects bad input without a GPU."""
import ctypes
import os
import re
import subprocess

import pytest

from snapy_linfel_b200 import _lib
from snapy_linfel_b200.config import HydroConfig, MeshBlockOptions, make_config

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "snapb.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(snapb_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "snapb_stage" in names and "snapb_hydro_forward" in names
    assert set(_lib.exported_symbols()) <= set(names)


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True).stdout
    for n in declared_functions():
        assert re.search(rf"\bT {n}\b", out), n


def test_abi_version():
    assert _lib.lib().snapb_abi_version() == 1


def test_config_struct_layout_matches_c():
    # offsets computed by the C compiler from the header
    src = f"""
#include <stdio.h>
#include <stddef.h>
#include "{HEADER}"
int main() {{
  printf("%zu %zu %zu %zu %zu %zu\\n", sizeof(snapb_hydro_config),
         offsetof(snapb_hydro_config, x1min), offsetof(snapb_hydro_config, recon1_type),
         offsetof(snapb_hydro_config, grav1), offsetof(snapb_hydro_config, bc),
         offsetof(snapb_hydro_config, reserved));
  return 0;
}}"""
    d = os.path.join(REPO, "_work")
    os.makedirs(d, exist_ok=True)
    c_path = os.path.join(d, "layout.c")
    exe = os.path.join(d, "layout")
    open(c_path, "w").write(src)
    subprocess.run(["gcc", c_path, "-o", exe], check=True)
    vals = list(map(int, subprocess.run([exe], capture_output=True, text=True).stdout.split()))
    py = [ctypes.sizeof(HydroConfig), HydroConfig.x1min.offset, HydroConfig.recon1_type.offset,
          HydroConfig.grav1.offset, HydroConfig.bc.offset, HydroConfig.reserved.offset]
    assert vals == py


def test_workspace_size_and_validation():
    lib = _lib.lib()
    c = make_config(nx1=64, nx2=32, implicit_scheme=1, grav=(-9.8, 0, 0))
    assert lib.snapb_workspace_size(ctypes.byref(c)) > 0
    bad = c.copy()
    bad.nghost = 2
    assert lib.snapb_workspace_size(ctypes.byref(bad)) == 0
    # entry points reject bad configs before touching the device
    rc = lib.snapb_stage(ctypes.byref(bad), 0, None, None, None, None, None, None, None, None, 0,
                         None)
    assert rc == 1
    assert b"nghost" in lib.snapb_last_error()
    rc = lib.snapb_stage(ctypes.byref(c), 0, ctypes.c_void_p(8), ctypes.c_void_p(8),
                         ctypes.c_void_p(8), ctypes.c_void_p(8), None, None, None,
                         ctypes.c_void_p(8), 16, None)
    assert rc == 4  # workspace too small
    rc = lib.snapb_riemann(ctypes.byref(c), 3, 3, ctypes.c_void_p(8), ctypes.c_void_p(8), 1,
                           ctypes.c_void_p(8), ctypes.c_void_p(8), ctypes.c_void_p(8), None)
    assert rc == 1 and b"not implemented" in lib.snapb_last_error()


YAML_SMALL = """
dynamics:
  equation-of-state: {type: ideal-gas, gammad: 1.4, density-floor: 1.e-10,
                      pressure-floor: 1.e-10, limiter: false}
  reconstruct:
    vertical: {type: weno5, scale: false, shock: false}
    horizontal: {type: weno5, scale: false, shock: false}
  riemann-solver: {type: lmars}
geometry:
  type: cartesian
  bounds: {x1min: 0., x1max: 1., x2min: 0., x2max: 1., x3min: 0., x3max: 1.}
  cells: {nx1: 10, nx2: 8, nx3: 6, nghost: 3}
boundary-condition:
  external: {x1-inner: reflecting, x1-outer: reflecting, x2-inner: periodic,
             x2-outer: periodic, x3-inner: outflow, x3-outer: outflow}
integration: {type: rk3, cfl: 0.8, implicit-scheme: 9}
forcing:
  const-gravity: {grav1: -9.8}
"""


def test_yaml_options(tmp_path):
    p = tmp_path / "block.yaml"
    p.write_text(YAML_SMALL)
    o = MeshBlockOptions.from_yaml(str(p))
    c = o.hydro
    assert (c.nx1, c.nx2, c.nx3, c.nghost) == (10, 8, 6, 3)
    assert c.shape == (5, 12, 14, 16)
    assert c.recon1_type == 5 and c.recon1_shock == 0
    assert c.riemann == 1 and c.implicit_scheme == 9
    assert list(c.bc) == [1, 1, 2, 2, 3, 3]
    assert c.grav1 == -9.8 and o.integration.cfl == 0.8


def test_yaml_rejects_unsupported(tmp_path):
    p = tmp_path / "bad.yaml"
    p.write_text(YAML_SMALL.replace("ideal-gas", "moist-mixture"))
    with pytest.raises(ValueError):
        MeshBlockOptions.from_yaml(str(p))
    p.write_text(YAML_SMALL.replace("implicit-scheme: 9", "implicit-scheme: 5"))
    with pytest.raises(ValueError):
        MeshBlockOptions.from_yaml(str(p))
    # implicit solve without const-gravity is an error, as in the reference
    txt = YAML_SMALL.replace("forcing:\n  const-gravity: {grav1: -9.8}\n", "")
    p.write_text(txt)
    with pytest.raises(ValueError):
        MeshBlockOptions.from_yaml(str(p))


def test_implicit_scheme_bits():
    # scheme 1 -> 3x3 partial blocks, 9 -> 5x5 full blocks
    for s, n in ((1, 3), (9, 5)):
        assert (5 if (s >> 3) & 1 else 3) == n


def test_ensemble_structs_match_c():
    from snapy_linfel_b200.ensemble import MemberF32, Tuning

    src = f"""
#include <stdio.h>
#include <stddef.h>
#include "{HEADER}"
int main() {{
  printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(snapb_member_f32),
         offsetof(snapb_member_f32, u), offsetof(snapb_member_f32, workspace),
         offsetof(snapb_member_f32, workspace_bytes), sizeof(snapb_ensemble_tuning),
         offsetof(snapb_ensemble_tuning, vic_regs), offsetof(snapb_ensemble_tuning, vic_kernel));
  return 0;
}}"""
    d = os.path.join(REPO, "_work")
    os.makedirs(d, exist_ok=True)
    c_path = os.path.join(d, "layout_ens.c")
    exe = os.path.join(d, "layout_ens")
    open(c_path, "w").write(src)
    subprocess.run(["gcc", c_path, "-o", exe], check=True)
    vals = list(map(int, subprocess.run([exe], capture_output=True, text=True).stdout.split()))
    py = [ctypes.sizeof(MemberF32), MemberF32.u.offset, MemberF32.workspace.offset,
          MemberF32.workspace_bytes.offset, ctypes.sizeof(Tuning), Tuning.vic_regs.offset,
          Tuning.vic_kernel.offset]
    assert vals == py


def test_module_surface_rejects_cpu_tensors():
    """the module classes have no CPU path: CPU tensors are refused before any
    device call"""
    torch = pytest.importorskip("torch")
    from snapy_linfel_b200 import _lib
    from snapy_linfel_b200.modules import (EquationOfState, Hydro, ImplicitHydro, Reconstruct,
                                           RiemannSolver)

    c = make_config(nx1=8, nx2=6)
    x = torch.zeros(c.shape, dtype=torch.float64)
    with pytest.raises(_lib.SnapbError):
        EquationOfState(c).compute("U->W", [x])
    with pytest.raises(_lib.SnapbError):
        Hydro(c).forward(0.1, x)
    with pytest.raises(_lib.SnapbError):
        Reconstruct(c).forward(x, 3)
    with pytest.raises(_lib.SnapbError):
        RiemannSolver(c, "hllc").forward(x, x, 3, x)
    with pytest.raises(_lib.SnapbError):
        ImplicitHydro(c).forward(x, x, 0.1)
    with pytest.raises(KeyError):
        RiemannSolver(c, "exact")

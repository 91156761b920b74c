"""The hand-written reverse-mode gradients of the implicit solve's bilinear
forms (csrc/bilinear_adj.cuh: y^T |A|(wl, wr) x and y^T J(w) x, used by the
adjoint's block-dependence contraction) against central differences of the
block formulas in long double, on the host: tests/cpp/bilinear_adj_check.cpp,
built here with the host C++ compiler."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def test_bilinear_form_gradients_match_central_differences(tmp_path):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    exe = tmp_path / "bilinear_adj_check"
    src = os.path.join(HERE, "cpp", "bilinear_adj_check.cpp")
    subprocess.run([cxx, "-O2", "-std=c++17", src, "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    assert out[0] == "worst"
    w3, w5 = float(out[1]), float(out[2])
    # long-double differences with step 1e-4 (velocities) / 1e-6 relative:
    # truncation and rounding stay below 1e-5 of the gradient
    assert w3 < 1e-5 and w5 < 1e-5, (w3, w5)

"""Build the C++ host extension ``_snapb_host`` (libtorch + pybind11) in-tree.

It links against the in-tree ``libsnapb.so`` (rpath $ORIGIN) and torch's
libraries; g++ only (the CUDA code lives in libsnapb.so).
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc", "host", "meshblock.cpp")
OUT = os.path.join(HERE, "_snapb_host" + sysconfig.get_config_var("EXT_SUFFIX"))


def build(force: bool = False) -> str:
    from torch.utils import cpp_extension

    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) > os.path.getmtime(SRC):
        return OUT
    inc = cpp_extension.include_paths() + [sysconfig.get_paths()["include"],
                                           "/usr/local/cuda/include"]
    libdirs = cpp_extension.library_paths()
    cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden", SRC, "-o", OUT,
           "-DTORCH_EXTENSION_NAME=_snapb_host", "-DTORCH_API_INCLUDE_EXTENSION_H",
           "-D_GLIBCXX_USE_CXX11_ABI=1"]
    cmd += [f"-I{d}" for d in inc] + [f"-L{d}" for d in libdirs]
    cmd += [f"-L{HERE}", "-lsnapb", "-Wl,-rpath,$ORIGIN"]
    cmd += [f"-Wl,-rpath,{d}" for d in libdirs]
    cmd += ["-lc10", "-lc10_cuda", "-ltorch", "-ltorch_cpu", "-ltorch_cuda", "-ltorch_python"]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="-f" in sys.argv))

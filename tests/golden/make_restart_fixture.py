"""Generate tests/golden/ref_restart.block0.00003.part with the reference's
own restart writer.

The reference writes a block's restart variables as a TorchScript archive of
buffers with ``save_tensors`` (python/write_init.py:12-22; the C++ path
kintera::save_tensors writes the same archive for RestartOutput,
src/output/restart.cpp:24-88).  python/write_init.py imports netCDF4 and
kintera at module level, neither of which is installed here, so this script
takes the ``save_tensors`` function out of the file's syntax tree and runs it
unchanged.  The tensors are seeded, so the fixture is reproducible.

Run in a container that has the reference sources:

    SNAPB_REFERENCE=<reference checkout> python tests/golden/make_restart_fixture.py
"""
import ast
import os
import sys

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "ref_restart.block0.00003.part")


def reference_save_tensors(ref_root):
    path = os.path.join(ref_root, "python", "write_init.py")
    with open(path) as f:
        tree = ast.parse(f.read(), filename=path)
    fn = next(n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == "save_tensors")
    mod = ast.Module(body=[fn], type_ignores=[])
    scope = {"torch": torch}
    exec(compile(mod, path, "exec"), scope)
    return scope["save_tensors"]


def fixture_tensors():
    """the variables RestartOutput stores for a block with two scalars
    (scalar_r left out: it is derived from scalar_s and hydro_u)"""
    g = torch.Generator().manual_seed(31)
    shape = (4, 6, 14)  # nc3, nc2, nc1
    u = torch.rand((5,) + shape, generator=g, dtype=torch.float64) + 0.5
    w = torch.rand((5,) + shape, generator=g, dtype=torch.float64) + 0.5
    s = torch.rand((2,) + shape, generator=g, dtype=torch.float64)
    return {"hydro_u": u, "hydro_w": w, "scalar_s": s,
            "last_time": torch.tensor([123.25], dtype=torch.float64),
            "last_cycle": torch.tensor([77], dtype=torch.int64),
            "file_number": torch.tensor([3, 12], dtype=torch.int64),
            "next_time": torch.tensor([130.0, 200.0], dtype=torch.float64)}


def main():
    ref = os.environ.get("SNAPB_REFERENCE",
                         os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(HERE))),
                                      "reference"))
    if not os.path.isfile(os.path.join(ref, "python", "write_init.py")):
        sys.exit(f"reference sources not found at {ref}")
    save = reference_save_tensors(ref)
    save(fixture_tensors(), OUT)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()

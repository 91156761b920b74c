"""Restart files in the reference's format, so a run can resume from (or hand
over to) the reference's restarts.

* One block's file, ``<basename>.block<rank>.<NNNNN>.part`` (or ``.final.part``):
  a TorchScript module archive whose buffers are the block's variables, moved
  to the CPU, with ``scalar_r`` left out when ``scalar_s`` and ``hydro_u`` are
  there, plus ``last_time`` (float64 [1]), ``last_cycle`` (int64 [1]),
  ``file_number`` (int64 [n]) and ``next_time`` (float64 [n]) of the output
  types (RestartOutput::write_output_file, src/output/restart.cpp:24-88; the
  archive is what kintera::save_tensors / the reference's
  python/write_init.py:12-22 write and src/input/read_restart_file.cpp reads).
* The combined file ``<basename>.<NNNNN>.restart``: the single part renamed, or
  a bundle of all parts — the line ``SNAPY_RESTART_BUNDLE_V1``, the part count,
  one ``<file name>\\t<byte size>`` line per part, an empty line, then the
  parts' bytes back to back (make_restart_bundle,
  src/output/combine_restart.cpp:35-73); the parts are removed after bundling.
* Reading: a bundle's entry for block ``<rank>`` (part name
  ``<basename>.block<rank>.<number>.part``) or a single archive
  (load_restart, src/input/read_restart_file.cpp:154-234).
"""
from __future__ import annotations

import glob
import os
import tempfile
import warnings

BUNDLE_MAGIC = "SNAPY_RESTART_BUNDLE_V1"


def _tensor_module_class():
    import torch

    class TensorModule(torch.nn.Module):
        def __init__(self, tensors):
            super().__init__()
            for name, tensor in tensors.items():
                self.register_buffer(name, tensor)

    return TensorModule


_TensorModule = None


def save_tensors(tensors: dict, path: str):
    """named tensors -> one TorchScript archive of buffers"""
    import torch

    global _TensorModule
    if _TensorModule is None:
        _TensorModule = _tensor_module_class()
    m = _TensorModule({k: v.detach().cpu().contiguous() for k, v in tensors.items()})
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")  # TorchScript is deprecated but is the format
        torch.jit.script(m).save(path)


def load_tensors(path: str) -> dict:
    import torch

    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        m = torch.jit.load(path, map_location="cpu")
    out = {k: v for k, v in m.named_buffers(recurse=False)}
    out.update({k: v for k, v in m.named_parameters(recurse=False)})
    return out


def part_name(basename: str, rank: int, file_number: int, final: bool = False) -> str:
    return f"{basename}.block{rank}.{'final' if final else f'{file_number:05d}'}.part"


def parse_part_name(name: str):
    """(basename, rank, file number string) of a part file name"""
    if not name.endswith(".part") or len(name) <= 5:
        raise ValueError("filename does not end with .part")
    core = name[:-5]
    d2 = core.rfind(".")
    if d2 < 0:
        raise ValueError("filename missing filenumber field")
    d1 = core.rfind(".", 0, d2)
    if d1 < 0:
        raise ValueError("filename missing block_id field")
    blockid = core[d1 + 1:d2]
    if not blockid.startswith("block"):
        raise ValueError("block id must read block<rank>")
    return core[:d1], int(blockid[5:]), core[d2 + 1:]


def write_part(variables: dict, output_dir: str, basename: str, rank: int, file_number: int,
               current_time: float, cycle: int, final: bool = False,
               output_file_numbers=(), output_next_times=()) -> str:
    """one block's restart part; variables: name -> tensor (any device)"""
    import torch

    out = {}
    skip_r = "scalar_s" in variables and "hydro_u" in variables
    for name, var in variables.items():
        if var is None or (skip_r and name == "scalar_r"):
            continue
        out[name] = var.detach().to("cpu")
    out["last_time"] = torch.tensor([float(current_time)], dtype=torch.float64)
    out["last_cycle"] = torch.tensor([int(cycle)], dtype=torch.int64)
    out["file_number"] = torch.tensor(list(output_file_numbers), dtype=torch.int64)
    out["next_time"] = torch.tensor(list(output_next_times), dtype=torch.float64)
    os.makedirs(output_dir, exist_ok=True)
    path = os.path.join(output_dir, part_name(basename, rank, file_number, final))
    save_tensors(out, path)
    return path


def make_bundle(bundle_path: str, files):
    """concatenate part files under the bundle header"""
    sizes = [os.path.getsize(f) for f in files]
    with open(bundle_path, "wb") as out:
        out.write(f"{BUNDLE_MAGIC}\n{len(files)}\n".encode())
        for f, n in zip(files, sizes):
            out.write(f"{os.path.basename(f)}\t{n}\n".encode())
        out.write(b"\n")
        for f in files:
            with open(f, "rb") as src:
                while True:
                    chunk = src.read(1 << 20)
                    if not chunk:
                        break
                    out.write(chunk)


def combine(output_dir: str, basename: str, file_number: int, final: bool = False) -> str:
    """the parts of one output number -> <basename>.<NNNNN>.restart"""
    tag = "final" if final else f"{file_number:05d}"
    files = sorted(glob.glob(os.path.join(output_dir, f"{basename}.block*.{tag}.part")))
    if not files:
        raise FileNotFoundError(f"no restart parts {basename}.block*.{tag}.part in {output_dir}")
    out = os.path.join(output_dir, f"{basename}.{tag}.restart")
    if os.path.exists(out):
        os.remove(out)
    if len(files) == 1:
        os.rename(files[0], out)
    else:
        make_bundle(out, files)
        for f in files:
            os.remove(f)
    return out


def _read_bundle_index(f):
    if f.readline().decode().rstrip("\n") != BUNDLE_MAGIC:
        raise ValueError("restart bundle missing expected magic header")
    line = f.readline().decode().rstrip("\n")
    if not line:
        raise ValueError("restart bundle missing entry count")
    entries = []
    for _ in range(int(line)):
        line = f.readline().decode().rstrip("\n")
        if "\t" not in line:
            raise ValueError("restart bundle index line missing tab")
        name, size = line.split("\t", 1)
        entries.append([name, int(size)])
    if f.readline().decode().rstrip("\n"):
        raise ValueError("restart bundle header missing terminator")
    off = f.tell()
    for e in entries:
        e.append(off)
        off += e[1]
    return entries


def is_bundle(path: str) -> bool:
    with open(path, "rb") as f:
        return f.readline().decode(errors="replace").rstrip("\n") == BUNDLE_MAGIC


def load_restart(path: str, block_rank: int = 0) -> dict:
    """the variables of block `block_rank` from a bundle, or of a single part"""
    if not is_bundle(path):
        return load_tensors(path)
    with open(path, "rb") as f:
        for name, size, off in _read_bundle_index(f):
            if not name.endswith(".part"):
                continue
            if parse_part_name(name)[1] != block_rank:
                continue
            f.seek(off)
            data = f.read(size)
            fd, tmp = tempfile.mkstemp(suffix=".part")
            try:
                with os.fdopen(fd, "wb") as t:
                    t.write(data)
                return load_tensors(tmp)
            finally:
                os.remove(tmp)
    raise KeyError(f"{path}: no block {block_rank} in the restart bundle")

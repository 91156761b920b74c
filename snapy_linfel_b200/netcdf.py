"""NetCDF output of a mesh block in the reference's data model.

NetcdfOutput::write_output_file (src/output/netcdf.cpp:34-508) writes, per
block and output, ``<basename>.block<rank>.<file_id>.<NNNNN>.nc`` with

* dimensions ``time`` (unlimited), ``x1``, ``x2``, ``x3`` (interior cells)
  and ``x1f``, ``x2f``, ``x3f`` (faces, on active axes);
* coordinate variables of those names (float) with ``axis`` (T, Z, X, Y),
  ``units`` and ``long_name`` attributes and ``domain_decomposition`` = [1,
  global cells, first, last] of the block along the axis (faces: [0, ...,
  first - 1, last]);
* the global attribute ``NumFilesInSet`` (blocks in the run);
* the output variables as float [time, x1, x3, x2] with ``units`` and
  ``long_name`` from the metadata table (src/output/output_utils.cpp:28-70):
  ``prim`` -> rho, press, vel1, vel2, vel3; ``cons`` -> dens, Etot, mom1,
  mom2, mom3 (src/output/load_hydro_output_data.cpp:72-145); single
  velocity components with ``v1``/``vx`` etc.; the block's scalars as s1,
  s2, ... when they are passed.

The reference links the netCDF library and creates NetCDF-4 (HDF5) files;
neither library is in this image, so the file is written here in the
NetCDF-3 64-bit-offset format (the published classic file format), which
carries the same dimensions, variables and attributes and is read by the
same tools (netCDF4-python, xarray, ncdump, scipy.io.netcdf_file).
"""
from __future__ import annotations

import os
import struct

import numpy as np

# NetCDF-3 header tags and external types
_ABSENT = b"\x00" * 8
_NC_DIMENSION, _NC_VARIABLE, _NC_ATTRIBUTE = 0x0A, 0x0B, 0x0C
_NC_CHAR, _NC_INT, _NC_FLOAT = 2, 4, 5

# short name -> (long name, units), from the reference's metadata table
METADATA = {
    "rho": ("density", "kg/m^3"),
    "press": ("pressure", "pa"),
    "vel1": ("vertical velocity", "m/s"),
    "vel2": ("horizontal velocity", "m/s"),
    "vel3": ("horizontal velocity", "m/s"),
}


def _pad4(b: bytes) -> bytes:
    return b + b"\x00" * (-len(b) % 4)


def _name(s: str) -> bytes:
    e = s.encode()
    return struct.pack(">i", len(e)) + _pad4(e)


def _attr(name: str, value) -> bytes:
    if isinstance(value, str):
        e = value.encode()
        return _name(name) + struct.pack(">ii", _NC_CHAR, len(e)) + _pad4(e)
    arr = np.atleast_1d(np.asarray(value))
    if arr.dtype.kind in "iu":
        return _name(name) + struct.pack(">ii", _NC_INT, arr.size) + arr.astype(">i4").tobytes()
    return _name(name) + struct.pack(">ii", _NC_FLOAT, arr.size) + arr.astype(">f4").tobytes()


def _attr_list(attrs: dict) -> bytes:
    if not attrs:
        return _ABSENT
    return struct.pack(">ii", _NC_ATTRIBUTE, len(attrs)) + b"".join(
        _attr(k, v) for k, v in attrs.items())


def write_classic(path: str, dims: list, variables: list, gattrs: dict):
    """Write a NetCDF-3 64-bit-offset file of float variables.

    dims: [(name, size)], size None for the unlimited dimension; variables:
    [(name, [dim names], {attrs}, data)], data in the row-major order of the
    dims; one record along the unlimited dimension (the reference writes one
    time level per file)."""
    dim_index = {n: k for k, (n, _) in enumerate(dims)}
    unlimited = {n for n, size in dims if size is None}
    dim_bytes = struct.pack(">ii", _NC_DIMENSION, len(dims)) + b"".join(
        _name(n) + struct.pack(">i", 0 if size is None else size) for n, size in dims)
    is_rec = [bool(vd) and vd[0] in unlimited for _, vd, _, _ in variables]
    vsizes = []
    for _, _, _, data in variables:
        n = int(np.asarray(data).size) * 4
        vsizes.append(n + (-n % 4))

    def var_list(begins):
        out = struct.pack(">ii", _NC_VARIABLE, len(variables))
        for (name, vd, attrs, _), vs, beg in zip(variables, vsizes, begins):
            out += _name(name) + struct.pack(">i", len(vd))
            out += b"".join(struct.pack(">i", dim_index[d]) for d in vd)
            out += _attr_list(attrs) + struct.pack(">ii", _NC_FLOAT, vs) + struct.pack(">q", beg)
        return out

    head = b"CDF\x02" + struct.pack(">i", 1 if unlimited else 0) + dim_bytes + \
        _attr_list(gattrs)
    off = len(head) + len(var_list([0] * len(variables)))
    begins = [0] * len(variables)
    order = [k for k in range(len(variables)) if not is_rec[k]] + \
            [k for k in range(len(variables)) if is_rec[k]]  # fixed data, then the record
    for k in order:
        begins[k] = off
        off += vsizes[k]
    with open(path, "wb") as f:
        f.write(head + var_list(begins))
        for k in order:
            data = np.ascontiguousarray(np.asarray(variables[k][3], dtype=">f4")).tobytes()
            f.write(_pad4(data))


def output_name(basename: str, rank: int, file_id: str, file_number: int) -> str:
    return f"{basename}.block{rank}.{file_id}.{file_number:05d}.nc"


def _host(a):
    if a is None:
        return None
    if hasattr(a, "detach"):
        a = a.detach().cpu().numpy()
    return np.asarray(a)


def write_block(cfg, hydro_w, hydro_u, output_dir: str, basename: str, file_number: int,
                current_time: float, file_id: str = "out1", variables=("prim",), rank: int = 0,
                block_loc=(0, 0, 0), blocks=(1, 1, 1), scalars=None) -> str:
    """One block's output file.  hydro_w / hydro_u: [nvar, nc3, nc2, nc1]
    arrays (numpy or tensors, ghosts included; either may be None when the
    selected variables do not need it); block_loc / blocks: the block's
    (lx1, lx2, lx3) and the block counts (nb1, nb2, nb3); scalars: the
    scalar array to write as s1, s2, ...  Returns the file's path."""
    w, u, s = _host(hydro_w), _host(hydro_u), _host(scalars)
    it = cfg.interior()
    n1, n2, n3 = cfg.nx1, cfg.nx2, cfg.nx3
    lx1, lx2, lx3 = block_loc
    nb1, nb2, nb3 = blocks

    dims = [("time", None)]
    for ax, n in ((1, n1), (2, n2), (3, n3)):
        dims.append((f"x{ax}", n))
        if n > 1:
            dims.append((f"x{ax}f", n + 1))
    out = [("time", ["time"], {"axis": "T", "units": "s", "long_name": "time"},
            np.array([current_time], dtype=np.float32))]
    for ax, n, lx, nb, axis, cname, fname in (
            (1, n1, lx1, nb1, "Z", "Z-coordinate at cell center", "Z-coordinate at cell face"),
            (2, n2, lx2, nb2, "X", "X-coordinate at cell center", "Y-coordinate at cell face"),
            (3, n3, lx3, nb3, "Y", "Y-coordinate at cell center", "X-coordinate at cell face")):
        lo, hi = getattr(cfg, f"x{ax}min"), getattr(cfg, f"x{ax}max")
        pos = np.array([1, n * nb, n * lx + 1, n * (lx + 1)], dtype=np.int32)
        centres = lo + (np.arange(n) + 0.5) * (hi - lo) / n
        out.append((f"x{ax}", [f"x{ax}"], {"axis": axis, "units": "m", "long_name": cname,
                                          "domain_decomposition": pos}, centres))
        if n > 1:
            posf = pos.copy()
            posf[0] -= 1
            posf[2] -= 1
            faces = lo + np.arange(n + 1) * (hi - lo) / n
            out.append((f"x{ax}f", [f"x{ax}f"], {"units": "m", "long_name": fname,
                                                 "domain_decomposition": posf}, faces))

    def add(name, a, v):
        if a is None:
            raise ValueError(f"output variable {name!r} needs its state array")
        lu = METADATA.get(name)
        attrs = {"units": lu[1], "long_name": lu[0]} if lu else {}
        data = np.transpose(a[v][it], (2, 0, 1))[None].astype(np.float32)  # [time, x1, x3, x2]
        out.append((name, ["time", "x1", "x3", "x2"], attrs, data))

    for sel in variables:
        if sel == "prim":
            add("rho", w, 0)
            add("press", w, 4)
            for v in (1, 2, 3):
                add(f"vel{v}", w, v)
        elif sel == "cons":
            add("dens", u, 0)
            add("Etot", u, 4)
            for v in (1, 2, 3):
                add(f"mom{v}", u, v)
        elif sel in ("v1", "vx", "v2", "vy", "v3", "vz"):
            v = {"v1": 1, "vx": 1, "v2": 2, "vy": 2, "v3": 3, "vz": 3}[sel]
            add(f"vel{v}", w, v)
        else:
            raise ValueError(f"output variable {sel!r} is not on this path")
    if s is not None:
        for n in range(s.shape[0]):
            add(f"s{n + 1}", s, n)
    os.makedirs(output_dir, exist_ok=True)
    path = os.path.join(output_dir, output_name(basename, rank, file_id, file_number))
    write_classic(path, dims, out, {"NumFilesInSet": np.int32(nb1 * nb2 * nb3)})
    return path

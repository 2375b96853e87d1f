"""Minimal netCDF-3 classic (CDF-1 / CDF-2 64-bit offset) writer and reader.

SFINCS reads its subgrid tables (``sbgfile``) and quadtree meshes (``qtrfile``)
through netcdf-fortran (``sfincs_subgrid.F90:94-122``, ``sfincs_quadtree.F90:310-438``).
No netCDF library exists in this image, so synthetic inputs are written in the
classic format from the public Unidata file-format specification: big-endian
header (magic, numrecs, dimension list, global attributes, variable list with
per-variable ``begin`` offsets) followed by the fixed-size variable data.  Only
fixed-size (non-record) variables are supported, which is all these files use.

Dimension order follows the netCDF (C) convention: a Fortran array
``tab(nlevels, np)`` is stored as a netCDF variable with dims ``("np", "levels")``.
"""
from __future__ import annotations

import struct
from typing import Dict, Iterable, Tuple

import numpy as np

NC_BYTE, NC_CHAR, NC_SHORT, NC_INT, NC_FLOAT, NC_DOUBLE = 1, 2, 3, 4, 5, 6
_NC_DIMENSION, _NC_VARIABLE, _NC_ATTRIBUTE = 0x0A, 0x0B, 0x0C

_NP2NC = {
    np.dtype("int8"): NC_BYTE,
    np.dtype("int16"): NC_SHORT,
    np.dtype("int32"): NC_INT,
    np.dtype("float32"): NC_FLOAT,
    np.dtype("float64"): NC_DOUBLE,
}
_NC2NP = {NC_BYTE: ">i1", NC_CHAR: "S1", NC_SHORT: ">i2", NC_INT: ">i4",
          NC_FLOAT: ">f4", NC_DOUBLE: ">f8"}
_NCSIZE = {NC_BYTE: 1, NC_CHAR: 1, NC_SHORT: 2, NC_INT: 4, NC_FLOAT: 4, NC_DOUBLE: 8}


def _pad4(n: int) -> int:
    return (n + 3) & ~3


def _name(s: str) -> bytes:
    b = s.encode()
    return struct.pack(">i", len(b)) + b + b"\0" * (_pad4(len(b)) - len(b))


def _attr_bytes(name: str, value) -> bytes:
    if isinstance(value, str):
        vb = value.encode()
        return _name(name) + struct.pack(">ii", NC_CHAR, len(vb)) + vb + b"\0" * (_pad4(len(vb)) - len(vb))
    arr = np.atleast_1d(np.asarray(value))
    if arr.dtype.kind == "f":
        arr = arr.astype(np.float32) if arr.dtype == np.float32 else arr.astype(np.float64)
    elif arr.dtype.kind in "iu":
        arr = arr.astype(np.int32)
    t = _NP2NC[arr.dtype]
    raw = arr.astype(_NC2NP[t]).tobytes()
    return _name(name) + struct.pack(">ii", t, arr.size) + raw + b"\0" * (_pad4(len(raw)) - len(raw))


def write(path: str, dims: Dict[str, int], variables: Dict[str, Tuple[Tuple[str, ...], np.ndarray]],
          gattrs: Dict[str, object] | None = None) -> None:
    """Write a CDF-2 (64-bit offset) file with fixed-size variables.

    ``variables`` maps name -> (dimension names, array); arrays are cast to the
    nearest netCDF type (int8/int16/int32/float32/float64) and written big-endian.
    """
    dim_names = list(dims)
    dim_index = {d: i for i, d in enumerate(dim_names)}
    gattrs = gattrs or {}
    arrays = {}
    for vname, (vdims, arr) in variables.items():
        arr = np.ascontiguousarray(arr)
        if arr.dtype not in _NP2NC:
            if arr.dtype.kind == "f":
                arr = arr.astype(np.float32)
            elif arr.dtype.kind in "iub":
                arr = arr.astype(np.int32)
        shape = tuple(dims[d] for d in vdims)
        if arr.shape != shape:
            raise ValueError(f"variable {vname}: shape {arr.shape} != dims {shape}")
        arrays[vname] = (vdims, arr)

    def header(begins: Iterable[int]) -> bytes:
        h = b"CDF\x02" + struct.pack(">i", 0)
        h += struct.pack(">ii", _NC_DIMENSION, len(dim_names)) if dim_names else struct.pack(">ii", 0, 0)
        for d in dim_names:
            h += _name(d) + struct.pack(">i", dims[d])
        if gattrs:
            h += struct.pack(">ii", _NC_ATTRIBUTE, len(gattrs))
            for k, v in gattrs.items():
                h += _attr_bytes(k, v)
        else:
            h += struct.pack(">ii", 0, 0)
        h += struct.pack(">ii", _NC_VARIABLE, len(arrays)) if arrays else struct.pack(">ii", 0, 0)
        for (vname, (vdims, arr)), begin in zip(arrays.items(), begins):
            t = _NP2NC[arr.dtype]
            vsize = _pad4(arr.size * _NCSIZE[t])
            h += _name(vname) + struct.pack(">i", len(vdims))
            for d in vdims:
                h += struct.pack(">i", dim_index[d])
            h += struct.pack(">ii", 0, 0)  # no variable attributes
            h += struct.pack(">ii", t, min(vsize, 0xFFFFFFFF)) + struct.pack(">q", begin)
        return h

    hlen = len(header([0] * len(arrays)))
    begins, off = [], hlen
    for vdims, arr in arrays.values():
        begins.append(off)
        off += _pad4(arr.size * arr.dtype.itemsize)
    with open(path, "wb") as f:
        f.write(header(begins))
        for vdims, arr in arrays.values():
            t = _NP2NC[arr.dtype]
            raw = arr.astype(_NC2NP[t], copy=False)
            raw.tofile(f)
            pad = _pad4(arr.nbytes) - arr.nbytes
            if pad:
                f.write(b"\0" * pad)


def read(path: str) -> Tuple[Dict[str, int], Dict[str, np.ndarray], Dict[str, object]]:
    """Read a CDF-1/CDF-2 file written with fixed-size variables (test helper)."""
    with open(path, "rb") as f:
        buf = f.read()
    if buf[:3] != b"CDF" or buf[3] not in (1, 2):
        raise ValueError("not a netCDF-3 classic file")
    off64 = buf[3] == 2
    pos = 8

    def i32():
        nonlocal pos
        v = struct.unpack_from(">i", buf, pos)[0]
        pos += 4
        return v

    def name():
        nonlocal pos
        n = i32()
        s = buf[pos:pos + n].decode()
        pos += _pad4(n)
        return s

    def attrs():
        nonlocal pos
        tag, n = i32(), i32()
        out = {}
        for _ in range(n if tag else 0):
            k = name()
            t, cnt = i32(), i32()
            raw = buf[pos:pos + cnt * _NCSIZE[t]]
            pos += _pad4(cnt * _NCSIZE[t])
            out[k] = raw.decode() if t == NC_CHAR else np.frombuffer(raw, _NC2NP[t]).astype(_NC2NP[t][1:])
        return out

    tag, nd = i32(), i32()
    dims, dlist = {}, []
    for _ in range(nd if tag else 0):
        d = name()
        dims[d] = i32()
        dlist.append(d)
    gat = attrs()
    tag, nv = i32(), i32()
    out = {}
    for _ in range(nv if tag else 0):
        vname = name()
        ndims = i32()
        ids = [i32() for _ in range(ndims)]
        attrs()
        t = i32()
        i32()  # vsize
        if off64:
            begin = struct.unpack_from(">q", buf, pos)[0]
            pos += 8
        else:
            begin = i32()
        shape = tuple(dims[dlist[i]] for i in ids)
        cnt = int(np.prod(shape)) if shape else 1
        out[vname] = np.frombuffer(buf, _NC2NP[t], count=cnt, offset=begin).reshape(shape).astype(_NC2NP[t][1:])
    return dims, out, gat

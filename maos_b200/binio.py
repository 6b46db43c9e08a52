"""maos ``.bin`` files: read and write dense arrays and cells.

The format (``sys/bin.h:34-58``, ``sys/bin.c`` ``write_header`` /
``read_bin_header``, ``math/cell.c`` ``writebin``): little-endian; each
array is an optional header-string block, then the magic ``M_SKIP``, the
type magic (uint32) and ``nx``, ``ny`` (uint64), then ``nx*ny`` elements
column-major (x fastest).  A header-string block is ``M_HEADER``, the
string length rounded up to 8 bytes (uint64), the NUL-terminated string
padded with zeros, the length again and ``M_HEADER`` again.  A cell is the
magic ``MCC_ANY`` with its ``nx``, ``ny`` followed by its elements, each a
whole array (an empty element is written as an empty ``0 x 0`` cell).  Files whose
name ends in ``.gz``, or that start with the gzip signature, are gzipped.

Arrays come back as numpy arrays of shape ``(nx, ny)`` in Fortran order
(so ``a[ix, iy]`` is maos' ``p[ix + nx*iy]``), cells as numpy object arrays
of shape ``(nx, ny)`` whose empty elements are ``None``.  Sparse matrices
and FITS files are not handled.  Used to exchange golden vectors with the
reference (``tests/test_binio.py`` checks it against the reference's own
writer and reader).
"""
from __future__ import annotations

import gzip
import struct
from typing import Optional, Tuple

import numpy as np

M_DBL = 0x6402
M_INT64 = 0x6403
M_CMP = 0x6404
M_INT32 = 0x6405
M_FLT = 0x6408
M_ZMP = 0x6409
M_INT8 = 0x640A
M_INT16 = 0x640B
MCC_ANY = 0x6421
M_HEADER = 0x6500
M_SKIP = 0x6600

_DTYPE = {M_DBL: np.dtype("<f8"), M_FLT: np.dtype("<f4"), M_CMP: np.dtype("<c16"), M_ZMP: np.dtype("<c8"),
          M_INT64: np.dtype("<i8"), M_INT32: np.dtype("<i4"), M_INT16: np.dtype("<i2"), M_INT8: np.dtype("<i1")}
_MAGIC = {np.dtype(v).newbyteorder("="): k for k, v in _DTYPE.items()}


def _open(path: str, mode: str):
    if mode == "rb":
        with open(path, "rb") as f:
            gz = f.read(2) == b"\x1f\x8b"
        return gzip.open(path, "rb") if gz else open(path, "rb")
    return gzip.open(path, "wb") if path.endswith(".gz") else open(path, "wb")


def _read_exact(f, n: int) -> bytes:
    b = f.read(n)
    if len(b) != n:
        raise EOFError("truncated .bin file")
    return b


def _read_one(f) -> Tuple[object, str]:
    hdr = []
    while True:
        raw = f.read(4)
        if len(raw) < 4:
            raise EOFError("no array in .bin file")
        magic = struct.unpack("<I", raw)[0]
        if (magic & M_SKIP) == M_SKIP:
            continue
        if magic == M_HEADER:
            n = struct.unpack("<Q", _read_exact(f, 8))[0]
            s = _read_exact(f, n)
            n2, m2 = struct.unpack("<QI", _read_exact(f, 12))
            if n2 != n or m2 != M_HEADER:
                raise ValueError("corrupt header string block")
            hdr.append(s.split(b"\0", 1)[0].decode("utf-8", "replace"))
            continue
        nx, ny = struct.unpack("<QQ", _read_exact(f, 16))
        header = "".join(hdr)
        if magic == MCC_ANY:
            if nx == 0 or ny == 0:
                return None, header  # the writer's form of an empty element
            out = np.empty((nx, ny), dtype=object)
            for iy in range(ny):
                for ix in range(nx):
                    out[ix, iy] = _read_one(f)[0]
            return out, header
        if magic not in _DTYPE:
            raise ValueError(f"unsupported .bin magic 0x{magic:x}")
        if nx == 0 or ny == 0:
            return None, header
        dt = _DTYPE[magic]
        data = np.frombuffer(_read_exact(f, dt.itemsize * nx * ny), dtype=dt)
        return data.astype(dt.newbyteorder("="), copy=True).reshape((nx, ny), order="F"), header


def read(path: str, header: bool = False):
    """The array or cell in ``path`` (and its header string when ``header``)."""
    with _open(path, "rb") as f:
        out, h = _read_one(f)
    return (out, h) if header else out


def _write_header(f, text: Optional[str]):
    if not text:
        return
    s = text.encode("utf-8") + b"\0"
    n = (len(s) + 7) // 8 * 8
    f.write(struct.pack("<IQ", M_HEADER, n))
    f.write(s + b"\0" * (n - len(s)))
    f.write(struct.pack("<QI", n, M_HEADER))


def _write_one(f, obj, text: Optional[str]):
    _write_header(f, text)
    if obj is None:  # as the reference writes an empty element: an empty cell
        f.write(struct.pack("<IIQQ", M_SKIP, MCC_ANY, 0, 0))
        return
    if isinstance(obj, (list, tuple)) or (isinstance(obj, np.ndarray) and obj.dtype == object):
        cell = np.empty(len(obj), dtype=object) if isinstance(obj, (list, tuple)) else obj
        if isinstance(obj, (list, tuple)):
            for i, e in enumerate(obj):
                cell[i] = e
        if cell.ndim == 1:
            cell = cell.reshape(-1, 1)
        nx, ny = cell.shape
        f.write(struct.pack("<IIQQ", M_SKIP, MCC_ANY, nx, ny))
        for iy in range(ny):
            for ix in range(nx):
                _write_one(f, cell[ix, iy], None)
        return
    a = np.asarray(obj)
    if a.ndim == 0:
        a = a.reshape(1, 1)
    elif a.ndim == 1:
        a = a.reshape(-1, 1)
    elif a.ndim != 2:
        raise ValueError("only 1-D and 2-D arrays map to .bin arrays")
    magic = _MAGIC.get(a.dtype.newbyteorder("="))
    if magic is None:
        raise ValueError(f"no .bin type for {a.dtype}")
    nx, ny = a.shape
    f.write(struct.pack("<IIQQ", M_SKIP, magic, nx, ny))
    f.write(np.asarray(a, dtype=_DTYPE[magic]).tobytes(order="F"))


def write(path: str, obj, header: Optional[str] = None):
    """Write an array (1-D as ``n x 1``), or a cell (a list, or an object
    array; ``None`` elements are empty), with an optional header string."""
    with _open(path, "wb") as f:
        _write_one(f, obj, header)

"""MATLAB level-5 MAT-file output of fields (the reference's src/MatFile.{h,cpp}).

Same use as the reference: ``MatFile(fname)``, ``addField(name, field)``, and
series of fields grouped in a cell array with ``startCell(name, n)`` /
``addField(field, inc)`` / ``endCell()``; ``inc >= 0`` appends ``_inc`` to a
top-level name (MatFile.h:69-73).  A field is written as an
ni x nj x nk double (or single) array whose data is the interior with i
fastest -- MATLAB's column-major q(i, j, k) -- like MatFile::addField
(MatFile.h:62-168).  Fields may be dense numpy arrays of shape (nk, nj, ni) or
library fields (then a Convection handle is needed to download them).
"""
from __future__ import annotations

import struct

import numpy as np

_MI_INT8, _MI_INT32, _MI_UINT32, _MI_SINGLE, _MI_DOUBLE, _MI_MATRIX = 1, 5, 6, 7, 9, 14
_MX_CELL, _MX_DOUBLE, _MX_SINGLE = 1, 6, 7


def _pad8(n: int) -> int:
    return (n + 7) // 8 * 8


def _element(mitype: int, payload: bytes) -> bytes:
    return struct.pack("<II", mitype, len(payload)) + payload + b"\0" * (_pad8(len(payload)) - len(payload))


def _matrix(name: str, dims, cls: int, body: bytes) -> bytes:
    flags = _element(_MI_UINT32, struct.pack("<II", cls, 0))
    dim = _element(_MI_INT32, struct.pack("<" + "i" * len(dims), *dims))
    nm = _element(_MI_INT8, name.encode())
    content = flags + dim + nm + body
    return struct.pack("<II", _MI_MATRIX, len(content)) + content


def _numeric(name: str, a: np.ndarray) -> bytes:
    a = np.ascontiguousarray(a)
    if a.dtype == np.float32:
        cls, mi = _MX_SINGLE, _MI_SINGLE
    else:
        a = a.astype(np.float64, copy=False)
        cls, mi = _MX_DOUBLE, _MI_DOUBLE
    nk, nj, ni = a.shape
    return _matrix(name, (ni, nj, nk), cls, _element(mi, a.tobytes()))


class MatFile:
    def __init__(self, fname: str, conv=None):
        self.f = open(fname, "wb")
        self.conv = conv
        text = b"MATLAB 5.0 MAT-file, stencilparareal_b200 field output"
        self.f.write(text.ljust(116, b" ") + b"\0" * 8 + struct.pack("<H", 0x0100) + b"IM")
        self._cell = None

    def _dense(self, field):
        if isinstance(field, np.ndarray):
            return field
        if self.conv is None:
            raise ValueError("a Convection handle is needed to write a device field")
        return self.conv.download(field)

    def addField(self, name_or_field, field=None, inc: int = -1):
        """addField(name, field[, inc]), or addField(field[, inc]) under the name "q"
        (the reference takes the field's own name, MatFile.h:171-174; the
        reference drivers name their solution fields "q").  Inside a cell the
        field becomes the next element and the name is not used."""
        if not isinstance(name_or_field, str):  # addField(field[, inc]): inc is the 2nd argument
            name_or_field, field, inc = "q", name_or_field, (inc if field is None else field)
        if self._cell is not None:
            self._cell[1].append(_numeric("", self._dense(field)))
            return
        name = name_or_field if inc < 0 else f"{name_or_field}_{inc}"
        self.f.write(_numeric(name, self._dense(field)))

    def startCell(self, name: str, n: int):
        self._cell = (name, [], n)

    def endCell(self):
        name, items, n = self._cell
        self._cell = None
        self.f.write(_matrix(name, (1, len(items)), _MX_CELL, b"".join(items)))

    def close(self):
        if self._cell is not None:
            self.endCell()
        self.f.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

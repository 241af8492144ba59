"""The reference's offline data file format (multi-key float32 N-d arrays).

Layout (cpp/external/binary/include/binary/binary_file.hpp:159-228,
cpp/TOOL_overview.md:5-69), little-endian:
    int32 nkeys
    nkeys x { int32 len; char name[len] }          # key names
    per key, same order: { int32 ndims; int32 dims[ndims]; float32 data[prod(dims)] }
The reference writes keys in sorted (std::map) order.  Complex sample
matrices are stored as [samples, antennas, 2] (binary_load.cpp:55-113).
"""
from __future__ import annotations

import struct
from pathlib import Path
from typing import Mapping

import numpy as np


def read(path: str | Path) -> dict[str, np.ndarray]:
    data = Path(path).read_bytes()
    off = 0

    def i32():
        nonlocal off
        (v,) = struct.unpack_from("<i", data, off)
        off += 4
        return v

    n = i32()
    if n < 0:
        raise ValueError(f"{path}: bad key count")
    names = []
    for _ in range(n):
        ln = i32()
        names.append(data[off:off + ln].decode())
        off += ln
    out: dict[str, np.ndarray] = {}
    for k in names:
        nd = i32()
        dims = [i32() for _ in range(nd)]
        cnt = int(np.prod(dims)) if dims else 1
        if off + 4 * cnt > len(data):
            raise ValueError(f"{path}: file truncated")
        out[k] = np.frombuffer(data, dtype="<f4", count=cnt, offset=off).reshape(dims).copy()
        off += 4 * cnt
    return out


def write(path: str | Path, arrays: Mapping[str, np.ndarray]) -> None:
    parts = [struct.pack("<i", len(arrays))]
    keys = sorted(arrays)
    for k in keys:
        b = k.encode()
        parts.append(struct.pack("<i", len(b)) + b)
    for k in keys:
        a = np.ascontiguousarray(arrays[k], dtype="<f4")
        parts.append(struct.pack("<i", a.ndim) + struct.pack(f"<{a.ndim}i", *a.shape))
        parts.append(a.tobytes())
    Path(path).write_bytes(b"".join(parts))


def complex_matrix(arr: np.ndarray, scale: complex = 1.0, antennas: int | None = None,
                   samples: int | None = None) -> np.ndarray:
    """[samples, antennas, 2] float array -> (antennas, samples) complex64 (loadData, binary_load.cpp:55-81)."""
    s, a = arr.shape[0], arr.shape[1]
    a = antennas or a
    s = samples or s
    c = arr[:s, :a, 0].astype(np.float32) + 1j * arr[:s, :a, 1].astype(np.float32)
    return (np.complex64(scale) * c.T.astype(np.complex64)).astype(np.complex64)


def to_array(m: np.ndarray) -> np.ndarray:
    """(antennas, samples) complex -> [samples, antennas, 2] float32 (BinaryFileWriter::addData)."""
    m = np.atleast_2d(np.asarray(m, np.complex64))
    out = np.empty((m.shape[1], m.shape[0], 2), np.float32)
    out[..., 0] = m.real.T
    out[..., 1] = m.imag.T
    return out

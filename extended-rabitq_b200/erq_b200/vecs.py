"""fvecs / ivecs file IO in the layout the reference drivers read.

Each row is a little-endian uint32 column count followed by that many 4-byte
values (float32 for .fvecs, int32/uint32 for .ivecs).  The reference reads
them with ``load_vecs`` (inc/utils/IO.hpp:53-83), which takes the column count
from the first row and the row count from the file size.
"""
from __future__ import annotations

import os

import numpy as np


def write_vecs(path: str | os.PathLike, mat: np.ndarray) -> None:
    """Write a 2-D float32 or (u)int32 array as .fvecs / .ivecs."""
    mat = np.ascontiguousarray(mat)
    if mat.ndim != 2:
        raise ValueError("write_vecs expects a 2-D array")
    if mat.dtype not in (np.float32, np.int32, np.uint32):
        raise ValueError(f"unsupported dtype {mat.dtype}")
    rows, cols = mat.shape
    out = np.empty((rows, cols + 1), dtype=np.uint32)
    out[:, 0] = cols
    out[:, 1:] = mat.view(np.uint32)
    out.tofile(path)


def read_vecs(path: str | os.PathLike, dtype=np.float32) -> np.ndarray:
    """Read a .fvecs / .ivecs file (dtype float32, int32 or uint32)."""
    raw = np.fromfile(path, dtype=np.uint32)
    if raw.size == 0:
        return np.zeros((0, 0), dtype=dtype)
    cols = int(raw[0])
    if raw.size % (cols + 1) != 0:
        raise ValueError(f"{path}: size is not a whole number of rows of {cols} columns")
    rows = raw.reshape(-1, cols + 1)
    if not np.all(rows[:, 0] == cols):
        raise ValueError(f"{path}: ragged rows")
    return np.ascontiguousarray(rows[:, 1:]).view(dtype)

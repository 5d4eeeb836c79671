"""BVA layout (qafold/f65521/src/layout.rs:34-155) for building prover inputs.

Each matrix is split into at most 4x4 aligned power-of-two buckets (the last
interval doubled), buckets are sorted by size descending then (matrix, row
offset, column offset), and concatenated; `logical` is the next power of two
of max(active, 1024).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Sequence, Tuple

import numpy as np


def intervals(length: int, budget: int = 4) -> List[Tuple[int, int]]:
    sizes, rem = [], length
    while rem > 0 and len(sizes) < budget:
        s = 1 << (rem.bit_length() - 1)
        sizes.append(s)
        rem -= s
    if rem > 0:
        sizes[-1] *= 2
    out, off = [], 0
    for s in sizes:
        out.append((off, s))
        off += s
    return out


@dataclass(frozen=True)
class Bucket:
    matrix: int
    row_offset: int
    col_offset: int
    rows: int
    cols: int
    physical_rows: int
    physical_cols: int
    offset: int


def buckets(shapes) -> Tuple[List[Bucket], int, int]:
    raw = []
    for m, s in enumerate(shapes):
        rows, cols = (s.rows, s.cols) if hasattr(s, "rows") else s
        for ro, r in intervals(rows):
            for co, c in intervals(cols):
                raw.append((m, ro, co, r, c, min(r, rows - ro), min(c, cols - co)))
    raw.sort(key=lambda b: (-(b[3] * b[4]), b[0], b[1], b[2]))
    out, active = [], 0
    for b in raw:
        out.append(Bucket(*b, active))
        active += b[3] * b[4]
    logical = 1 << (max(active, 1024) - 1).bit_length()
    return out, active, logical


def encode(shapes, matrices: Sequence[np.ndarray], dtype=None) -> np.ndarray:
    """`dtype` defaults to the first matrix's (int8 weights or int16 payloads)."""
    bs, active, _ = buckets(shapes)
    if dtype is None:
        dtype = np.asarray(matrices[0]).dtype if len(matrices) else np.int8
    out = np.zeros(active, dtype=dtype)
    for b in bs:
        m = np.asarray(matrices[b.matrix])
        block = m[b.row_offset: b.row_offset + b.physical_rows, b.col_offset: b.col_offset + b.physical_cols]
        view = out[b.offset: b.offset + b.rows * b.cols].reshape(b.rows, b.cols)
        view[: b.physical_rows, : b.physical_cols] = block
    return out


def demo_matrices(shapes, dtype=np.int8) -> List[np.ndarray]:
    """The demo weights of main.rs:139-141: (entry * 73 + index * 19) truncated
    to the payload width (as u8 as i8; for 16-bit payloads as u16 as i16)."""
    mats = []
    unsigned = {np.dtype(np.int8): np.uint8, np.dtype(np.int16): np.uint16}[np.dtype(dtype)]
    mask = np.iinfo(unsigned).max
    for i, s in enumerate(shapes):
        rows, cols = (s.rows, s.cols) if hasattr(s, "rows") else s
        e = np.arange(rows * cols, dtype=np.int64)
        mats.append(((e * 73 + i * 19) & mask).astype(unsigned).view(dtype).reshape(rows, cols))
    return mats

"""The reference's dense BVA stream: a JSON description plus the raw bytes of
the `active` BVA entries, read into page-locked host memory for the
streamed (recompute-mode) commitment of weight sets larger than HBM.

The description (qafold/f65521/src/main.rs:116-153, koalabear main.rs:116-157):

    {"format": "parcomm-dense-bva-stream-description",
     "storage_dtype": "i8" | "i16",
     "shapes": [[rows, cols], ...],
     "stream_bytes": active * entry bytes,
     "layout": {"logical_entries": next_power_of_two(active)}}

The stream holds exactly `stream_bytes` bytes: int8 entries, or int16
payloads little-endian (main.rs:146-173).  A short stream, an excess byte, a
foreign format or dtype and a layout that disagrees with the shapes are
rejected with the reference's messages.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path
from typing import BinaryIO, Optional, Sequence, Tuple, Union

import numpy as np

from . import FIELD_F65521, FIELD_KOALABEAR, Config, Parameters, QfError, QF_E_ARGUMENT, Shape
from .layout import buckets

FORMAT = "parcomm-dense-bva-stream-description"
# int16 payloads are read in place as they lie in the stream (little-endian).
if sys.byteorder != "little":
    raise ImportError("parcomm_b200.stream reads little-endian streams in place; this host is big-endian")
_DTYPES = {"i8": (np.dtype(np.int8), FIELD_F65521), "i16": (np.dtype(np.int16), FIELD_KOALABEAR)}
_PIECE = 8 << 20  # bytes per read, as the reference's 8 MiB buffer


def _next_pow2(n: int) -> int:
    return 1 if n <= 1 else 1 << (n - 1).bit_length()


def describe(shapes: Sequence[Tuple[int, int]], storage_dtype: str = "i8") -> dict:
    """The description of a stream over `shapes` (what a converter writes)."""
    if storage_dtype not in _DTYPES:
        raise QfError(QF_E_ARGUMENT, f"unknown storage dtype {storage_dtype!r}")
    _, active, _ = buckets([Shape(int(r), int(c)) for r, c in shapes])
    width = np.dtype(_DTYPES[storage_dtype][0]).itemsize
    return {"format": FORMAT, "storage_dtype": storage_dtype, "shapes": [[int(r), int(c)] for r, c in shapes],
            "stream_bytes": active * width, "layout": {"logical_entries": _next_pow2(active)}}


def read_description(description: Union[str, Path, dict], storage_dtype: Optional[str] = None):
    """Parses and checks a description: returns (field, shapes, dtype, active).
    `storage_dtype` ("i8" for qafold/f65521, "i16" for qafold/koalabear)
    pins the crate the caller stands for, as each reference binary accepts
    only its own dtype."""
    d = description if isinstance(description, dict) else json.loads(Path(description).read_bytes())
    want = storage_dtype or d.get("storage_dtype")
    if d.get("format") != FORMAT or want not in _DTYPES or d.get("storage_dtype") != want:
        raise QfError(QF_E_ARGUMENT, f"requires signed-{want} stream description" if want in _DTYPES
                      else "requires signed-i8 stream description")
    dt, field = _DTYPES[want]
    try:
        shapes = [(int(r), int(c)) for r, c in d["shapes"]]
    except (KeyError, TypeError, ValueError):
        raise QfError(QF_E_ARGUMENT, "stream description shapes")
    _, active, _ = buckets([Shape(r, c) for r, c in shapes])
    layout = d.get("layout") or {}
    if d.get("stream_bytes") != active * np.dtype(dt).itemsize or layout.get("logical_entries") != _next_pow2(active):
        raise QfError(QF_E_ARGUMENT, "converter/ParComm layout mismatch")
    return field, shapes, np.dtype(dt), active


def _host_buffer(n: int, dtype, pinned: bool):
    """An `n`-entry host array; page-locked (a pinned torch tensor) when
    requested and a CUDA device is present.  Returns (numpy view, owner)."""
    if pinned:
        try:
            import torch
            if torch.cuda.is_available():
                t = torch.empty(n, dtype=torch.int8 if np.dtype(dtype).itemsize == 1 else torch.int16, pin_memory=True)
                return t.numpy(), t
        except ImportError:
            pass
    a = np.empty(n, dtype=dtype)
    return a, a


def read_stream(source: Union[str, Path, BinaryIO], n: int, dtype, pinned: bool = True):
    """Reads exactly n entries from a path ("-" is stdin) or a binary file
    object into host memory, in 8 MiB pieces; returns (array, owner).  The
    owner (a pinned tensor or the array) must outlive a streamed commitment."""
    arr, owner = _host_buffer(n, dtype, pinned)
    raw = memoryview(arr.view(np.uint8).reshape(-1))
    close = False
    if isinstance(source, (str, Path)):
        if str(source) == "-":
            f = sys.stdin.buffer
        else:
            f, close = open(source, "rb", buffering=0), True
    else:
        f = source
    try:
        got = 0
        while got < len(raw):
            k = f.readinto(raw[got: got + min(_PIECE, len(raw) - got)])
            if not k:
                raise QfError(QF_E_ARGUMENT, "truncated BVA input")
            got += k
        if f.read(1):
            raise QfError(QF_E_ARGUMENT, "excess BVA input")
    finally:
        if close:
            f.close()
    return arr, owner


def write_stream(description_path: Union[str, Path], stream_path: Union[str, Path],
                 shapes: Sequence[Tuple[int, int]], bva: np.ndarray) -> dict:
    """Writes a description and its stream for a BVA of `active` entries
    (int8, or int16 written little-endian)."""
    bva = np.asarray(bva)
    storage = "i8" if bva.dtype == np.int8 else "i16"
    d = describe(shapes, storage)
    if bva.size * bva.dtype.itemsize != d["stream_bytes"]:
        raise QfError(QF_E_ARGUMENT, "converter/ParComm layout mismatch")
    Path(description_path).write_text(json.dumps(d))
    with open(stream_path, "wb") as f:
        f.write(np.ascontiguousarray(bva, dtype=_DTYPES[storage][0]).tobytes())
    return d


class StreamedModel:
    """A stream opened for proving: its parameters and BVA in host memory."""

    def __init__(self, params: Parameters, bva: np.ndarray, owner):
        self.params, self.bva, self._owner = params, bva, owner

    def commit(self, cache_mode: str = "recompute", resident_bytes: Optional[int] = None):
        """`cache_mode` "recompute" (main.rs --cache-mode recompute: the BVA
        stays in page-locked host memory and every pass streams it; at most
        `resident_bytes` of blocks stay in HBM, None = what fits) or "cached"
        (copied into HBM once).  Both write the same roots and proofs; a
        statement of a single PCS block is committed cached, since the
        streamed pass needs two blocks or more."""
        if cache_mode == "recompute" and self.params.blocks >= 2:
            c = self.params.commit_recomputed(self._owner if hasattr(self._owner, "data_ptr") else self.bva,
                                              resident_bytes=resident_bytes)
            c._keep = self._owner
            return c
        if cache_mode in ("cached", "recompute"):
            return self.params.commit(self.bva)
        raise QfError(QF_E_ARGUMENT, f"unknown cache mode {cache_mode!r}")


def open_stream(description: Union[str, Path, dict], source: Union[str, Path, BinaryIO], config: Config = Config(),
                storage_dtype: Optional[str] = None, pinned: bool = True) -> StreamedModel:
    """Description + stream -> parameters and a host BVA ready to commit."""
    field, shapes, dt, active = read_description(description, storage_dtype)
    params = Parameters(shapes, config, field=field)
    if params.active != active:
        raise QfError(QF_E_ARGUMENT, "converter/ParComm layout mismatch")
    bva, owner = read_stream(source, active, dt, pinned)
    return StreamedModel(params, bva, owner)

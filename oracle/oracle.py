"""ORACLE (test infrastructure only): ctypes wrapper of oracle/libqforacle.so.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, as the checker.  The product package never imports it.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libqforacle.so"
_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = ctypes.CDLL(str(LIB))
        P, S = ctypes.c_void_p, ctypes.c_size_t
        BPP = ctypes.POINTER(ctypes.POINTER(ctypes.c_uint8))
        L.qfo_last_error.restype = ctypes.c_char_p
        L.qfo_free.argtypes = [P]
        L.qfo_free.restype = None
        L.qfo_prove.argtypes = [ctypes.POINTER(ctypes.c_uint64), S, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                P, ctypes.c_uint64, ctypes.c_char_p, S, BPP, ctypes.POINTER(S), BPP, ctypes.POINTER(S),
                                BPP, ctypes.POINTER(S), ctypes.POINTER(ctypes.c_double)]
        L.qfo_commit_roots.argtypes = [ctypes.POINTER(ctypes.c_uint64), S, ctypes.c_uint32, ctypes.c_uint32,
                                       ctypes.c_uint32, P, ctypes.c_uint64, ctypes.c_char_p, S]
        L.qfo_demo.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
        L.qfo_wire_fixture.argtypes = [ctypes.c_char_p]
        L.qfo_verify.argtypes = [ctypes.POINTER(ctypes.c_uint64), S, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                 ctypes.c_char_p, ctypes.c_char_p, S, ctypes.c_char_p, S]
        _lib = L
    return _lib


class OracleError(RuntimeError):
    pass


def _check(rc):
    if rc != 0:
        raise OracleError(f"oracle rc={rc}: {lib().qfo_last_error().decode()}")


def _shapes(shapes):
    flat = []
    for s in shapes:
        r, c = (s.rows, s.cols) if hasattr(s, "rows") else s
        flat += [r, c]
    return (ctypes.c_uint64 * len(flat))(*flat), len(shapes)


def _take(p, n):
    try:
        return ctypes.string_at(p, n.value)
    finally:
        lib().qfo_free(ctypes.cast(p, ctypes.c_void_p))


def prove(shapes, chunk_log, packed_log, values, claims: bytes | None = None, rf_bits=100):
    """Returns (roots, claims, proof, (commit_ms, open_ms)) from the CPU restatement."""
    arr, n = _shapes(shapes)
    v = np.ascontiguousarray(values, dtype=np.int8)
    outs = [ctypes.POINTER(ctypes.c_uint8)() for _ in range(3)]
    lens = [ctypes.c_size_t() for _ in range(3)]
    t = (ctypes.c_double * 2)()
    _check(lib().qfo_prove(arr, n, chunk_log, packed_log, rf_bits, v.ctypes.data, v.size, claims,
                           len(claims) if claims else 0, ctypes.byref(outs[0]), ctypes.byref(lens[0]),
                           ctypes.byref(outs[1]), ctypes.byref(lens[1]), ctypes.byref(outs[2]), ctypes.byref(lens[2]), t))
    return _take(outs[0], lens[0]), _take(outs[1], lens[1]), _take(outs[2], lens[2]), (t[0], t[1])


def commit_roots(shapes, chunk_log, packed_log, values, rf_bits=100):
    arr, n = _shapes(shapes)
    v = np.ascontiguousarray(values, dtype=np.int8)
    buf = ctypes.create_string_buffer(32 * 128)
    _check(lib().qfo_commit_roots(arr, n, chunk_log, packed_log, rf_bits, v.ctypes.data, v.size, buf, 32 * 128))
    return buf.raw


def demo():
    d = ctypes.create_string_buffer(32)
    pl, jl = ctypes.c_uint64(), ctypes.c_uint64()
    _check(lib().qfo_demo(d, ctypes.byref(pl), ctypes.byref(jl)))
    return d.raw, pl.value, jl.value


def wire_fixture():
    d = ctypes.create_string_buffer(32)
    _check(lib().qfo_wire_fixture(d))
    return d.raw


def verify(shapes, chunk_log, packed_log, roots: bytes, claims: bytes, proof: bytes, rf_bits=100) -> bool:
    arr, n = _shapes(shapes)
    rc = lib().qfo_verify(arr, n, chunk_log, packed_log, rf_bits, roots, claims, len(claims), proof, len(proof))
    return rc == 0

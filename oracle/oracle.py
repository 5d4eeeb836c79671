"""ORACLE (test infrastructure only): ctypes wrapper of oracle/libqforacle.so.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, to compare results with.  The product package never imports it.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libqforacle.so"
_lib = None
# int gather(void* ctx, const void* in, size_t n, void* out)
GATHER = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p)
# int reduce(void* ctx, uint64_t* data, size_t n)
REDUCE = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64), ctypes.c_size_t)


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
        for name in ("qfo_prove", "qfo_prove_kb"):
            getattr(L, name).argtypes = [ctypes.POINTER(ctypes.c_uint64), S, ctypes.c_uint32, ctypes.c_uint32,
                                         ctypes.c_uint32, P, ctypes.c_uint64, ctypes.c_char_p, S, BPP, ctypes.POINTER(S),
                                         BPP, ctypes.POINTER(S), BPP, ctypes.POINTER(S), ctypes.POINTER(ctypes.c_double)]
        for name in ("qfo_commit_roots", "qfo_commit_roots_kb"):
            getattr(L, name).argtypes = [ctypes.POINTER(ctypes.c_uint64), S, ctypes.c_uint32, ctypes.c_uint32,
                                         ctypes.c_uint32, P, ctypes.c_uint64, ctypes.c_char_p, S]
        for name in ("qfo_demo", "qfo_demo_kb"):
            getattr(L, name).argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
        L.qfo_wire_fixture.argtypes = [ctypes.c_char_p]
        for name in ("qfo_verify", "qfo_verify_kb"):
            getattr(L, name).argtypes = [ctypes.POINTER(ctypes.c_uint64), S, ctypes.c_uint32, ctypes.c_uint32,
                                         ctypes.c_uint32, ctypes.c_char_p, ctypes.c_char_p, S, ctypes.c_char_p, S]
        for name in ("qfo_prove_sharded", "qfo_prove_sharded_kb"):
            getattr(L, name).argtypes = [ctypes.POINTER(ctypes.c_uint64), S, ctypes.c_uint32, ctypes.c_uint32,
                                         ctypes.c_uint32, P, ctypes.c_uint64, ctypes.c_char_p, S, ctypes.c_int,
                                         ctypes.c_int, GATHER, REDUCE, P, BPP, ctypes.POINTER(S), BPP,
                                         ctypes.POINTER(S), BPP, ctypes.POINTER(S)]
        for name in ("qfo_tbv_dense", "qfo_tbv_dense_kb"):
            getattr(L, name).argtypes = [ctypes.POINTER(ctypes.c_uint64), S, ctypes.c_uint32, ctypes.c_uint32,
                                         ctypes.c_uint32, P, ctypes.c_uint64, ctypes.c_char_p, S, ctypes.c_uint32, BPP,
                                         ctypes.POINTER(S)]
        for name in ("qfo_field_ops", "qfo_field_ops_kb"):
            getattr(L, name).argtypes = [ctypes.c_char_p, ctypes.c_char_p, S, P, P, P]
        for name in ("qfo_packed_open", "qfo_packed_open_kb"):
            getattr(L, name).argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_char_p, P,
                                         ctypes.c_char_p, ctypes.c_char_p, S, ctypes.c_char_p, ctypes.c_char_p, BPP,
                                         ctypes.POINTER(S)]
        for name in ("qfo_packed_verify", "qfo_packed_verify_kb"):
            getattr(L, name).argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_char_p,
                                         ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, S,
                                         ctypes.c_char_p, S]
        for name in ("qfo_packed_open_batch", "qfo_packed_open_batch_kb"):
            getattr(L, name).argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_char_p,
                                         ctypes.c_uint32, P, ctypes.c_char_p, ctypes.c_char_p, S, ctypes.c_char_p,
                                         ctypes.c_char_p, BPP, ctypes.POINTER(S)]
        for name in ("qfo_packed_verify_batch", "qfo_packed_verify_batch_kb"):
            getattr(L, name).argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_char_p,
                                         ctypes.c_uint32, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_uint32,
                                         ctypes.c_char_p, ctypes.c_char_p, S, ctypes.c_char_p, S]
        for name in ("qfo_codeword_fold", "qfo_codeword_fold_kb"):
            getattr(L, name).argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_char_p,
                                         ctypes.c_uint32, P, P, ctypes.c_char_p, P, ctypes.POINTER(ctypes.c_int)]
        for name in ("qfo_prove_unchecked", "qfo_prove_unchecked_kb"):
            getattr(L, name).argtypes = [ctypes.POINTER(ctypes.c_uint64), S, ctypes.c_uint32, ctypes.c_uint32,
                                         ctypes.c_uint32, P, ctypes.c_uint64, ctypes.c_char_p, S, BPP,
                                         ctypes.POINTER(S)]
        L.qfo_blake2s_stream.argtypes = [ctypes.c_char_p, S, P, S, ctypes.c_char_p]
        L.qfo_blake2s_compress.argtypes = [P, ctypes.c_char_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_int, P]
        L.qfo_stdrng.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_int, P, S, ctypes.c_char_p, S]
        for name in ("qfo_query_counts", "qfo_query_counts_kb"):
            getattr(L, name).argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, P, S, ctypes.POINTER(S),
                                         ctypes.POINTER(ctypes.c_double)]
        L.qfo_layout.argtypes = [ctypes.POINTER(ctypes.c_uint64), S, P, S, ctypes.POINTER(S)]
        for name in ("qfo_prove_sharded_threads", "qfo_prove_sharded_threads_kb"):
            getattr(L, name).argtypes = [ctypes.POINTER(ctypes.c_uint64), S, ctypes.c_uint32, ctypes.c_uint32,
                                         ctypes.c_uint32, P, ctypes.c_uint64, ctypes.c_char_p, S, ctypes.c_int, BPP,
                                         ctypes.POINTER(S), BPP, ctypes.POINTER(S), BPP, ctypes.POINTER(S),
                                         ctypes.POINTER(ctypes.c_int)]
        L.qfo_encode_column.argtypes = [ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_char_p, S,
                                        ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(S)]
        for name in ("qfo_range_audit", "qfo_range_audit_kb"):
            getattr(L, name).argtypes = [P, ctypes.c_uint64, ctypes.c_char_p, P, ctypes.c_char_p, ctypes.c_char_p,
                                         ctypes.c_char_p]
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


# field: "f65521" (F65521^8, signed 8-bit weights) or "koalabear" (KoalaBear^4,
# signed 16-bit payloads).
_SUFFIX = {"f65521": ("", np.int8), "koalabear": ("_kb", np.int16)}


def prove(shapes, chunk_log, packed_log, values, claims: bytes | None = None, rf_bits=100, field="f65521"):
    """Returns (roots, claims, proof, (commit_ms, open_ms)) from the CPU restatement."""
    sfx, dt = _SUFFIX[field]
    arr, n = _shapes(shapes)
    v = np.ascontiguousarray(values, dtype=dt)
    outs = [ctypes.POINTER(ctypes.c_uint8)() for _ in range(3)]
    lens = [ctypes.c_size_t() for _ in range(3)]
    t = (ctypes.c_double * 2)()
    _check(getattr(lib(), "qfo_prove" + sfx)(arr, n, chunk_log, packed_log, rf_bits, v.ctypes.data, v.size, claims,
                                            len(claims) if claims else 0, ctypes.byref(outs[0]), ctypes.byref(lens[0]),
                                            ctypes.byref(outs[1]), ctypes.byref(lens[1]), ctypes.byref(outs[2]),
                                            ctypes.byref(lens[2]), t))
    return _take(outs[0], lens[0]), _take(outs[1], lens[1]), _take(outs[2], lens[2]), (t[0], t[1])


def prove_sharded(shapes, chunk_log, packed_log, values, rank, world, all_gather, claims: bytes | None = None,
                  rf_bits=100, field="f65521", all_reduce=None):
    """One rank of a block-sharded proof, the CPU shard standing in for the
    rank's device.  `all_gather(data: bytes) -> bytes` returns every rank's
    bytes in rank order; `all_reduce(a: np.ndarray)`, if given, sums a uint64
    array over the ranks in place (else sums go through the gather).
    Returns (roots, claims, proof)."""
    sfx, dt = _SUFFIX[field]
    arr, n = _shapes(shapes)
    v = np.ascontiguousarray(values, dtype=dt)

    def gather(_ctx, src, size, dst):
        try:
            out = all_gather(ctypes.string_at(src, size))
            if len(out) != size * world:
                return 1
            ctypes.memmove(dst, out, len(out))
            return 0
        except Exception:  # the C side turns a nonzero status into an error
            return 1

    def reduce(_ctx, data, size):
        try:
            all_reduce(np.ctypeslib.as_array(data, shape=(size,)))
            return 0
        except Exception:
            return 1

    cb = GATHER(gather)
    rcb = REDUCE(reduce) if all_reduce is not None else ctypes.cast(None, REDUCE)
    outs = [ctypes.POINTER(ctypes.c_uint8)() for _ in range(3)]
    lens = [ctypes.c_size_t() for _ in range(3)]
    _check(getattr(lib(), "qfo_prove_sharded" + sfx)(arr, n, chunk_log, packed_log, rf_bits, v.ctypes.data, v.size,
                                                    claims, len(claims) if claims else 0, rank, world, cb, rcb, None,
                                                    ctypes.byref(outs[0]), ctypes.byref(lens[0]), ctypes.byref(outs[1]),
                                                    ctypes.byref(lens[1]), ctypes.byref(outs[2]), ctypes.byref(lens[2])))
    return _take(outs[0], lens[0]), _take(outs[1], lens[1]), _take(outs[2], lens[2])


def tbv_dense(shapes, chunk_log, packed_log, values, claims: bytes, stride=16, rf_bits=100, field="f65521"):
    """The query that tbv::compile makes of `claims` from a fresh transcript, in
    dense form: (dense weights, query claim, point, evaluation at the point,
    positive cross terms, negative cross terms), each element 16 canonical bytes."""
    sfx, dt = _SUFFIX[field]
    arr, n = _shapes(shapes)
    v = np.ascontiguousarray(values, dtype=dt)
    out, size = ctypes.POINTER(ctypes.c_uint8)(), ctypes.c_size_t()
    _check(getattr(lib(), "qfo_tbv_dense" + sfx)(arr, n, chunk_log, packed_log, rf_bits, v.ctypes.data, v.size, claims,
                                                len(claims), stride, ctypes.byref(out), ctypes.byref(size)))
    blob = _take(out, size)
    logical = 1 << (max(v.size, 1024) - 1).bit_length()
    bits = logical.bit_length() - 1
    cut = [logical, 1, bits, 1, stride - 1, stride - 1]
    assert len(blob) == 16 * sum(cut)
    parts, pos = [], 0
    for k in cut:
        parts.append([blob[pos + 16 * i: pos + 16 * (i + 1)] for i in range(k)])
        pos += 16 * k
    dense, (claim,), point, (evaluation,), positive, negative = parts
    return dense, claim, point, evaluation, positive, negative


def field_ops(a: bytes, b: bytes, field="f65521"):
    """Element-wise (a * b, a^-1 with 0 for 0, a^p) of canonical 16-byte
    elements, as concatenated bytes."""
    assert len(a) == len(b) and len(a) % 16 == 0
    out = [ctypes.create_string_buffer(len(a)) for _ in range(3)]
    _check(getattr(lib(), "qfo_field_ops" + _SUFFIX[field][0])(a, b, len(a) // 16, *out))
    return tuple(o.raw for o in out)


def packed_open(log_n, columns, bits, seed: bytes, values, point: bytes, ctx: bytes, field="f65521"):
    """Single-block packed PCS: commit the 2^log_n canonical base values, open
    at `point` (log_n elements).  Returns (root, claimed value, proof bytes)."""
    v = np.ascontiguousarray(values, dtype=np.int32)
    assert v.size == 1 << log_n and len(seed) == 32 and len(point) == 16 * log_n
    root, value = ctypes.create_string_buffer(32), ctypes.create_string_buffer(16)
    out, size = ctypes.POINTER(ctypes.c_uint8)(), ctypes.c_size_t()
    _check(getattr(lib(), "qfo_packed_open" + _SUFFIX[field][0])(log_n, columns, bits, seed, v.ctypes.data, point, ctx,
                                                                len(ctx), root, value, ctypes.byref(out),
                                                                ctypes.byref(size)))
    return root.raw, value.raw, _take(out, size)


def packed_verify(log_n, columns, bits, seed: bytes, root: bytes, point: bytes, value: bytes, proof: bytes, ctx: bytes,
                  field="f65521") -> bool:
    assert len(seed) == 32 and len(root) == 32 and len(point) == 16 * log_n and len(value) == 16
    rc = getattr(lib(), "qfo_packed_verify" + _SUFFIX[field][0])(log_n, columns, bits, seed, root, point, value, proof,
                                                                len(proof), ctx, len(ctx))
    return rc == 0


def packed_open_batch(log_n, columns, bits, seed: bytes, blocks, values, point: bytes, ctx: bytes, field="f65521"):
    """Batched packed PCS over `blocks` tables of 2^log_n canonical base
    values (block after block): returns (roots, claimed value, proof bytes)."""
    v = np.ascontiguousarray(values, dtype=np.int32)
    assert v.size == blocks << log_n and len(seed) == 32
    assert blocks >= 2 and blocks & (blocks - 1) == 0 and len(point) == 16 * (log_n + blocks.bit_length() - 1)
    roots, value = ctypes.create_string_buffer(32 * blocks), ctypes.create_string_buffer(16)
    out, size = ctypes.POINTER(ctypes.c_uint8)(), ctypes.c_size_t()
    _check(getattr(lib(), "qfo_packed_open_batch" + _SUFFIX[field][0])(log_n, columns, bits, seed, blocks, v.ctypes.data,
                                                                      point, ctx, len(ctx), roots, value,
                                                                      ctypes.byref(out), ctypes.byref(size)))
    return roots.raw, value.raw, _take(out, size)


def packed_verify_batch(log_n, columns, bits, seed: bytes, roots: bytes, point: bytes, value: bytes, proof: bytes,
                        ctx: bytes, field="f65521") -> bool:
    assert len(seed) == 32 and len(roots) % 32 == 0 and len(point) % 16 == 0 and len(value) == 16
    rc = getattr(lib(), "qfo_packed_verify_batch" + _SUFFIX[field][0])(log_n, columns, bits, seed, len(roots) // 32,
                                                                      roots, point, len(point) // 16, value, proof,
                                                                      len(proof), ctx, len(ctx))
    return rc == 0


def codeword_fold_accepted(log_n, columns, bits, pcs_seed: bytes, blocks, values, fold_weights, seed: bytes,
                           check_weights, field="f65521") -> bool:
    """Fold the blocks with `fold_weights`, write the binding rows that `seed`
    samples, and return whether the verifier accepts them under `check_weights`
    (base-field weights, one per block)."""
    v = np.ascontiguousarray(values, dtype=np.int32)
    fw = np.ascontiguousarray(fold_weights, dtype=np.uint32)
    cw = np.ascontiguousarray(check_weights, dtype=np.uint32)
    assert v.size == blocks << log_n and fw.size == cw.size == blocks
    ok = ctypes.c_int()
    _check(getattr(lib(), "qfo_codeword_fold" + _SUFFIX[field][0])(log_n, columns, bits, pcs_seed, blocks,
                                                                  v.ctypes.data, fw.ctypes.data, seed, cw.ctypes.data,
                                                                  ctypes.byref(ok)))
    return bool(ok.value)


def prove_unchecked(shapes, chunk_log, packed_log, values, claims: bytes, rf_bits=100, field="f65521") -> bytes:
    """The prover over `values` (up to the logical length) without the layout
    check of the weights, against the given claims; returns the proof bytes."""
    sfx, dt = _SUFFIX[field]
    arr, n = _shapes(shapes)
    v = np.ascontiguousarray(values, dtype=dt)
    out, size = ctypes.POINTER(ctypes.c_uint8)(), ctypes.c_size_t()
    _check(getattr(lib(), "qfo_prove_unchecked" + sfx)(arr, n, chunk_log, packed_log, rf_bits, v.ctypes.data, v.size,
                                                      claims, len(claims), ctypes.byref(out), ctypes.byref(size)))
    return _take(out, size)


def blake2s_stream(data: bytes, cuts=()) -> bytes:
    """The host BLAKE2s-256 of `data`, fed in pieces ending at `cuts`."""
    c = np.ascontiguousarray(cuts, dtype=np.uint64)
    out = ctypes.create_string_buffer(32)
    _check(lib().qfo_blake2s_stream(data, len(data), c.ctypes.data, c.size, out))
    return out.raw


def blake2s_compress(h, block: bytes, t: int, last: bool, ssse3: bool):
    """One host BLAKE2s compression (scalar or SSSE3 path) of the 8-word state h."""
    hi = np.ascontiguousarray(h, dtype=np.uint32)
    ho = np.zeros(8, dtype=np.uint32)
    assert hi.size == 8 and len(block) == 64
    _check(lib().qfo_blake2s_compress(hi.ctypes.data, block, t, int(last), int(ssse3), ho.ctypes.data))
    return ho


def stdrng(ops, seed: bytes | None = None, seed_u64: int | None = None) -> bytes:
    """Draws from the host StdRng: op k > 0 is fill_bytes(k), -1 next_u32,
    -2 next_u64; the outputs concatenated (little-endian)."""
    o = np.ascontiguousarray(ops, dtype=np.int32)
    size = sum(k if k > 0 else (4 if k == -1 else 8) for k in ops)
    out = ctypes.create_string_buffer(max(size, 1))
    _check(lib().qfo_stdrng(seed, seed_u64 or 0, int(seed_u64 is not None), o.ctypes.data, o.size, out, size))
    return out.raw[:size]


def query_counts(log_n, columns=32, bits=100, field="f65521"):
    """Per level of the packed PCS code sequence: (message_len, index,
    codeword_len, queries with the codeword's rows available, queries
    unlimited); and log2 of the field's size."""
    rows = np.zeros(5 * 64, dtype=np.uint64)
    n, card = ctypes.c_size_t(), ctypes.c_double()
    _check(getattr(lib(), "qfo_query_counts" + _SUFFIX[field][0])(log_n, columns, bits, rows.ctypes.data, rows.size,
                                                                 ctypes.byref(n), ctypes.byref(card)))
    return [tuple(int(x) for x in rows[5 * i: 5 * i + 5]) for i in range(n.value)], card.value


def host_layout(shapes):
    """The host C++ layout: (bucket rows of (matrix, offset, row_offset,
    col_offset, rows, cols, physical_rows, physical_cols), active, logical)."""
    arr, n = _shapes(shapes)
    cap = 8 * 16 * max(n, 1) + 2
    out = np.zeros(cap, dtype=np.uint64)
    nb = ctypes.c_size_t()
    _check(lib().qfo_layout(arr, n, out.ctypes.data, cap, ctypes.byref(nb)))
    rows = [tuple(int(x) for x in out[8 * i: 8 * i + 8]) for i in range(nb.value)]
    return rows, int(out[8 * nb.value]), int(out[8 * nb.value + 1])


def prove_sharded_threads(shapes, chunk_log, packed_log, values, world, claims: bytes | None = None, rf_bits=100,
                          field="f65521"):
    """Every rank of a block-sharded proof as a thread of this process (CPU
    shards).  Returns (roots, claims, proof) of rank 0 and whether all ranks
    wrote the same."""
    sfx, dt = _SUFFIX[field]
    arr, n = _shapes(shapes)
    v = np.ascontiguousarray(values, dtype=dt)
    outs = [ctypes.POINTER(ctypes.c_uint8)() for _ in range(3)]
    lens = [ctypes.c_size_t() for _ in range(3)]
    same = ctypes.c_int()
    _check(getattr(lib(), "qfo_prove_sharded_threads" + sfx)(arr, n, chunk_log, packed_log, rf_bits, v.ctypes.data,
                                                            v.size, claims, len(claims) if claims else 0, world,
                                                            ctypes.byref(outs[0]), ctypes.byref(lens[0]),
                                                            ctypes.byref(outs[1]), ctypes.byref(lens[1]),
                                                            ctypes.byref(outs[2]), ctypes.byref(lens[2]),
                                                            ctypes.byref(same)))
    return _take(outs[0], lens[0]), _take(outs[1], lens[1]), _take(outs[2], lens[2]), bool(same.value)


def encode_column(log_n, message: bytes, bits=100, field="f65521"):
    """The top code of the packed PCS over 2^log_n values: (alphas[1], the
    codeword of `message`), each a list of 16-byte elements."""
    n = len(message) // 16
    alpha, cw, rows = ctypes.create_string_buffer(16 * n), ctypes.create_string_buffer(32 * n), ctypes.c_size_t()
    _check(lib().qfo_encode_column(int(field == "koalabear"), log_n, bits, message, n, alpha, cw, ctypes.byref(rows)))
    split = lambda raw, k: [raw[16 * i: 16 * (i + 1)] for i in range(k)]
    return split(alpha.raw, n), split(cw.raw, 2 * n)


def top_rows(log_n, field="f65521"):
    """Message length of the top code (the codeword rows' count is twice it)."""
    lanes = 8 if field == "f65521" else 4
    return 1 << (log_n - (lanes.bit_length() - 1) - 5)


def commit_roots(shapes, chunk_log, packed_log, values, rf_bits=100, field="f65521"):
    sfx, dt = _SUFFIX[field]
    arr, n = _shapes(shapes)
    v = np.ascontiguousarray(values, dtype=dt)
    buf = ctypes.create_string_buffer(32 * 128)
    _check(getattr(lib(), "qfo_commit_roots" + sfx)(arr, n, chunk_log, packed_log, rf_bits, v.ctypes.data, v.size, buf,
                                                   32 * 128))
    return buf.raw


def demo(field="f65521"):
    d = ctypes.create_string_buffer(32)
    pl, jl = ctypes.c_uint64(), ctypes.c_uint64()
    _check(getattr(lib(), "qfo_demo" + _SUFFIX[field][0])(d, ctypes.byref(pl), ctypes.byref(jl)))
    return d.raw, pl.value, jl.value


def wire_fixture():
    d = ctypes.create_string_buffer(32)
    _check(lib().qfo_wire_fixture(d))
    return d.raw


def verify(shapes, chunk_log, packed_log, roots: bytes, claims: bytes, proof: bytes, rf_bits=100, field="f65521") -> bool:
    arr, n = _shapes(shapes)
    rc = getattr(lib(), "qfo_verify" + _SUFFIX[field][0])(arr, n, chunk_log, packed_log, rf_bits, roots, claims,
                                                         len(claims), proof, len(proof))
    return rc == 0


def range_audit(values, seed: bytes, field="f65521"):
    """LogUp range audit of BVA values: (multiplicities, alpha, lhs, rhs), the
    field elements as 16 canonical bytes; bin k counts the value k - 128
    (int8) or k - 32768 (int16)."""
    sfx, dt = _SUFFIX[field]
    v = np.ascontiguousarray(values, dtype=dt)
    mult = np.zeros(256 if dt == np.int8 else 65536, dtype=np.uint64)
    a, l, r = (ctypes.create_string_buffer(16) for _ in range(3))
    assert len(seed) == 32
    _check(getattr(lib(), "qfo_range_audit" + sfx)(v.ctypes.data, v.size, seed, mult.ctypes.data, a, l, r))
    return mult, a.raw, l.raw, r.raw

"""B200 QAFold commit+open: Python mirror of the reference prover's public API.

The reference crate `parcomm-qafold` exposes `Parameters::{new, commit,
commit_recomputed, prove, verify}`, `Proof::{to_bytes, from_bytes}` and
`tbv::evaluate_claims` (qafold/f65521/src/protocol.rs:108-321, tbv.rs:143-185).
This module exposes the same calls over the C ABI of libparcomm_qafold.so
(include/parcomm_qafold.h).  Proving runs on the GPU through hand-written
sm_100a kernels; there is no CPU fallback: without a CUDA device `commit`
raises `QfError(QF_E_NO_DEVICE)`.  Verification is host-only, as in the
reference (its verifier always runs on one thread, main.rs:215-217).
"""
from __future__ import annotations

import ctypes
import dataclasses
import hashlib
from pathlib import Path
from typing import List, Optional, Sequence, Tuple

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "_lib" / "libparcomm_qafold.so"

FIELD_F65521 = 1
FIELD_KOALABEAR = 2
RESIDENT_AUTO = (1 << 64) - 1  # QF_RESIDENT_AUTO
ERRORS = {
    -1: "EncodingError", -2: "HashingError", -3: "InvalidCommitment", -4: "InvalidNumberOfVariables",
    -5: "InvalidParameters", -6: "TranscriptError", -7: "ProtocolError", -8: "CudaError", -9: "ArgumentError",
    -10: "NoDevice",
}
QF_E_ARGUMENT = -9
QF_E_NO_DEVICE = -10


class QfError(RuntimeError):
    """A rejected call: `code` is the QF_E_* value, the message the reference's check string."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{ERRORS.get(code, code)}: {message}")
        self.code = code


class _Shape(ctypes.Structure):
    _fields_ = [("rows", ctypes.c_uint64), ("cols", ctypes.c_uint64)]


class _Config(ctypes.Structure):
    _fields_ = [("chunk_log", ctypes.c_uint32), ("packed_log", ctypes.c_uint32), ("query_rf_bits", ctypes.c_uint32)]


class _Profile(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "commit_ms", "upload_ms", "eo_ms", "projection_ms", "folding_ms", "sumcheck_ms", "binding_ms",
        "native_opening_ms", "decide_ms", "open_ms")] + [("kernel_launches", ctypes.c_uint64)]


_lib = None

EXPORTED = (
    "qf_params_new", "qf_params_free", "qf_params_info", "qf_commit", "qf_committed_free", "qf_statement_json",
    "qf_benchmark_points", "qf_eval_claims", "qf_prove", "qf_verify", "qf_free_bytes", "qf_last_error",
    "qf_kernel_timing", "qf_kernel_stats", "qf_kernel_launches", "qf_commit_block_noalloc", "qf_commit_streamed",
    "qf_committed_stream_info", "qf_open", "qf_device_cache_limit", "qf_range_audit", "qf_kernel_int_peaks",
    "qf_kernel_option", "qf_prove_sharded",
)

# int gather(void* ctx, const void* in, size_t n, void* out); int reduce(void* ctx, uint64_t* data, size_t n)
GATHER_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p)
REDUCE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64), ctypes.c_size_t)


def lib() -> ctypes.CDLL:
    """Loads the in-tree library (built by `parcomm_b200.build`)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise QfError(-9, f"{LIB_PATH} is missing; run `python -m parcomm_b200.build`")
        L = ctypes.CDLL(str(LIB_PATH))
        P, S, U64, U32 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_uint32
        BP = ctypes.POINTER(ctypes.c_uint8)
        L.qf_params_new.argtypes = [ctypes.c_int, ctypes.POINTER(_Shape), S, ctypes.POINTER(_Config), ctypes.POINTER(P)]
        L.qf_params_free.argtypes = [P]
        L.qf_params_free.restype = None
        L.qf_params_info.argtypes = [P, ctypes.POINTER(U64), ctypes.POINTER(U64), ctypes.POINTER(U64),
                                     ctypes.POINTER(U64), ctypes.c_char_p]
        L.qf_commit.argtypes = [P, P, U64, ctypes.c_int, ctypes.POINTER(P), ctypes.c_char_p]
        L.qf_commit_streamed.argtypes = [P, P, U64, U64, ctypes.POINTER(P), ctypes.c_char_p]
        L.qf_committed_stream_info.argtypes = [P, ctypes.POINTER(U64), ctypes.POINTER(U64), ctypes.POINTER(U64)]
        L.qf_committed_free.argtypes = [P]
        L.qf_committed_free.restype = None
        L.qf_statement_json.argtypes = [P, ctypes.c_char_p, ctypes.c_char_p, S, ctypes.POINTER(S)]
        L.qf_benchmark_points.argtypes = [P, ctypes.c_char_p, ctypes.c_char_p, S, ctypes.POINTER(S)]
        L.qf_eval_claims.argtypes = [P, P, ctypes.c_char_p, S, ctypes.c_char_p, S, ctypes.POINTER(S)]
        L.qf_prove.argtypes = [P, P, ctypes.c_char_p, S, ctypes.POINTER(BP), ctypes.POINTER(S), ctypes.POINTER(_Profile)]
        L.qf_verify.argtypes = [P, ctypes.c_char_p, ctypes.c_char_p, S, ctypes.c_char_p, S]
        L.qf_open.argtypes = [P, P, ctypes.c_char_p, S, ctypes.POINTER(BP), ctypes.POINTER(S), ctypes.POINTER(_Profile)]
        L.qf_free_bytes.argtypes = [P]
        L.qf_free_bytes.restype = None
        L.qf_last_error.argtypes = [ctypes.c_char_p, S]
        L.qf_last_error.restype = S
        L.qf_kernel_timing.argtypes = [ctypes.c_int]
        L.qf_kernel_stats.argtypes = [ctypes.c_char_p, S, ctypes.POINTER(S)]
        L.qf_kernel_launches.argtypes = []
        L.qf_kernel_launches.restype = U64
        L.qf_device_cache_limit.argtypes = [U64]
        L.qf_kernel_int_peaks.argtypes = [ctypes.POINTER(ctypes.c_double)]
        L.qf_kernel_option.argtypes = [ctypes.c_char_p, ctypes.c_int]
        L.qf_commit_block_noalloc.argtypes = [P, P, U64, U64, P, P]
        L.qf_range_audit.argtypes = [P, P, ctypes.c_char_p, P, S, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                     ctypes.POINTER(ctypes.c_int)]
        L.qf_prove_sharded.argtypes = [P, P, U64, ctypes.c_int, ctypes.c_int, GATHER_FN, REDUCE_FN, P, ctypes.c_char_p,
                                       S, ctypes.c_char_p, ctypes.POINTER(BP), ctypes.POINTER(S)]
        for name in EXPORTED:
            if not hasattr(L, name):
                raise QfError(-9, f"library does not export {name}")
        _lib = L
    return _lib


def _ready(t) -> None:
    """The library reads device weights on its own streams: the stream that
    produced a CUDA tensor must have finished writing it."""
    if getattr(t, "is_cuda", False):
        import torch
        torch.cuda.current_stream(t.device).synchronize()


def _check(rc: int) -> None:
    if rc != 0:
        buf = ctypes.create_string_buffer(4096)
        lib().qf_last_error(buf, 4096)
        raise QfError(rc, buf.value.decode(errors="replace"))


@dataclasses.dataclass(frozen=True)
class Shape:
    rows: int
    cols: int


@dataclasses.dataclass(frozen=True)
class Config:
    """protocol::Config (protocol.rs:18-32)."""
    chunk_log: int = 30
    packed_log: int = 4
    query_rf_bits: int = 100


@dataclasses.dataclass
class Claim:
    """tbv::Claim: row/col points and value, 16-byte canonical scalars each."""
    row: List[bytes]
    col: List[bytes]
    value: bytes


@dataclasses.dataclass
class ProverProfile:
    commit_ms: float
    upload_ms: float
    eo_ms: float
    projection_ms: float
    folding_ms: float
    sumcheck_ms: float
    binding_ms: float
    native_opening_ms: float
    decide_ms: float
    open_ms: float
    kernel_launches: int


def _row_bits(n: int) -> int:
    return (n - 1).bit_length() if n > 1 else 0


def claims_to_bytes(claims: Sequence[Claim]) -> bytes:
    out = bytearray()
    for c in claims:
        for v in c.row:
            out += v
        for v in c.col:
            out += v
        out += c.value
    return bytes(out)


def claims_from_bytes(shapes: Sequence[Shape], data: bytes, with_value: bool = True) -> List[Claim]:
    claims, off = [], 0
    for s in shapes:
        r = [data[off + 16 * i: off + 16 * i + 16] for i in range(_row_bits(s.rows))]
        off += 16 * len(r)
        c = [data[off + 16 * i: off + 16 * i + 16] for i in range(_row_bits(s.cols))]
        off += 16 * len(c)
        v = b"\x00" * 16
        if with_value:
            v = data[off: off + 16]
            off += 16
        claims.append(Claim(r, c, v))
    if off != len(data):
        raise QfError(-9, "claims length mismatch")
    return claims


class Committed:
    """Committed state: weights, codewords and Merkle trees resident in HBM,
    or (recompute mode) the roots only, over weights kept in host memory."""

    def __init__(self, params: "Parameters", handle: int, roots: List[bytes], keep=None):
        self.params = params
        self._h = ctypes.c_void_p(handle)
        self.roots = roots
        self.consumed = False
        self._keep = keep  # host weights the handle streams from

    @property
    def statement(self) -> "Commitment":
        return Commitment(self.params, list(self.roots))

    def stream_info(self) -> Tuple[int, int, int]:
        """Recompute mode: (host->device bytes of weights copied so far,
        blocks kept in HBM, blocks holding weights)."""
        v = [ctypes.c_uint64() for _ in range(3)]
        _check(lib().qf_committed_stream_info(self._h, *[ctypes.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def stream_bytes(self) -> int:
        return self.stream_info()[0]

    def range_audit(self, seed: Optional[bytes] = None) -> "RangeAudit":
        """LogUp range audit of the committed weights over the entry type's
        table (qf_range_audit); not part of the proof.  The default seed is
        BLAKE2s of the concatenated roots, which ties alpha to the
        commitment."""
        if seed is None:
            seed = hashlib.blake2s(b"".join(self.roots)).digest()
        if len(seed) != 32:
            raise QfError(QF_E_ARGUMENT, "range audit seed must be 32 bytes")
        bins = 256 if self.params.field == FIELD_F65521 else 65536
        mult = np.zeros(bins, dtype=np.uint64)
        a, l, r = (ctypes.create_string_buffer(16) for _ in range(3))
        holds = ctypes.c_int()
        _check(lib().qf_range_audit(self.params._h, self._h, seed, mult.ctypes.data, bins, a, l, r, ctypes.byref(holds)))
        return RangeAudit(mult, a.raw, l.raw, r.raw, bool(holds.value))

    def close(self) -> None:
        if self._h:
            lib().qf_committed_free(self._h)
            self._h = ctypes.c_void_p(0)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclasses.dataclass
@dataclasses.dataclass
class RangeAudit:
    """Result of Committed.range_audit: multiplicities (bin k counts the value
    k - 128 for int8, k - 32768 for int16), alpha, lhs = sum_i 1/(alpha - v_i),
    rhs = sum_t m_t/(alpha - t) (16 canonical bytes each), and whether the
    identity holds."""
    multiplicities: np.ndarray
    alpha: bytes
    lhs: bytes
    rhs: bytes
    holds: bool


class Commitment:
    """protocol::Commitment: version 2, config, shapes, parameter digest, block roots."""
    params: "Parameters"
    roots: List[bytes]

    def to_json(self) -> bytes:
        return self.params.statement_json(self.roots)


class Proof:
    """The bincode-fixint wire of protocol::Proof (protocol.rs:88-107)."""

    def __init__(self, data: bytes):
        self.data = bytes(data)

    def to_bytes(self) -> bytes:
        return self.data

    @staticmethod
    def from_bytes(data: bytes) -> "Proof":
        if len(data) > 256 * 1024 * 1024:
            raise QfError(-7, "oversize ParComm proof")
        return Proof(data)


class Parameters:
    """protocol::Parameters::new(shapes, config).

    `field` picks the message field: FIELD_F65521 (F65521^8, signed 8-bit
    weights; qafold/f65521) or FIELD_KOALABEAR (KoalaBear^4, signed 16-bit
    payloads; qafold/koalabear)."""

    def __init__(self, shapes: Sequence[Tuple[int, int]] | Sequence[Shape], config: Config = Config(),
                 field: int = FIELD_F65521):
        self.shapes = [s if isinstance(s, Shape) else Shape(int(s[0]), int(s[1])) for s in shapes]
        self.config = config
        self.field = field
        self.weight_dtype = np.int16 if field == FIELD_KOALABEAR else np.int8
        arr = (_Shape * len(self.shapes))(*[_Shape(s.rows, s.cols) for s in self.shapes])
        cfg = _Config(config.chunk_log, config.packed_log, config.query_rf_bits)
        h = ctypes.c_void_p()
        _check(lib().qf_params_new(field, arr, len(self.shapes), ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        a, l, b, k = (ctypes.c_uint64() for _ in range(4))
        dig = ctypes.create_string_buffer(32)
        _check(lib().qf_params_info(self._h, ctypes.byref(a), ctypes.byref(l), ctypes.byref(b), ctypes.byref(k), dig))
        self.active, self.logical, self.blocks, self.buckets = a.value, l.value, b.value, k.value
        self.parameter_digest = dig.raw

    def __del__(self):
        try:
            if self._h:
                lib().qf_params_free(self._h)
        except Exception:
            pass

    # -- commit (protocol.rs:131-185); cached and recompute modes give identical bytes
    def commit(self, values, on_device: bool = False) -> Committed:
        if on_device:
            if int(values.element_size()) != np.dtype(self.weight_dtype).itemsize:
                raise QfError(-9, f"device weights must be {np.dtype(self.weight_dtype).name}")
            _ready(values)
            ptr, n = int(values.data_ptr()), int(values.numel())
        else:
            arr = np.ascontiguousarray(values, dtype=self.weight_dtype)
            ptr, n = arr.ctypes.data, arr.size
        h = ctypes.c_void_p()
        roots = ctypes.create_string_buffer(32 * max(self.blocks, 1))
        _check(lib().qf_commit(self._h, ctypes.c_void_p(ptr), n, int(on_device), ctypes.byref(h), roots))
        return Committed(self, h.value, [roots.raw[32 * i: 32 * i + 32] for i in range(self.blocks)])

    def commit_recomputed(self, values, resident_bytes: Optional[int] = 0) -> Committed:
        """Parameters::commit_recomputed: the reference's recompute mode: only
        the roots stay on the device and binding re-encodes each block.  Host
        weights (a numpy array, or a CPU tensor, ideally in pinned memory) stay
        where they are and are streamed into HBM one PCS block at a time for
        every pass; `resident_bytes` of leading blocks are kept in HBM after
        the first pass (None: as many as the device's free memory allows next
        to the proof's own peak).  A CUDA tensor stays where it is and is read
        in place.  The weights must stay unchanged while the handle lives.
        The roots, claims and proof bytes equal those of `commit`."""
        if hasattr(values, "data_ptr"):
            if int(values.element_size()) != np.dtype(self.weight_dtype).itemsize or not values.is_contiguous():
                raise QfError(-9, f"host weights must be contiguous {np.dtype(self.weight_dtype).name}")
            _ready(values)
            keep, ptr, n = values, int(values.data_ptr()), int(values.numel())
        else:
            keep = np.ascontiguousarray(values, dtype=self.weight_dtype)
            ptr, n = keep.ctypes.data, keep.size
        h = ctypes.c_void_p()
        roots = ctypes.create_string_buffer(32 * max(self.blocks, 1))
        budget = RESIDENT_AUTO if resident_bytes is None else int(resident_bytes)
        _check(lib().qf_commit_streamed(self._h, ctypes.c_void_p(ptr), n, budget, ctypes.byref(h), roots))
        return Committed(self, h.value, [roots.raw[32 * i: 32 * i + 32] for i in range(self.blocks)], keep=keep)

    def block_root_noalloc(self, bva, block: int, root, stream: int = 0) -> None:
        """qf_commit_block_noalloc: the root of PCS block `block` of the
        device BVA tensor `bva` (int8, active entries) into the 32-byte
        device tensor `root`, asynchronously on the CUDA stream handle
        `stream`, with no device allocation (blocks of at most 2^20 weights)."""
        _check(lib().qf_commit_block_noalloc(self._h, ctypes.c_void_p(int(bva.data_ptr())), int(bva.numel()), int(block),
                                             ctypes.c_void_p(int(root.data_ptr())), ctypes.c_void_p(int(stream))))

    def statement_json(self, roots: Sequence[bytes]) -> bytes:
        r = b"".join(roots)
        n = ctypes.c_size_t()
        _check(lib().qf_statement_json(self._h, r, None, 0, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        _check(lib().qf_statement_json(self._h, r, buf, n.value, ctypes.byref(n)))
        return buf.raw[: n.value]

    def benchmark_points(self, roots: Sequence[bytes]) -> bytes:
        """The points of main.rs:190-204 (transcript over the statement)."""
        r = b"".join(roots)
        n = ctypes.c_size_t()
        _check(lib().qf_benchmark_points(self._h, r, None, 0, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(max(n.value, 1))
        _check(lib().qf_benchmark_points(self._h, r, buf, n.value, ctypes.byref(n)))
        return buf.raw[: n.value]

    def evaluate_claims(self, committed: Committed, points: bytes) -> List[Claim]:
        """tbv::evaluate_claims over the committed weights (on the GPU)."""
        n = ctypes.c_size_t()
        cap = len(points) + 16 * len(self.shapes)
        buf = ctypes.create_string_buffer(cap)
        _check(lib().qf_eval_claims(self._h, committed._h, points, len(points), buf, cap, ctypes.byref(n)))
        return claims_from_bytes(self.shapes, buf.raw[: n.value])

    def prove(self, committed: Committed, claims: Sequence[Claim]) -> Tuple[Proof, ProverProfile]:
        cb = claims_to_bytes(claims)
        out = ctypes.POINTER(ctypes.c_uint8)()
        n = ctypes.c_size_t()
        prof = _Profile()
        _check(lib().qf_prove(self._h, committed._h, cb, len(cb), ctypes.byref(out), ctypes.byref(n), ctypes.byref(prof)))
        try:
            data = ctypes.string_at(out, n.value)
        finally:
            lib().qf_free_bytes(ctypes.cast(out, ctypes.c_void_p))
        committed.consumed = True
        return Proof(data), ProverProfile(*[getattr(prof, f) for f, _ in _Profile._fields_])

    def open(self, committed: Committed, claims: Sequence[Claim]) -> Tuple[Proof, ProverProfile]:
        """`prove` without consuming the commitment (qf_open): a pool answers
        many claims on one commitment.  Calls on one commitment must not
        overlap."""
        cb = claims_to_bytes(claims)
        out = ctypes.POINTER(ctypes.c_uint8)()
        n = ctypes.c_size_t()
        prof = _Profile()
        _check(lib().qf_open(self._h, committed._h, cb, len(cb), ctypes.byref(out), ctypes.byref(n), ctypes.byref(prof)))
        try:
            data = ctypes.string_at(out, n.value)
        finally:
            lib().qf_free_bytes(ctypes.cast(out, ctypes.c_void_p))
        return Proof(data), ProverProfile(*[getattr(prof, f) for f, _ in _Profile._fields_])

    def prove_sharded(self, values, rank: int, world: int, all_gather, all_reduce=None,
                      claims: Optional[Sequence[Claim]] = None) -> Tuple[List[bytes], Proof]:
        """One rank of a proof whose PCS blocks are spread over `world` ranks
        (qf_prove_sharded): rank r holds blocks [B r / world, B (r + 1) /
        world) of the host BVA `values` (every rank passes the same array) on
        the current device.  `all_gather(data: bytes) -> bytes` returns every
        rank's bytes in rank order; `all_reduce(a)`, if given, sums a uint64
        numpy array over the ranks in place.  `claims` None takes the
        benchmark points.  Every rank returns the roots and the proof that
        one device holding all blocks writes."""
        v = np.ascontiguousarray(values, dtype=self.weight_dtype)

        def gather(_ctx, src, size, dst):
            try:
                out = all_gather(ctypes.string_at(src, size))
                if len(out) != size * world:
                    return 1
                ctypes.memmove(dst, out, len(out))
                return 0
            except Exception:  # the library turns a nonzero status into an error
                return 1

        def reduce(_ctx, data, size):
            try:
                all_reduce(np.ctypeslib.as_array(data, shape=(size,)))
                return 0
            except Exception:
                return 1

        g = GATHER_FN(gather)
        r = REDUCE_FN(reduce) if all_reduce is not None else ctypes.cast(None, REDUCE_FN)
        cb = claims_to_bytes(claims) if claims is not None else None
        roots = ctypes.create_string_buffer(32 * self.blocks)
        out = ctypes.POINTER(ctypes.c_uint8)()
        n = ctypes.c_size_t()
        _check(lib().qf_prove_sharded(self._h, v.ctypes.data, v.size, rank, world, g, r, None, cb,
                                      len(cb) if cb else 0, roots, ctypes.byref(out), ctypes.byref(n)))
        try:
            data = ctypes.string_at(out, n.value)
        finally:
            lib().qf_free_bytes(ctypes.cast(out, ctypes.c_void_p))
        return [roots.raw[32 * b: 32 * (b + 1)] for b in range(self.blocks)], Proof(data)

    def verify(self, statement: Commitment | Sequence[bytes], claims: Sequence[Claim], proof: Proof | bytes) -> None:
        """Raises QfError when the proof is rejected (protocol.rs:266-320)."""
        roots = statement.roots if isinstance(statement, Commitment) else list(statement)
        pb = proof.to_bytes() if isinstance(proof, Proof) else bytes(proof)
        cb = claims_to_bytes(claims)
        _check(lib().qf_verify(self._h, b"".join(roots), cb, len(cb), pb, len(pb)))


def kernel_timing(enable: bool) -> None:
    """Enables per-kernel CUDA-event timing (diagnostics; adds event records per launch)."""
    _check(lib().qf_kernel_timing(int(enable)))


def kernel_stats() -> dict:
    """{kernel: {"launches", "ms", "bytes"}} since the last kernel_timing(True)."""
    import json
    n = ctypes.c_size_t()
    _check(lib().qf_kernel_stats(None, 0, ctypes.byref(n)))
    buf = ctypes.create_string_buffer(n.value + 1)
    _check(lib().qf_kernel_stats(buf, n.value + 1, ctypes.byref(n)))
    return json.loads(buf.raw[: n.value].decode())


def device_cache_limit(nbytes: int) -> None:
    """At most `nbytes` of released device buffers stay cached for reuse."""
    _check(lib().qf_device_cache_limit(int(nbytes)))


def kernel_launches() -> int:
    return int(lib().qf_kernel_launches())


def kernel_option(name: str, value: int) -> None:
    """qf_kernel_option: "imma" (tensor-core weight passes, default off),
    "per_matrix" (one launch per term / bucket / block, default off) or
    "core_dots" (where the EO, sumcheck and LiteBullet product sums run: 0
    per kernel as measured fastest, 1 CUDA cores, 2 tensor cores); every
    setting writes identical bytes."""
    _check(lib().qf_kernel_option(name.encode(), int(value)))


def int_peaks() -> dict:
    """The device's measured integer issue peaks (thread-level operations/s):
    the ALU pipe (XOR chains), the FMA pipe (multiply-add chains), both
    interleaved, and widening 32 x 32 -> 64-bit multiply-adds; the
    denominators of the integer roofline."""
    out = (ctypes.c_double * 6)()
    _check(lib().qf_kernel_int_peaks(out))
    return {"alu_ops_per_s": out[0], "fma_ops_per_s": out[1], "issue_ops_per_s": out[2], "mad_wide_per_s": out[3],
            "dp4a_per_s": out[4], "rotate_per_s": out[5]}


def demo_shapes() -> List[Shape]:
    """The demo collection of main.rs:108-115."""
    return [Shape(31, 37), Shape(65, 17), Shape(1, 7), Shape(9, 1)]


def encode_bva(layout_params: Parameters, matrices: Sequence[np.ndarray]) -> np.ndarray:
    """Layout::encode (layout.rs:115-135): dense matrices -> BVA of `active` entries."""
    from .layout import encode
    return encode(layout_params.shapes, matrices, layout_params.weight_dtype)

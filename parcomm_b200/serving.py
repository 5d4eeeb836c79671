"""Continuous-batching request loop over a pool of QAFold commitments.

The pool holds committed matrices in HBM, each its own statement
(`Parameters` over one shape).  In cache mode the weights, codewords and
Merkle trees stay resident and openings read them.  In recompute mode only
the weights stay resident, and each opening re-encodes its block: this is
the mode for sets whose codewords do not fit.  There are two request kinds:

  OpenRequest(matrices, points)  claims at fresh points for 1..64 pooled
                                 matrices: one proof per matrix (qf_open,
                                 which keeps the commitment for later requests)
  CommitRequest(weights)         a new matrix is committed and joins the pool

Scheduling is continuous batching, not a queue of whole requests:

- A request is split into tasks (one per matrix) that enter one FIFO.
- `slots` worker threads take tasks from its head. A task starts when a slot
  is free and its HBM estimate fits the budget left by the tasks in flight
  (and by the matrices the pool has gained).
- A request that arrives while others run is admitted as slots and memory
  free up. Its tasks interleave with theirs. Each commitment owns a CUDA
  stream, and the library releases the GIL inside every call, so the
  kernels and host rounds of different requests overlap on the device.
- Tasks on one commitment take its lock: calls on one handle never overlap.

A proof depends only on the commitment and the claims. The same request
therefore gives the same bytes alone and in any mix; the GPU tests check
this.
"""
from __future__ import annotations

import dataclasses
import itertools
import threading
import time
from collections import deque
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import FIELD_F65521, FIELD_KOALABEAR, Config, Parameters, QfError, Shape, claims_to_bytes

ELEMENT_BYTES = 16


# ---------------------------------------------------------------- memory model
def proof_bytes_estimate(params: Parameters, recompute: bool) -> int:
    """Device memory one opening of `params` holds at its peak: the EO round
    vectors (2.5 x N/stride elements) or the batch opening's tables and
    codewords (about 7.5 x packed elements), plus the re-encoded block in
    recompute mode (2.25 x packed elements)."""
    lanes = 4 if params.field == FIELD_KOALABEAR else 8
    block_len = params.logical // max(params.blocks, 1)
    m = block_len // lanes
    rows = params.logical >> params.config.packed_log
    peak = max(rows * 5 // 2, m * 15 // 2) * ELEMENT_BYTES
    if recompute:
        peak += m * 9 // 4 * ELEMENT_BYTES
    return int(peak)


def resident_bytes_estimate(params: Parameters, recompute: bool) -> int:
    """HBM a commitment keeps: its weights, plus every block's codeword and
    Merkle tree (2.25 x packed elements per block) in cache mode."""
    entry = np.dtype(params.weight_dtype).itemsize
    lanes = 4 if params.field == FIELD_KOALABEAR else 8
    block_len = params.logical // max(params.blocks, 1)
    codewords = 0 if recompute else params.blocks * (block_len // lanes) * 9 // 4 * ELEMENT_BYTES
    return int(params.active * entry + codewords)


# ---------------------------------------------------------------- pool
@dataclasses.dataclass
class PoolEntry:
    key: int
    shape: Tuple[int, int]
    params: Parameters
    committed: object
    recompute: bool
    weights: object  # the resident weights (kept alive with the commitment)
    lock: threading.Lock = dataclasses.field(default_factory=threading.Lock)


class Pool:
    """Committed matrices by key; one `Parameters` per (shape, field, config)."""

    def __init__(self, field: int = FIELD_F65521):
        self.field = field
        self._entries: Dict[int, PoolEntry] = {}
        self._params: Dict[Tuple, Parameters] = {}
        self._keys = itertools.count()
        self._mu = threading.Lock()

    def params_for(self, shape: Tuple[int, int], config: Config) -> Parameters:
        k = (tuple(shape), config)
        with self._mu:
            p = self._params.get(k)
        if p is None:
            p = Parameters([shape], config, field=self.field)
            with self._mu:
                p = self._params.setdefault(k, p)
        return p

    def commit(self, weights, config: Config, recompute: bool) -> PoolEntry:
        """Commits a device tensor of one matrix (rows x cols) laid out as its BVA."""
        shape = (int(weights.shape[0]), int(weights.shape[1]))
        p = self.params_for(shape, config)
        bva = layout_bva(p, weights)
        c = p.commit_recomputed(bva) if recompute else p.commit(bva, on_device=True)
        # Cache mode copies the weights into the commitment; recompute mode reads them in place.
        e = PoolEntry(next(self._keys), shape, p, c, recompute, bva if recompute else None)
        with self._mu:
            self._entries[e.key] = e
        return e

    def get(self, key: int) -> PoolEntry:
        with self._mu:
            return self._entries[key]

    def keys(self) -> List[int]:
        with self._mu:
            return list(self._entries)

    def __len__(self) -> int:
        with self._mu:
            return len(self._entries)

    def resident_bytes(self) -> int:
        with self._mu:
            return sum(resident_bytes_estimate(e.params, e.recompute) for e in self._entries.values())


def layout_bva(params: Parameters, weights):
    """The BVA of a single-matrix statement from a device tensor: its buckets
    in layout order (layout.rs), padding zeroed."""
    import torch
    from .layout import buckets

    bs, active, _ = buckets(params.shapes)
    out = torch.zeros(active, dtype=weights.dtype, device=weights.device)
    for b in bs:
        dst = out[b.offset: b.offset + b.rows * b.cols].view(b.rows, b.cols)
        dst[: b.physical_rows, : b.physical_cols] = weights[b.row_offset: b.row_offset + b.physical_rows,
                                                            b.col_offset: b.col_offset + b.physical_cols]
    return out


# ---------------------------------------------------------------- requests and tasks
@dataclasses.dataclass
class OpenRequest:
    """Claims at `points[i]` (row point then column point, 16-byte canonical
    coordinates) on pooled matrix `matrices[i]`."""
    matrices: Sequence[int]
    points: Sequence[bytes]


@dataclasses.dataclass
class CommitRequest:
    """A new matrix (device tensor, rows x cols) to commit into the pool."""
    weights: object
    config: Config = Config(30, 4)
    recompute: bool = True


@dataclasses.dataclass
class Result:
    rid: int
    kind: str
    arrival: float
    started: Optional[float] = None
    done: Optional[float] = None
    outputs: List = dataclasses.field(default_factory=list)  # per task: (claims bytes, proof bytes) or pool key
    weights: int = 0  # matrix entries opened or committed
    error: Optional[str] = None

    @property
    def latency(self) -> float:
        return self.done - self.arrival


class Task:
    """One unit of work: `fn()` returns its output; `mem` is its HBM estimate
    while it runs, of which `keep` stays taken after it succeeds (a commitment
    that joins the pool)."""

    def __init__(self, result: Result, index: int, mem: int, fn: Callable[[], object], weights: int, keep: int = 0):
        self.result, self.index, self.mem, self.fn, self.weights, self.keep = result, index, mem, fn, weights, keep


def open_tasks(pool: Pool, req: OpenRequest, result: Result) -> List[Task]:
    tasks = []
    for i, (key, pts) in enumerate(zip(req.matrices, req.points)):
        e = pool.get(key)

        def run(e=e, pts=pts):
            with e.lock:
                claims = e.params.evaluate_claims(e.committed, pts)
                proof, _ = e.params.open(e.committed, claims)
            return claims_to_bytes(claims), proof.to_bytes()

        tasks.append(Task(result, i, proof_bytes_estimate(e.params, e.recompute), run, e.shape[0] * e.shape[1]))
    return tasks


def commit_task(pool: Pool, req: CommitRequest, result: Result) -> List[Task]:
    shape = (int(req.weights.shape[0]), int(req.weights.shape[1]))
    p = pool.params_for(shape, req.config)
    keep = resident_bytes_estimate(p, req.recompute)

    def run():
        return pool.commit(req.weights, req.config, req.recompute).key

    return [Task(result, 0, keep + proof_bytes_estimate(p, True), run, shape[0] * shape[1], keep)]


# ---------------------------------------------------------------- engine
class Engine:
    """`slots` workers over one FIFO of tasks, admitted under `hbm_budget`
    bytes (None: no limit).  `submit` returns the request's Result, filled in
    when its last task finishes; `drain` waits for everything submitted."""

    def __init__(self, pool: Optional[Pool], slots: int = 4, hbm_budget: Optional[int] = None,
                 make_tasks: Optional[Callable] = None):
        self.pool = pool
        self.slots = slots
        self.budget = hbm_budget
        self._make_tasks = make_tasks or self._default_tasks
        self._queue: deque = deque()
        self._cv = threading.Condition()
        self._in_use = 0
        self._peak_in_use = 0
        self._running = 0
        self._peak_running = 0
        self._pending: Dict[int, int] = {}  # rid -> tasks left
        self._results: List[Result] = []
        self._rids = itertools.count()
        self._stop = False
        self._workers = [threading.Thread(target=self._work, daemon=True) for _ in range(slots)]
        for w in self._workers:
            w.start()

    def _default_tasks(self, req, result: Result) -> List[Task]:
        if isinstance(req, OpenRequest):
            return open_tasks(self.pool, req, result)
        if isinstance(req, CommitRequest):
            return commit_task(self.pool, req, result)
        raise QfError(-9, f"unknown request {type(req).__name__}")

    def submit(self, req, arrival: Optional[float] = None) -> Result:
        r = Result(next(self._rids), type(req).__name__, time.perf_counter() if arrival is None else arrival)
        tasks = self._make_tasks(req, r)
        r.weights = sum(t.weights for t in tasks)
        with self._cv:
            if self.budget is not None:
                for t in tasks:
                    if t.mem > self.budget:
                        raise QfError(-9, f"task needs {t.mem} bytes, more than the whole budget {self.budget}")
            self._results.append(r)
            self._pending[r.rid] = len(tasks)
            if not tasks:
                r.started = r.done = time.perf_counter()
            self._queue.extend(tasks)
            self._cv.notify_all()
        return r

    def _fits(self, t: Task) -> bool:
        return self.budget is None or self._in_use + t.mem <= self.budget

    def _work(self):
        while True:
            with self._cv:
                # Strict FIFO: the head task starts once it fits next to the tasks in flight.
                while not self._stop and not (self._queue and self._fits(self._queue[0])):
                    if self._queue and self._running == 0:
                        break  # nothing in flight will free memory: the head cannot ever fit
                    self._cv.wait()
                if self._stop:
                    return
                t = self._queue.popleft()
                if not self._fits(t):
                    self._finish(t, None, "HBM budget exhausted by the pool")
                    continue
                self._in_use += t.mem
                self._running += 1
                self._peak_in_use = max(self._peak_in_use, self._in_use)
                self._peak_running = max(self._peak_running, self._running)
                if t.result.started is None:
                    t.result.started = time.perf_counter()
            out, err = None, None
            try:
                out = t.fn()
            except Exception as e:  # recorded on the request; the loop keeps serving
                err = f"{type(e).__name__}: {e}"
            with self._cv:
                self._in_use -= t.mem - (t.keep if err is None else 0)
                self._running -= 1
                self._finish(t, out, err)

    def _finish(self, t: Task, out, err: Optional[str]):
        """Records a task's output (under the lock) and completes its request
        with its last task."""
        r = t.result
        if r.started is None:
            r.started = time.perf_counter()
        while len(r.outputs) <= t.index:
            r.outputs.append(None)
        r.outputs[t.index] = out
        if err and not r.error:
            r.error = err
        self._pending[r.rid] -= 1
        if self._pending[r.rid] == 0:
            r.done = time.perf_counter()
        self._cv.notify_all()

    def drain(self, timeout: Optional[float] = None) -> List[Result]:
        end = None if timeout is None else time.perf_counter() + timeout
        with self._cv:
            while any(v > 0 for v in self._pending.values()):
                left = None if end is None else end - time.perf_counter()
                if left is not None and left <= 0:
                    raise TimeoutError("requests still in flight")
                self._cv.wait(left)
            return list(self._results)

    def close(self):
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        for w in self._workers:
            w.join()

    @property
    def peak_in_use(self) -> int:
        return self._peak_in_use

    @property
    def in_use(self) -> int:
        return self._in_use

    @property
    def peak_running(self) -> int:
        return self._peak_running


# ---------------------------------------------------------------- load generation and statistics
def poisson_arrivals(rate: float, n: int, seed: int) -> np.ndarray:
    """Arrival offsets (seconds) of a seeded Poisson process of `rate` per second."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, n))


def run_arrivals(engine: Engine, requests: Sequence, offsets: Sequence[float]) -> Tuple[List[Result], float]:
    """Submits request i at start + offsets[i] (sleeping until then), waits
    for all, and returns the results and the makespan in seconds."""
    t0 = time.perf_counter()
    results = []
    for req, off in zip(requests, offsets):
        delay = t0 + off - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        results.append(engine.submit(req, arrival=t0 + off))
    engine.drain()
    return results, time.perf_counter() - t0


def summarize(results: Sequence[Result], makespan: float) -> dict:
    lat = np.array([r.latency for r in results]) * 1000.0
    opened = [r for r in results if r.kind == "OpenRequest"]
    return {
        "requests": len(results),
        "errors": sum(1 for r in results if r.error),
        "first_error": next((r.error for r in results if r.error), None),
        "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
        "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
        "mean_ms": float(lat.mean()) if len(lat) else None,
        "requests_per_s": len(results) / makespan,
        "openings_per_s": sum(len(r.outputs) for r in opened) / makespan,
        "weights_per_s": sum(r.weights for r in results) / makespan,
        "makespan_s": makespan,
    }


def random_points(params: Parameters, rng: np.random.Generator) -> bytes:
    """Fresh uniform extension-field coordinates for a single-matrix claim:
    canonical little-endian coefficients below the field's modulus."""
    (s,) = params.shapes
    coords = (max(s.rows - 1, 0).bit_length()) + (max(s.cols - 1, 0).bit_length())
    if params.field == FIELD_KOALABEAR:
        return rng.integers(0, 2130706433, coords * 4, dtype=np.uint64).astype("<u4").tobytes()
    return rng.integers(0, 65521, coords * 8).astype("<u2").tobytes()

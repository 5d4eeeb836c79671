"""QAFold commit+open throughput on B200: the 8B-shape batched workloads.

Workload (one step): commit every 2^30-entry PCS block of the 226-matrix
8B-shape collection and prove the benchmark claims, producing the
reference's proof bytes.  `--workload 8b8` (the default): int8 round(N(0,
20^2)) clipped to +-127 with 0.1% of entries forced to +-127, F65521^8,
chunk_log 30, packed_log 4.  `--workload 8b16`: the raw 16-bit payloads of
BF16 values drawn from N(0, 0.02^2) (the embedding from N(0, 1)),
KoalaBear^4, chunk_log 30, packed_log 4.  `--workload 70b16`: the 562 shapes
of the 70B set, BF16 payloads from N(0, 0.02^2) (141 GB), KoalaBear^4,
chunk_log 30, packed_log 6; the weights exceed HBM, so they stay in pinned
host memory and every pass streams them (the recompute mode,
Parameters.commit_recomputed), `--resident-gb` of leading blocks staying in
HBM after the first pass.  As in the reference
prover timer (main.rs:176-210) a step is commit + prove + serialisation;
setup and claim generation are outside it.  The claims are computed once
(their points derive from the committed roots, identical every step).

  value  : weights/s with the BVA already in HBM (Parameters.commit(on_device)).
  e2e    : weights/s through the same public API from a pinned host BVA
           (host->device copy of the weights and proof bytes back per step).
  per_matrix : the same statement and proof bytes with the weight passes
           launched one term / bucket / PCS block at a time (the per-matrix
           launch sequence) instead of once over all of them.
  separate_statements : the same 226 shapes, each committed and proven as
           its own single-matrix statement (its own proof).
  range_audit : the LogUp range audit of the same weights (Committed.range_audit),
           a check beside the proof, timed once outside the step.
  recompute : the same step in the reference's measured mode (--cache-mode
           recompute, Parameters.commit_recomputed): only the roots stay on
           the device and binding re-encodes every block; same proof bytes.

`--impl reference` times the CPU restatement of the reference prover (the
oracle; the Rust reference cannot be built in this image) with all host
threads on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
WEIGHTS_8B = 8_029_995_008


def shapes_8b():
    s = []
    for _ in range(32):
        s += [(4096, 4096), (1024, 4096), (1024, 4096), (4096, 4096), (14336, 4096), (14336, 4096), (4096, 14336)]
    return [(128256, 4096)] + s + [(128256, 4096)]


def shapes_70b():
    s = []
    for _ in range(80):
        s += [(8192, 8192), (1024, 8192), (1024, 8192), (8192, 8192), (28672, 8192), (28672, 8192), (8192, 28672)]
    return [(128256, 8192)] + s + [(128256, 8192)]


def make_bva_on_host(shapes, seed: int = 0, sigma: float = 0.02):
    """BF16 payloads of N(0, sigma^2) laid out as the BVA in pinned host memory,
    generated on the GPU one matrix at a time."""
    import torch
    from parcomm_b200 import layout

    buckets, active, _ = layout.buckets(shapes)
    # Page-locked by registration: torch's pinned allocator rounds a request up
    # to a power of two, which 141 GB does not survive.
    out = torch.empty(active, dtype=torch.int16)
    pinned = int(torch.cuda.cudart().cudaHostRegister(out.data_ptr(), out.numel() * 2, 0)) == 0
    by_matrix = {}
    for b in buckets:
        by_matrix.setdefault(b.matrix, []).append(b)
    covered = 0
    g = torch.Generator(device="cuda")
    for m, (rows, cols) in enumerate(shapes):
        g.manual_seed(seed * 100003 + m)
        w = torch.randn(rows * cols, generator=g, device="cuda", dtype=torch.float32)
        w = w.mul_(sigma).to(torch.bfloat16).view(torch.int16).view(rows, cols)
        for b in by_matrix[m]:
            blk = torch.zeros(b.rows, b.cols, dtype=torch.int16, device="cuda")
            blk[: b.physical_rows, : b.physical_cols] = w[b.row_offset: b.row_offset + b.physical_rows,
                                                         b.col_offset: b.col_offset + b.physical_cols]
            out[b.offset: b.offset + b.rows * b.cols].copy_(blk.view(-1))
            covered += b.rows * b.cols
            del blk
        del w
    assert covered == active
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return out, active, pinned


def force_extremes(w, n_forced: int, g):
    """Sets n_forced positions of the flat float tensor w, drawn with
    generator g, to -127 or +127.  A position drawn more than once takes its
    first draw's sign: a scatter with repeated indices would leave the winner
    unspecified, and the weights would differ between runs."""
    import torch
    idx = torch.randint(0, w.numel(), (n_forced,), generator=g, device=w.device)
    sign = torch.randint(0, 2, (n_forced,), generator=g, device=w.device).float().mul_(254.0).sub_(127.0)
    order = torch.sort(idx, stable=True).indices
    idx, sign = idx[order], sign[order]
    first = torch.ones_like(idx, dtype=torch.bool)
    first[1:] = idx[1:] != idx[:-1]
    w[idx[first]] = sign[first]


def make_bva_on_device(shapes, seed: int = 0, bf16: bool = False, embedding_first: bool = False):
    """Deterministic synthetic weights laid out as the BVA, generated on the GPU:
    int8 round(N(0, 20^2)) clipped to +-127 with 0.1% forced to +-127, or (bf16)
    the int16 bit patterns of BF16 values from N(0, 0.02^2), matrix 0 from N(0, 1)
    when `embedding_first`."""
    import torch
    from parcomm_b200 import layout

    buckets, active, _ = layout.buckets(shapes)
    out = torch.zeros(active, dtype=torch.int16 if bf16 else torch.int8, device="cuda")
    by_matrix = {}
    for b in buckets:
        by_matrix.setdefault(b.matrix, []).append(b)
    g = torch.Generator(device="cuda")
    for m, (rows, cols) in enumerate(shapes):
        g.manual_seed(seed * 100003 + m)
        w = torch.randn(rows * cols, generator=g, device="cuda", dtype=torch.float32)
        if bf16:
            sigma = 1.0 if (embedding_first and m == 0) else 0.02
            w = w.mul_(sigma).to(torch.bfloat16).view(torch.int16).view(rows, cols)
        else:
            w = w.mul_(20.0).round_().clamp_(-127, 127)
            n_forced = max(1, (rows * cols) // 1000)
            force_extremes(w, n_forced, g)
            w = w.to(torch.int8).view(rows, cols)
        for b in by_matrix[m]:
            dst = out[b.offset: b.offset + b.rows * b.cols].view(b.rows, b.cols)
            dst[: b.physical_rows, : b.physical_cols] = w[b.row_offset: b.row_offset + b.physical_rows,
                                                           b.col_offset: b.col_offset + b.physical_cols]
        del w
    torch.cuda.synchronize()
    return out, active


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, path: Path):
        self.path = path
        self.proc = None

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self, device_index: int = 0):
        if not self.path.exists():
            return None
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9 or parts[0] != str(device_index):
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d["hbm_gbs"], "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel: str, alg_bytes_per_launch: float, field: str = ""):
    """Per-launch DRAM bytes of `kernel`: the committed ncu capture's ratio of
    dram__bytes_read.sum + dram__bytes_write.sum to algorithmic bytes (taken
    on a smaller case of the same kernel and field), times this run's
    algorithmic bytes per launch; None without a capture."""
    p = ROOT / "profiles" / "ncu_traffic.json"
    if not p.exists():
        return None
    table = json.loads(p.read_text())
    d = table.get(f"{kernel}/{field}") if field else table.get(kernel)
    if not d:
        return None
    return d["dram_bytes_per_alg_byte"] * alg_bytes_per_launch


def step_alg_bytes(active: int, logical: int, chunk_log: int, packed_log: int, lanes: int, entry_bytes: int,
                   streamed: bool):
    """Compulsory bytes of one proof in this design's dataflow: every
    materialised vector is written once and read once per dependent pass.
    n = 2^chunk_log entries per block, m = n / lanes extension elements, s =
    2^packed_log.  Commit reads the weights and writes + reads (hashing) the
    2m-element codeword of each live block (and of one zero block, if any);
    the EO reads the weights twice and its 16 B vectors of N / s elements
    (rounds: 128 B per element over the geometric sum); projection and block
    fold read the weights once more; the folded table is committed; the
    sumcheck and the native top round read m-element vectors.  Binding
    re-encodes every block only for streamed weights (resident codewords stay
    in HBM).  Returns (total, per-stage)."""
    n = 1 << chunk_log
    m, s = n // lanes, 1 << packed_log
    live = -(-active // n)
    blocks = max(logical // n, 1)
    zero = 1 if live < blocks else 0
    w = entry_bytes
    terms = {
        "commit": (live + zero) * n * (w + 64 / lanes),
        "eo_cross": active * w,
        "eo_witness": active * w + 16 * logical / s,
        "eo_query_fold": 16 * logical / s,
        "eo_rounds": 128 * logical / s,
        "projection": live * n * w + 32 * m,
        "block_fold": live * n * w + 16 * m,
        "folded_commit": 16 * m + 64 * n / lanes,
        "sumcheck": 128 * m,
        "binding": (live + zero) * n * (w + 64 / lanes) if streamed else 0,
        "native_top_round": 32 * m,
    }
    return sum(terms.values()), terms


def max_over_ranks(ms: float, world: int, device: str = "cuda") -> float:
    """Step time of the slowest rank (every rank calls this collectively)."""
    if world <= 1:
        return ms
    import torch
    import torch.distributed as dist

    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def measure_h2d_gbs(nbytes: int = 1 << 31, reps: int = 3) -> float:
    """Pinned host -> device copy bandwidth (best of `reps` copies of 2 GiB),
    the bound of a workload streamed from host memory."""
    import torch
    src = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    dst = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    best = 0.0
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        dst.copy_(src, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, nbytes / (e0.elapsed_time(e1) / 1000.0) / 1e9)
    del src, dst
    torch.cuda.empty_cache()
    return best


def job_throughput(weights_per_rank: int, world: int, ms_per_step: float) -> float:
    """Whole-job weights/s: every rank proves its own model of `weights_per_rank`."""
    return weights_per_rank * world / (ms_per_step / 1000.0)


def per_matrix_path(qf, shapes, seed_base: int, field: int, bf16: bool):
    """The plain per-matrix path: every matrix committed and proven as its own
    single-matrix statement (its own layout, parameters and proof), one after
    another, through the same library.  Returns (timed seconds of one pass over
    all matrices, setup seconds).  Parameters (setup) and each matrix's claims
    are made once, outside the timed pass, as in the batched path; that
    preparation pass also warms the kernels up."""
    import torch

    t0 = time.time()
    params = {}
    for s in shapes:
        if s not in params:
            params[s] = qf.Parameters([s], qf.Config(30, 4), field=field)
    setup_s = time.time() - t0
    jobs = []
    for m, s in enumerate(shapes):
        bva, _ = make_bva_on_device([s], seed=seed_base + m, bf16=bf16, embedding_first=bf16 and m == 0)
        p = params[s]
        c = p.commit(bva, on_device=True)
        claims = p.evaluate_claims(c, p.benchmark_points(c.roots))
        proof, _ = p.prove(c, claims)
        c.close()
        jobs.append((p, bva, claims))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for p, bva, claims in jobs:
        c = p.commit(bva, on_device=True)
        p.prove(c, claims)
        c.close()
    torch.cuda.synchronize()
    return time.perf_counter() - t0, setup_s


def int8_matrix(rows: int, cols: int, seed: int):
    """int8 round(N(0, 20^2)) clipped to +-127 with 0.1% forced to +-127, on the GPU."""
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    w = torch.randn(rows * cols, generator=g, device="cuda", dtype=torch.float32).mul_(20.0).round_().clamp_(-127, 127)
    force_extremes(w, max(1, (rows * cols) // 1000), g)
    return w.to(torch.int8).view(rows, cols)


def run_serve(args):
    """The serving loop: a device-resident pool of the 8B-shape 8-bit set
    (226 single-matrix commitments in cache mode: weights, codewords and
    trees resident) and the 70B-shape 8-bit set (562 single-matrix
    commitments in recompute mode: weights resident, each opening re-encodes;
    F65521^8, packed_log 6).  Seeded Poisson arrivals per rate: 90% opening
    requests of 1-64 random pooled matrices at fresh uniform points, 10%
    commits of new int8 matrices (1024-28672 rows x 4096 or 8192 columns).
    Each rate runs the same requests twice: through the engine (continuous
    batching over --slots workers under the HBM budget) and one plain
    request at a time.  Prints one JSON line."""
    import numpy as np
    import torch
    import parcomm_b200 as qf
    from parcomm_b200 import serving
    from parcomm_b200.build import build

    build()
    torch.cuda.set_device(0)
    t0 = time.time()
    pool = serving.Pool()
    sets = [("8B-shape 8-bit", shapes_8b(), qf.Config(30, 4), False),
            ("70B-shape 8-bit", shapes_70b(), qf.Config(30, 6), True)]
    if args.serve_scale < 1.0:  # a subset of each set, for quick runs
        sets = [(n, sh[:max(1, int(len(sh) * args.serve_scale))], c, r) for n, sh, c, r in sets]
    pool_weights = 0
    for si, (_, shapes, cfg, recompute) in enumerate(sets):
        for m, (r, c) in enumerate(shapes):
            pool.commit(int8_matrix(r, c, 1000 * si + m), cfg, recompute)
            pool_weights += r * c
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    load_s = time.time() - t0
    # The engine budgets HBM itself: bound the library's cache of released
    # buffers and keep it, plus headroom for torch, outside the budget.
    cache = 16 << 30
    qf.device_cache_limit(cache)
    free_b, total_b = torch.cuda.mem_get_info()
    budget = int(free_b - cache - (8 << 30))
    keys = pool.keys()

    def make_requests(n, seed):
        rng = np.random.default_rng(seed)
        out = []
        for k in range(n):
            if rng.random() < 0.1:
                rows, cols = int(rng.integers(1024, 28673)), int(rng.choice([4096, 8192]))
                out.append(serving.CommitRequest(int8_matrix(rows, cols, 777_000 + seed * 1000 + k), qf.Config(30, 4), True))
            else:
                pick = list(rng.choice(keys, size=min(len(keys), int(rng.integers(1, 65))), replace=False))
                out.append(serving.OpenRequest(pick, [serving.random_points(pool.get(m).params, rng) for m in pick]))
        return out

    # Warm-up: one request of each kind through the engine.
    eng = serving.Engine(pool, slots=args.slots, hbm_budget=budget)
    for q in make_requests(4, 12345):
        eng.submit(q)
    eng.drain()
    eng.close()
    rates = []
    for ri, rate in enumerate(args.serve_rates):
        reqs = make_requests(args.serve_requests, 100 + ri)
        offsets = serving.poisson_arrivals(rate, len(reqs), args.serve_seed + ri)
        row = {"rate_per_s": rate}
        for name, slots in (("engine", args.slots), ("one_at_a_time", 1)):
            eng = serving.Engine(pool, slots=slots, hbm_budget=budget)
            res, span = serving.run_arrivals(eng, reqs, offsets)
            eng.close()
            row[name] = serving.summarize(res, span)
            row[name]["peak_tasks_in_flight"] = eng.peak_running
        row["p99_speedup"] = row["one_at_a_time"]["p99_ms"] / row["engine"]["p99_ms"]
        rates.append(row)
        print(json.dumps({"progress": row}), file=sys.stderr)
    line = {
        "metric": "QAFold serving: opening latency p50/p99 and throughput under Poisson load",
        "unit": "ms (latency), weights/s and requests/s (throughput)",
        "n_gpus": 1,
        "data": "synthetic",
        "dtype": "int8",
        "config": {"workload": "serving loop (C5)", "pool": [n for n, *_ in sets], "pool_matrices": len(pool),
                   "pool_weights": pool_weights, "field": "F65521^8", "slots": args.slots,
                   "hbm_budget_bytes": budget, "device_cache_limit_bytes": cache,
                   "requests_per_rate": args.serve_requests,
                   "open": "1-64 random pooled matrices, fresh uniform points, one proof each (qf_open)",
                   "commit": "10%: new int8 matrix, 1024-28672 rows x 4096/8192 cols, recompute mode",
                   "scale": args.serve_scale},
        "load_s": load_s,
        "rates": rates,
    }
    print(json.dumps(line))


def run_reference(args):
    """CPU restatement of the reference prover on a bounded sample of the workload."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import numpy as np
    import oracle
    from parcomm_b200 import layout

    # One decoder layer's attention projections (4 matrices, 41.9M weights),
    # chunk_log 24 so the sample keeps the batched multi-block opening.
    shapes = [(4096, 4096), (1024, 4096), (1024, 4096), (4096, 4096)]
    sixteen = args.workload in ("8b16", "layers16", "70b16")
    field = "koalabear" if sixteen else "f65521"
    packed_log = 6 if args.workload == "70b16" else 4
    chunk_log = 24
    if args.workload == "70b16":  # one 70B decoder layer's attention projections
        shapes = [(8192, 8192), (1024, 8192), (1024, 8192)]
    elif args.workload == "smoke":  # the whole smoke configuration
        shapes, chunk_log = [(1024, 4096)], 20
    rng = np.random.default_rng(0)
    mats = []
    for r, c in shapes:
        if sixteen:
            f = rng.normal(0, 0.02, r * c).astype(np.float32)
            # BF16 bit pattern: the high half of the f32 word, rounded to nearest even.
            u = f.view(np.uint32).astype(np.uint64)
            u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
            w = u.astype(np.uint16).view(np.int16)
        else:
            w = np.clip(np.rint(rng.normal(0, 20, r * c)), -127, 127).astype(np.int8)
            idx = rng.choice(r * c, (r * c) // 1000, replace=False)
            w[idx] = np.where(rng.random(idx.size) < 0.5, -127, 127)
        mats.append(w.reshape(r, c))
    bva = layout.encode(shapes, mats)
    weights = sum(r * c for r, c in shapes)
    threads = os.cpu_count() or 1
    times = []
    for step in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        roots, claims, proof, (commit_ms, open_ms) = oracle.prove(shapes, chunk_log, packed_log, bva, field=field)
        dt = time.perf_counter() - t0
        if step >= args.warmup:
            times.append((commit_ms + open_ms) / 1000.0)
    sec = statistics.mean(times)
    value = weights / sec
    layer = {"70b16": "3 matrices of one 70B decoder layer (q,k,v", "smoke": "the whole smoke workload (1024x4096"}.get(
        args.workload, "4 matrices of one 8B decoder layer (q,k,v,o")
    sample = (f"{layer}: {weights} "
              f"{'BF16 payloads' if sixteen else 'int8 weights'}), chunk_log {chunk_log}, packed_log {packed_log}, "
              f"C++ restatement of the reference CPU prover (OpenMP, {threads} threads)")
    line = {
        "impl": "reference", "metric": "QAFold commit+open weights/s", "value": value, "unit": "weights/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1000.0,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int16" if sixteen else "int8",
        "data": "synthetic", "config": {"workload": {"70b16": "70B-shape 16-bit weights, streamed (sample)",
                                                     "smoke": "smoke 1024x4096 int8"}.get(
                                            args.workload, f"8B-shape {16 if sixteen else 8}-bit weights, batched (sample)"),
                                        "field": "KoalaBear^4" if sixteen else "F65521^8",
                                        "chunk_log": chunk_log, "packed_log": packed_log, "sample": sample},
        "cpu_baseline": {"value": value, "unit": "weights/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "weights/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="8b8",
                    choices=["8b8", "8b16", "70b16", "layers", "layers16", "layers70", "smoke", "serve"],
                    help="8b8 / 8b16: the 8B shape set with 8-bit weights (F65521^8) or 16-bit BF16 "
                         "payloads (KoalaBear^4); layers / layers16: the first --layers transformer layers "
                         "(7 matrices each) at --chunk-log, a small case for profiling")
    ap.add_argument("--layers", type=int, default=2)
    ap.add_argument("--slots", type=int, default=8, help="serve: concurrent tasks")
    ap.add_argument("--serve-rates", type=float, nargs="+", default=[1.0, 5.0, 20.0, 50.0])
    ap.add_argument("--serve-requests", type=int, default=10, help="serve: requests per rate")
    ap.add_argument("--serve-seed", type=int, default=0)
    ap.add_argument("--serve-scale", type=float, default=1.0, help="serve: fraction of each pool set to load")
    ap.add_argument("--resident-gb", type=float, default=None,
                    help="70b16 / layers70: GB of leading weight blocks kept in HBM after the first streamed pass "
                         "(default: what free HBM allows next to the proof's own peak)")
    ap.add_argument("--chunk-log", type=int, default=28)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-per-matrix", action="store_true",
                    help="skip the per-matrix comparison (each matrix proven on its own)")
    ap.add_argument("--no-audit", action="store_true", help="skip the LogUp range audit measurement")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip the same-bytes comparisons (dp4a kernels, per-matrix launch sequence)")
    ap.add_argument("--no-recompute", action="store_true",
                    help="skip the recompute-mode measurement (the reference's --cache-mode recompute)")
    ap.add_argument("--profile-range", action="store_true",
                    help="bracket the device-resident timed steps with cudaProfilerStart/Stop "
                         "(for ncu --profile-from-start off)")
    ap.add_argument("--out", default=str(ROOT / "bench_out"), help="directory for the clock samples and kernel stats")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload == "serve":
        if rank == 0:
            run_serve(args)
        return
    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return

    import torch
    import parcomm_b200 as qf
    from parcomm_b200.build import build

    build()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    sixteen = args.workload in ("8b16", "layers16", "70b16", "layers70")
    streamed = args.workload in ("70b16", "layers70")
    field = qf.FIELD_KOALABEAR if sixteen else qf.FIELD_F65521
    bits = 16 if sixteen else 8
    if args.workload in ("8b8", "8b16"):
        shapes, cfg, name = shapes_8b(), qf.Config(30, 4), f"8B-shape {bits}-bit weights, batched (226 matrices)"
    elif args.workload == "70b16":
        shapes, cfg = shapes_70b(), qf.Config(30, 6)
        name = "70B-shape 16-bit weights, streamed from pinned host memory (562 matrices)"
    elif args.workload == "layers70":
        shapes, cfg = shapes_70b()[1:1 + 7 * args.layers], qf.Config(args.chunk_log, 6)
        name = f"70B-shape 16-bit weights, first {args.layers} layers, chunk 2^{args.chunk_log}, streamed"
    elif args.workload in ("layers", "layers16"):
        shapes = shapes_8b()[1:1 + 7 * args.layers]
        cfg = qf.Config(args.chunk_log, 4)
        name = f"8B-shape {bits}-bit weights, first {args.layers} layers, chunk 2^{args.chunk_log}"
    else:
        shapes, cfg, name = [(1024, 4096)], qf.Config(20, 4), "smoke 1024x4096 int8"
    weights = sum(r * c for r, c in shapes)

    t0 = time.time()
    params = qf.Parameters(shapes, cfg, field=field)
    setup_s = time.time() - t0
    t0 = time.time()
    host_pinned = True
    if streamed:
        bva_host, active, host_pinned = make_bva_on_host(shapes, seed=rank)
        bva_dev = None
        resident = None if args.resident_gb is None else int(args.resident_gb * 1e9)

        def commit(on_device: bool):
            return params.commit_recomputed(bva_host, resident_bytes=resident)
    else:
        bva_dev, active = make_bva_on_device(shapes, seed=rank, bf16=sixteen, embedding_first=args.workload == "8b16")
        bva_host = torch.empty(active, dtype=bva_dev.dtype, pin_memory=True)
        bva_host.copy_(bva_dev)

        def commit(on_device: bool):
            return params.commit(bva_dev if on_device else bva_host, on_device=on_device)
    entry_bytes = bva_host.element_size()
    input_s = time.time() - t0

    # Claims once: their points derive from the (step-invariant) roots.
    c = commit(True)
    claims = params.evaluate_claims(c, params.benchmark_points(c.roots))
    proof, prof = params.prove(c, claims)
    c.close()
    verify_s = None
    if rank == 0:
        t0 = time.time()
        params.verify(c.roots, claims, proof)
        verify_s = time.time() - t0
    proof_bytes = len(proof.to_bytes())

    res_blocks = [0, 0]

    def step(on_device: bool, commit_fn=None):
        cc = (commit_fn or commit)(on_device)
        pr, pf = params.prove(cc, claims)
        if streamed:
            h2d, res_blocks[0], res_blocks[1] = cc.stream_info()
        elif commit_fn is not None:  # recompute mode: the copies the stream made (none for device weights)
            h2d = cc.stream_info()[0]
        else:
            h2d = 0 if on_device else active * entry_bytes
        cc.close()
        return pr, pf, h2d

    for _ in range(max(args.warmup - 1, 0)):
        step(True)

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def timed(on_device: bool, steps: int, commit_fn=None):
        barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        launches0 = qf.kernel_launches()
        profiled = args.profile_range and on_device and commit_fn is None
        if profiled:  # a profiler started with its capture off records only this region
            torch.cuda.profiler.start()
        ev0.record()
        last = None
        for _ in range(steps):
            last = step(on_device, commit_fn)
        ev1.record()
        barrier()
        if profiled:
            torch.cuda.profiler.stop()
        ms = max_over_ranks(ev0.elapsed_time(ev1), world)
        return ms / steps, last, qf.kernel_launches() - launches0

    out_dir = Path(args.out)
    out_dir.mkdir(exist_ok=True)
    with ClockSampler(out_dir / "bench_clocks.csv") as clocks:
        ms_dev, (pr_dev, pf_dev, h2d_dev), launches = timed(True, args.steps)
    if streamed:  # the weights only exist in host memory: the timed run is already end to end
        ms_e2e, pr_e2e, h2d_e2e = ms_dev, pr_dev, h2d_dev
    else:
        ms_e2e, (pr_e2e, pf_e2e, h2d_e2e), _ = timed(False, max(1, args.steps))
    assert pr_dev.to_bytes() == proof.to_bytes() == pr_e2e.to_bytes(), "proof bytes changed between steps"

    # The reference's measured mode (--cache-mode recompute): only the roots
    # stay on the device after the commit, and binding re-encodes every block
    # and checks its root (qafold_short_batch.rs:118-160).  Same weights, same
    # claims, same proof bytes; timed the same way, after its own warm-up.
    recompute = None
    if not args.no_recompute and not streamed:
        def commit_rc(on_device: bool):
            return params.commit_recomputed(bva_dev if on_device else bva_host, resident_bytes=None)

        for _ in range(max(args.warmup, 1)):
            step(True, commit_rc)
        ms_rc, (pr_rc, pf_rc, _), _ = timed(True, args.steps, commit_rc)
        ms_rc_e2e, (pr_rc_e2e, _, h2d_rc), _ = timed(False, max(1, args.steps), commit_rc)
        assert pr_rc.to_bytes() == proof.to_bytes() == pr_rc_e2e.to_bytes(), "recompute-mode proof bytes differ"
        rc_alg, rc_terms = step_alg_bytes(active, params.logical, cfg.chunk_log, cfg.packed_log, 4 if sixteen else 8,
                                          entry_bytes, True)
        recompute = {
            "value": job_throughput(weights, world, ms_rc), "unit": "weights/s", "ms_per_step": ms_rc,
            "e2e": {"value": job_throughput(weights, world, ms_rc_e2e), "unit": "weights/s", "ms_per_step": ms_rc_e2e,
                    "h2d_bytes_per_step": h2d_rc, "d2h_bytes_per_step": len(pr_rc.to_bytes())},
            "stage_ms": {k: getattr(pf_rc, k) for k in ("commit_ms", "eo_ms", "projection_ms", "folding_ms",
                                                       "sumcheck_ms", "binding_ms", "native_opening_ms", "decide_ms",
                                                       "open_ms")},
            "step_alg_bytes": rc_alg, "binding_alg_gb": round(rc_terms["binding"] / 1e9, 2),
            "what": "Parameters.commit_recomputed over the same weights (device-resident for value, pinned host "
                    "memory for e2e): only roots kept, binding re-encodes and root-checks every block; proof bytes "
                    "identical to the cache-mode step"}

    # Per-kernel device time (CUDA events on each launch's own stream), one extra step.
    qf.kernel_timing(True)
    step(True)
    torch.cuda.synchronize()
    stats = qf.kernel_stats()
    qf.kernel_timing(False)
    # "host:<section>" entries are host wall-clock sections and "_gaps" the idle
    # time between launches, not kernels.
    dominant = max((k for k in stats if not k.startswith(("host:", "_"))), key=lambda k: stats[k]["ms"])
    d = stats[dominant]
    achieved = d["bytes"] / (d["ms"] / 1000.0) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = ncu_traffic(dominant, d["bytes"] / d["launches"], "koalabear" if sixteen else "")

    alg_total, alg_terms = step_alg_bytes(active, params.logical, cfg.chunk_log, cfg.packed_log,
                                          4 if sixteen else 8, entry_bytes, streamed)
    # Integer roofline: the measured issue peaks (microbenchmark) against the
    # algorithmic integer operations the library counts per launch.
    int_peaks = qf.int_peaks()
    issue_peak = int_peaks["issue_ops_per_s"]
    kernel_stats = {k: v for k, v in stats.items() if not k.startswith(("host:", "_"))}
    step_ops = sum(v.get("ops", 0) for v in kernel_stats.values())
    counted_ms = sum(v["ms"] for v in kernel_stats.values() if v.get("ops", 0))
    hbm_frac = alg_total / (ms_dev / 1000.0) / 1e9 / peak
    alu_frac = step_ops / (ms_dev / 1000.0) / issue_peak
    step_roofline = {"bound": "hbm", "alg_bytes": alg_total, "achieved": alg_total / (ms_dev / 1000.0) / 1e9,
                     "peak": peak, "unit": "GB/s", "frac": hbm_frac,
                     "peak_source": peak_kind, "terms_gb": {k: round(v / 1e9, 2) for k, v in alg_terms.items()},
                     "alu": {"alg_ops": step_ops, "achieved_ops_per_s": step_ops / (ms_dev / 1000.0),
                             "peak_ops_per_s": issue_peak, "frac": alu_frac, "counted_kernel_ms": counted_ms,
                             "what": "integer operations the arithmetic needs (transform butterflies, reductions, "
                                     "extension products, BLAKE2s compressions) in the kernels that count them, over "
                                     "the step time, against the measured issue peak of both integer pipes"},
                     "max_frac": max(hbm_frac, alu_frac), "max_bound": "alu" if alu_frac > hbm_frac else "hbm",
                     "what": "the whole step's compulsory bytes (each materialised vector written once, read once "
                             "per dependent pass) and counted integer operations over its time"}

    link = None
    if streamed:  # the host link bounds a streamed step: bytes copied per step against a measured copy
        h2d_peak = measure_h2d_gbs()
        h2d_achieved = h2d_dev / (ms_dev / 1000.0) / 1e9
        link = {"bound": "h2d", "achieved": h2d_achieved, "peak": h2d_peak, "unit": "GB/s",
                "frac": h2d_achieved / h2d_peak, "bytes_per_step": h2d_dev,
                "peak_source": "pinned 2 GiB host->device copy, best of 3, measured in this run"}

    # The exact integer-limb tensor-core forms of the weight passes against
    # the dp4a / IMAD kernels the library runs (F65521): one more profiled
    # step with them switched on, same bytes.
    imma_cmp = None
    if not sixteen and not args.no_compare:
        qf.kernel_option("imma", 1)
        qf.kernel_timing(True)
        pr_on, _, _ = step(True)
        torch.cuda.synchronize()
        on_stats = qf.kernel_stats()
        qf.kernel_timing(False)
        qf.kernel_option("imma", 0)
        assert pr_on.to_bytes() == proof.to_bytes(), "tensor-core path proof bytes differ"
        off = stats
        pairs = {"eo_witness": ("k_eo_witness_mma", "k_eo_witness"), "block_fold": ("k_block_fold_mma", "k_block_fold"),
                 "eq_projection": ("k_eq_project_mma", "k_eq_project_blocks")}
        imma_cmp = {}
        for name, (on_k, off_k) in pairs.items():
            a, b = on_stats.get(on_k), off.get(off_k)
            if a and b:
                imma_cmp[name] = {"imma_ms": a["ms"], "dp4a_ms": b["ms"], "speedup": b["ms"] / a["ms"],
                                  "imma_hbm_frac": a["bytes"] / (a["ms"] / 1000.0) / 1e9 / peak,
                                  "dp4a_hbm_frac": b["bytes"] / (b["ms"] / 1000.0) / 1e9 / peak}
        imma_cmp["what"] = ("per-step kernel time of the exact integer-limb tensor-core kernels (mma.sync s8 x u8 -> "
                            "s32) against the dp4a / IMAD kernels, same proof bytes")

    # The extension-product sums of the EO, sumcheck and LiteBullet rounds on
    # the tensor cores against the CUDA-core kernels: two more profiled steps,
    # all kernels one way and then the other (core_dots 2 and 1), same bytes
    # (both fields).  The library's default takes, per kernel, the faster one.
    dots_cmp = None
    if not args.no_compare:
        runs = {}
        for mode in (2, 1):
            qf.kernel_option("core_dots", mode)
            qf.kernel_timing(True)
            pr_cd, _, _ = step(True)
            torch.cuda.synchronize()
            runs[mode] = qf.kernel_stats()
            qf.kernel_timing(False)
            assert pr_cd.to_bytes() == proof.to_bytes(), "product-sum path proof bytes differ"
        qf.kernel_option("core_dots", 0)
        dots_cmp = {}
        tc_ms = cc_ms = 0.0
        for k in ("k_eo_dot_cross", "k_eo_fold_query_cross", "k_eo_fold_cross", "k_sum_message", "k_sum_fold_message",
                  "k_lb_cross", "k_lb_fold_cross", "k_dot"):
            a, b = runs[2].get(k + "_mma"), runs[1].get(k)
            if a and b:
                dots_cmp[k] = {"tensor_ms": a["ms"], "cuda_core_ms": b["ms"], "speedup": b["ms"] / a["ms"],
                               "tensor_hbm_frac": a["bytes"] / (a["ms"] / 1000.0) / 1e9 / peak,
                               "cuda_core_hbm_frac": b["bytes"] / (b["ms"] / 1000.0) / 1e9 / peak,
                               "default": "tensor" if (k + "_mma") in stats else "cuda_core"}
                tc_ms += a["ms"]
                cc_ms += b["ms"]
        dots_cmp["total"] = {"tensor_ms": tc_ms, "cuda_core_ms": cc_ms}
        dots_cmp["what"] = ("per-step kernel time of the exact integer-limb tensor-core product sums (mma.sync u8 x u8 -> "
                            "s32 over the elements' storage bytes) against the CUDA-core 64-bit multiply-add kernels, "
                            "same proof bytes; 'default' is the library's choice for the kernel")

    # The same statement with the weight passes issued one launch per term,
    # bucket or block (the per-matrix launch sequence) instead of one launch
    # over all of them: same bytes, timed the same way.
    per_matrix_launches = None
    if not args.no_compare and not streamed:
        qf.kernel_option("per_matrix", 1)
        step(True)
        ms_pm, (pr_pm, _, _), launches_pm = timed(True, args.steps)
        qf.kernel_option("per_matrix", 0)
        assert pr_pm.to_bytes() == proof.to_bytes(), "per-matrix launch sequence proof bytes differ"
        per_matrix_launches = {"value": job_throughput(weights, world, ms_pm), "unit": "weights/s", "ms_per_step": ms_pm,
                               "gpu_launches": launches_pm // max(args.steps, 1),
                               "batched_over_per_matrix": ms_pm / ms_dev,
                               "what": "the same proof (identical bytes) with the weight passes launched per term, "
                                       "bucket or PCS block instead of once over all of them"}

    # LogUp range audit of the same weights (beside the proof, outside the
    # timed region): one warm-up call, then one timed call.
    range_audit = None
    if not args.no_audit and not streamed:
        ca = commit(True)
        ca.range_audit()
        torch.cuda.synchronize()
        qf.kernel_timing(True)
        t0 = time.perf_counter()
        ra = ca.range_audit()
        audit_s = time.perf_counter() - t0
        ks = qf.kernel_stats().get("k_range_audit", {})
        qf.kernel_timing(False)
        ca.close()
        k_ms = ks.get("ms")
        range_audit = {
            "holds": ra.holds, "values": active, "ms": audit_s * 1000.0, "values_per_s": active / audit_s,
            "kernel_ms": k_ms, "kernel_launches": ks.get("launches"),
            "kernel_values_per_s": active / (k_ms / 1000.0) if k_ms else None,
            "kernel_hbm_frac": (active * entry_bytes / (k_ms / 1000.0) / 1e9) / peak if k_ms else None,
            "nonzero_bins": int((ra.multiplicities > 0).sum()),
            "what": "LogUp range audit beside the proof (never in it): per-value fraction sum and multiplicities "
                    "on the device, the table side on the host"}

    per_matrix = None
    if not args.no_per_matrix and args.workload in ("8b8", "8b16"):
        del bva_host
        pm_s, pm_setup = per_matrix_path(qf, [(r, c) for r, c in shapes], 1_000_003 * (rank + 1), field, sixteen)
        pm_ms = max_over_ranks(pm_s * 1000.0, world)
        per_matrix = {"value": job_throughput(weights, world, pm_ms), "unit": "weights/s", "ms_per_pass": pm_ms,
                      "proofs_per_pass": len(shapes), "setup_s": pm_setup,
                      "batched_over_per_matrix": pm_ms / ms_dev,
                      "how": "each of the 226 matrices committed and proven as its own single-matrix statement, "
                             "one after another (device-resident weights); one timed pass after a preparation "
                             "pass that makes the claims"}

    if world > 1:
        torch.distributed.destroy_process_group()
    if rank != 0:
        return
    cpu_baseline = None
    if not args.no_cpu_baseline:
        try:
            r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                                "--warmup", "0", "--workload", args.workload], capture_output=True, text=True,
                               timeout=900)
            cpu_baseline = json.loads(r.stdout.strip().splitlines()[-1])["cpu_baseline"]
        except Exception as e:  # reported, not fatal
            cpu_baseline = {"error": str(e)[:200]}
    value = job_throughput(weights, world, ms_dev)
    line = {
        "metric": "QAFold commit+open weights/s",
        "value": value,
        "unit": "weights/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_dev,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "int16" if sixteen else "int8",
        "data": "synthetic",
        "config": {"workload": name, "field": "KoalaBear^4" if sixteen else "F65521^8", "chunk_log": cfg.chunk_log,
                   "packed_log": cfg.packed_log, "weights": weights, "active_entries": active, "pcs_blocks": params.blocks,
                   "l2": "inputs larger than L2 (BVA of 8 to 141 GB, 4 or 8 GiB codeword per block)",
                   "weights_in": (("pinned" if host_pinned else "pageable") + " host memory, streamed per pass, "
                                  + (f"{args.resident_gb} GB of blocks resident" if args.resident_gb is not None
                                     else f"{res_blocks[0]} of {res_blocks[1]} live blocks resident (auto)")
                                  if streamed else "HBM (value); pinned host memory (e2e)"),
                   "parallelism": "replicas" if world > 1 else "single"},
        "e2e": {"value": job_throughput(weights, world, ms_e2e), "unit": "weights/s",
                "h2d_bytes_per_step": h2d_e2e, "d2h_bytes_per_step": proof_bytes},
        "gpu_launches": launches // max(args.steps, 1),
        "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "traffic": traffic, "kernel_ms_per_step": d["ms"], "kernel_launches": d["launches"],
                     "alg_bytes_per_launch": d["bytes"] / max(d["launches"], 1),
                     "alu": ({"alg_ops_per_launch": d["ops"] / max(d["launches"], 1),
                              "achieved_ops_per_s": d["ops"] / (d["ms"] / 1000.0), "peak_ops_per_s": issue_peak,
                              "frac": d["ops"] / (d["ms"] / 1000.0) / issue_peak, "peak_source": "measured in this run"}
                             if d.get("ops") else None)},
        "int_peaks": int_peaks,
        "kernels": {k: {"launches": v["launches"], "ms": round(v["ms"], 3),
                        "hbm_frac": round(v["bytes"] / (v["ms"] / 1000.0) / 1e9 / peak, 3) if v["ms"] > 0 else None,
                        "alu_frac": (round(v["ops"] / (v["ms"] / 1000.0) / issue_peak, 3)
                                     if v.get("ops") and v["ms"] > 0 else None)}
                    for k, v in sorted(kernel_stats.items(), key=lambda kv: -kv[1]["ms"])[:14]},
        "step_roofline": step_roofline,
        "link_roofline": link,
        "cpu_baseline": cpu_baseline,
        "per_matrix": per_matrix_launches,
        "separate_statements": per_matrix,
        "recompute": recompute,
        "imma_vs_dp4a": imma_cmp,
        "tensor_vs_cuda_core_products": dots_cmp,
        "range_audit": range_audit,
        "clocks": clocks.summary(local),
        "proof_bytes": proof_bytes,
        "stage_ms": {k: getattr(pf_dev, k) for k in ("commit_ms", "eo_ms", "projection_ms", "folding_ms", "sumcheck_ms",
                                                     "binding_ms", "native_opening_ms", "decide_ms", "open_ms")},
        "setup_s": setup_s,
        "input_s": input_s,
        "verify_s": verify_s,
    }
    (out_dir / "bench_kernels.json").write_text(json.dumps(stats, indent=1))
    print(json.dumps(line))


if __name__ == "__main__":
    main()

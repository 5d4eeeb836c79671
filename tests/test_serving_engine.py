"""The serving engine's scheduling on the CPU: fake tasks stand in for the
GPU calls (slots, strict FIFO admission under an HBM budget, continuous
batching of late arrivals, memory kept by commitments, the exhaustion guard,
Poisson load and its statistics)."""
import threading
import time

import numpy as np
import pytest

from parcomm_b200 import serving


class Fake:
    """A request of `n` tasks, each sleeping `sec` and claiming `mem` bytes
    (`keep` of them after it succeeds); `fail` makes task 0 raise."""

    def __init__(self, n=1, sec=0.01, mem=0, keep=0, fail=False, tag=None):
        self.n, self.sec, self.mem, self.keep, self.fail, self.tag = n, sec, mem, keep, fail, tag


def fake_tasks(log):
    lock = threading.Lock()

    def make(req, result):
        tasks = []
        for i in range(req.n):
            def run(i=i, req=req):
                with lock:
                    log.append(("start", req.tag, i, time.perf_counter()))
                time.sleep(req.sec)
                if req.fail and i == 0:
                    raise RuntimeError("planted")
                with lock:
                    log.append(("end", req.tag, i, time.perf_counter()))
                return (req.tag, i)
            tasks.append(serving.Task(result, i, req.mem, run, 1, req.keep))
        return tasks
    return make


def test_slots_bound_concurrency_and_outputs_keep_task_order():
    log = []
    eng = serving.Engine(None, slots=3, make_tasks=fake_tasks(log))
    rs = [eng.submit(Fake(n=5, sec=0.01, tag=k)) for k in range(4)]
    eng.drain(timeout=30)
    eng.close()
    assert eng.peak_running <= 3
    for k, r in enumerate(rs):
        assert r.error is None and r.outputs == [(k, i) for i in range(5)]
        assert r.done >= r.started >= r.arrival


def test_budget_is_never_exceeded_and_oversized_tasks_are_refused():
    log = []
    eng = serving.Engine(None, slots=8, hbm_budget=100, make_tasks=fake_tasks(log))
    for _ in range(6):
        eng.submit(Fake(n=4, sec=0.005, mem=30))
    eng.drain(timeout=30)
    assert eng.peak_in_use <= 100 and eng.peak_running <= 3
    with pytest.raises(Exception):
        eng.submit(Fake(n=1, mem=101))
    eng.close()


def test_late_arrivals_are_admitted_while_earlier_requests_run():
    """Continuous batching: a short request arriving after a long one starts
    on a free slot and finishes first; a slot-by-slot queue of whole requests
    would make it wait."""
    log = []
    eng = serving.Engine(None, slots=2, make_tasks=fake_tasks(log))
    long = eng.submit(Fake(n=1, sec=0.3, tag="long"))
    time.sleep(0.02)
    short = eng.submit(Fake(n=2, sec=0.01, tag="short"))
    eng.drain(timeout=30)
    eng.close()
    assert short.done < long.done
    assert short.started < long.done


def test_strict_fifo_head_waits_for_memory():
    """A big head task waits until memory frees, and later small tasks do not
    overtake it."""
    log = []
    eng = serving.Engine(None, slots=4, hbm_budget=100, make_tasks=fake_tasks(log))
    a = eng.submit(Fake(n=1, sec=0.1, mem=60, tag="a"))
    time.sleep(0.01)
    b = eng.submit(Fake(n=1, sec=0.01, mem=60, tag="b"))
    c = eng.submit(Fake(n=1, sec=0.01, mem=10, tag="c"))
    eng.drain(timeout=30)
    eng.close()
    starts = {tag: t for kind, tag, _, t in log if kind == "start"}
    assert starts["b"] >= a.done - 1e-3 and starts["c"] >= starts["b"]


def test_commitments_keep_memory_and_exhaustion_fails_instead_of_waiting():
    log = []
    eng = serving.Engine(None, slots=2, hbm_budget=100, make_tasks=fake_tasks(log))
    r1 = eng.submit(Fake(n=1, mem=70, keep=60))  # a commitment keeps 60
    eng.drain(timeout=30)
    assert r1.error is None and eng.in_use == 60
    r2 = eng.submit(Fake(n=1, mem=50))  # can never fit next to the pool
    eng.drain(timeout=30)
    assert r2.error and "exhausted" in r2.error
    r3 = eng.submit(Fake(n=1, mem=30, fail=True))  # a failed commit keeps nothing
    eng.drain(timeout=30)
    assert r3.error and "planted" in r3.error and eng.in_use == 60
    eng.close()


def test_poisson_load_and_summary():
    off = serving.poisson_arrivals(50.0, 200, seed=3)
    assert np.all(np.diff(off) > 0)
    assert np.allclose(off, serving.poisson_arrivals(50.0, 200, seed=3))
    assert 2.0 < off[-1] < 6.5  # mean 200 / 50 = 4 s
    log = []
    eng = serving.Engine(None, slots=4, make_tasks=fake_tasks(log))
    res, span = serving.run_arrivals(eng, [Fake(n=2, sec=0.002) for _ in range(20)],
                                     serving.poisson_arrivals(200.0, 20, seed=1))
    eng.close()
    s = serving.summarize(res, span)
    assert s["requests"] == 20 and s["errors"] == 0
    assert 0 < s["p50_ms"] <= s["p99_ms"]
    assert all(r.latency >= 0.002 for r in res)

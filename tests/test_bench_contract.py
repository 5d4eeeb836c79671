"""The bench's whole-step compulsory-byte count on the CPU: the 8B int8 and
int16 workloads and the streamed 70B set, whose binding re-encodes every
block (each materialised vector written once and read once per dependent
pass)."""
import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

import bench  # noqa: E402
from parcomm_b200 import layout  # noqa: E402


def active_of(shapes):
    return layout.buckets(shapes)[1]


def test_8b_step_bytes():
    a = active_of(bench.shapes_8b())
    assert a == 8_053_063_680
    t8, terms8 = bench.step_alg_bytes(a, 1 << 33, 30, 4, 8, 1, False)
    assert abs(t8 / 1e9 - 235.1) < 0.1 and terms8["binding"] == 0
    assert terms8["commit"] == 8 * (1 << 30) * 9          # 8 live blocks, 1 + 64/8 bytes per entry
    t16, terms16 = bench.step_alg_bytes(a, 1 << 33, 30, 4, 4, 2, False)
    assert abs(t16 / 1e9 - 384.4) < 0.1 and terms16["commit"] == 8 * (1 << 30) * 18


def test_streamed_70b_step_bytes_include_binding():
    a = active_of(bench.shapes_70b())
    assert a == 70_598_524_928
    t, terms = bench.step_alg_bytes(a, 1 << 37, 30, 6, 4, 2, True)
    live = -(-a // (1 << 30))
    assert live == 66 and terms["binding"] == terms["commit"] == (live + 1) * (1 << 30) * 18
    assert 3.5e12 < t < 3.7e12


def test_forced_extremes_are_deterministic_with_repeated_draws():
    """A forced position drawn twice keeps its first draw's sign, so the
    synthetic weights are the same on every run (CPU generator here)."""
    import torch
    draws = []
    for _ in range(2):
        g = torch.Generator()
        g.manual_seed(7)
        w = torch.zeros(64)
        bench.force_extremes(w, 200, g)  # far more draws than positions: many repeats
        draws.append(w.clone())
    assert torch.equal(draws[0], draws[1])
    assert set(draws[0].unique().tolist()) <= {-127.0, 0.0, 127.0}
    g = torch.Generator()
    g.manual_seed(7)
    idx = torch.randint(0, 64, (200,), generator=g)
    sign = torch.randint(0, 2, (200,), generator=g).float().mul_(254.0).sub_(127.0)
    for pos in idx.unique().tolist():
        first = int((idx == pos).nonzero()[0])
        assert draws[0][pos] == sign[first]

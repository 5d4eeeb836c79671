"""LogUp range audit on a B200: multiplicities, alpha, lhs and rhs through the
C ABI equal the oracle's bytes for both fields, on resident and streamed
weights, with a ragged tail and with enough values per CTA to flush the
int16 counters many times; the audit leaves the commitment usable."""
import hashlib

import numpy as np
import pytest

import oracle
import parcomm_b200 as qf
from parcomm_b200 import layout

pytestmark = pytest.mark.gpu

FIELDS = {"f65521": (qf.FIELD_F65521, np.int8), "koalabear": (qf.FIELD_KOALABEAR, np.int16)}


def weights(shapes, dt, seed):
    rng = np.random.default_rng(seed)
    info = np.iinfo(dt)
    return [rng.integers(info.min, info.max + 1, size=s).astype(dt) for s in shapes]


def check(committed, bva, field, seed=None):
    res = committed.range_audit(seed)
    s = seed if seed is not None else hashlib.blake2s(b"".join(committed.roots)).digest()
    mult, a, l, r = oracle.range_audit(bva, s, field)
    assert np.array_equal(res.multiplicities, mult)
    assert (res.alpha, res.lhs, res.rhs) == (a, l, r)
    assert res.holds and int(mult.sum()) == bva.size
    return res


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
@pytest.mark.parametrize("mode", ["resident", "streamed"])
def test_audit_matches_the_oracle(field, mode):
    fid, dt = FIELDS[field]
    shapes = [(300, 700), (129, 65), (77, 1), (9, 1)]  # 219,671 active entries: a 7-value tail
    params = qf.Parameters(shapes, qf.Config(14, 4), field=fid)
    bva = qf.encode_bva(params, weights(shapes, dt, 1))
    assert bva.size % 16 == 7
    c = params.commit(bva) if mode == "resident" else params.commit_recomputed(bva, resident_bytes=0)
    check(c, bva, field)
    check(c, bva, field, seed=b"\x5a" * 32)
    # The commitment still proves after the audit.
    pts = params.benchmark_points(c.roots)
    claims = params.evaluate_claims(c, pts)
    proof, _ = params.prove(c, claims)
    params.verify(c.roots, claims, proof)


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
def test_audit_at_sixteen_million_values(field):
    """2^24 entries: every CTA runs many rounds (and flushes its int16
    counters every 64,512 values)."""
    fid, dt = FIELDS[field]
    shapes = [(4096, 4096)]
    params = qf.Parameters(shapes, qf.Config(20, 4), field=fid)
    rng = np.random.default_rng(9)
    if dt == np.int8:
        w = np.clip(np.rint(rng.normal(0, 20, size=shapes[0])), -127, 127).astype(np.int8)
    else:  # BF16 bit patterns of N(0, 0.02^2), read as int16: a concentrated histogram
        f = rng.normal(0, 0.02, size=shapes[0]).astype(np.float32)
        w = (f.view(np.uint32) >> 16).astype(np.uint16).view(np.int16)
        w.reshape(-1)[::8] = 0  # pruned entries: one bin far above 2^16
    bva = qf.encode_bva(params, [w])
    c = params.commit(bva)
    res = check(c, bva, field)
    assert int(res.multiplicities.max()) > 65536


def test_audit_of_the_demo_collection():
    """2,305 entries: most CTAs see no value, and one value is left over."""
    params = qf.Parameters(qf.demo_shapes(), qf.Config(10, 4))
    mats = [((np.arange(r * c).reshape(r, c) * 73 + 19 * i) % 256).astype(np.uint8).view(np.int8)
            for i, (r, c) in enumerate((s.rows, s.cols) for s in qf.demo_shapes())]
    bva = qf.encode_bva(params, mats)
    assert bva.size % 16 == 1
    c = params.commit(bva)
    check(c, bva, "f65521", seed=bytes(32))

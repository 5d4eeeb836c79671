"""The serving loop on a B200: every request's claims and proofs are the same
bytes alone (one request at a time) and in a concurrent mix, every proof
verifies, and pooled commitments answer repeated openings."""
import numpy as np
import pytest

import oracle
import parcomm_b200 as qf
from parcomm_b200 import layout, serving

pytestmark = pytest.mark.gpu


def make_pool(seed=0):
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    pool = serving.Pool()
    shapes = [(300, 700), (129, 65), (1024, 1024), (77, 1), (512, 4096), (64, 64)]
    for i, (r, c) in enumerate(shapes):
        w = torch.randint(-127, 128, (r, c), generator=g, device="cuda", dtype=torch.int32).to(torch.int8)
        pool.commit(w, qf.Config(14, 4), recompute=(i % 2 == 0))
    return pool


def requests(pool, seed):
    import torch
    rng = np.random.default_rng(seed)
    keys = pool.keys()
    reqs = []
    for k in range(8):
        pick = list(rng.choice(keys, size=int(rng.integers(1, 5)), replace=False))
        reqs.append(serving.OpenRequest(pick, [serving.random_points(pool.get(m).params, rng) for m in pick]))
        if k == 3:
            g = torch.Generator(device="cuda")
            g.manual_seed(seed + 99)
            w = torch.randint(-127, 128, (1500, 4096), generator=g, device="cuda", dtype=torch.int32).to(torch.int8)
            reqs.append(serving.CommitRequest(w, qf.Config(18, 4), recompute=True))
    return reqs


def outputs(pool, results):
    out = []
    for r in results:
        assert r.error is None, r.error
        if r.kind == "CommitRequest":
            out.append(b"".join(pool.get(r.outputs[0]).committed.roots))
        else:
            out.append(r.outputs)
    return out


def test_same_bytes_alone_and_in_the_mix():
    pool = make_pool()
    reqs = requests(pool, 5)
    alone = serving.Engine(pool, slots=1)
    seq = []
    for q in reqs:
        seq.append(alone.submit(q))
        alone.drain(timeout=600)
    alone.close()
    mixed = serving.Engine(pool, slots=4)
    mix = [mixed.submit(q) for q in reqs]
    mixed.drain(timeout=600)
    mixed.close()
    assert mixed.peak_running > 1
    assert outputs(pool, seq) == outputs(pool, mix)
    # Every proof verifies against its commitment and claims.
    for q, r in zip(reqs, mix):
        if isinstance(q, serving.OpenRequest):
            for key, (claims_b, proof_b) in zip(q.matrices, r.outputs):
                e = pool.get(key)
                claims = qf.claims_from_bytes(e.params.shapes, claims_b)
                e.params.verify(e.committed.roots, claims, proof_b)


def test_pooled_opening_matches_the_oracle():
    import torch
    pool = make_pool(seed=7)
    e = pool.get(pool.keys()[2])  # 1024 x 1024, recompute mode
    rng = np.random.default_rng(1)
    eng = serving.Engine(pool, slots=2)
    r = eng.submit(serving.OpenRequest([e.key], [serving.random_points(e.params, rng)]))
    eng.drain(timeout=600)
    eng.close()
    claims_b, proof_b = r.outputs[0]
    bva = e.weights.cpu().numpy()
    o_roots, o_claims, o_proof, _ = oracle.prove(e.params.shapes, 14, 4, bva, claims=claims_b)
    assert o_roots == b"".join(e.committed.roots) and o_claims == claims_b and o_proof == proof_b

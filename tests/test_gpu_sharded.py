"""The device shard of the block-sharded proof (qf_prove_sharded) on one
B200: one rank, and two or three ranks as threads of this process sharing
the GPU (each with its own stream and device copy; the collectives are an
all-gather through shared memory on the host, so no kernel waits on another
rank).  Every rank's roots and proof bytes equal the CPU oracle's
single-rank proof, in both fields, with the benchmark claims summed from the
ranks' parts and with given claims.  Requires a B200."""
import threading

import numpy as np
import pytest

import oracle
import parcomm_b200 as qf
from parcomm_b200 import layout

pytestmark = pytest.mark.gpu

SHAPES = [(300, 700), (129, 65), (1, 5000), (64, 64)]


class _Group:
    """An all-gather among `n` threads, every wait bounded."""

    def __init__(self, n):
        self.slots = [None] * n
        self.barrier = threading.Barrier(n, timeout=60)

    def gather(self, rank):
        def g(data: bytes) -> bytes:
            self.slots[rank] = data
            self.barrier.wait()
            out = b"".join(self.slots)
            self.barrier.wait()
            return out
        return g


def _bva(field):
    dt = np.int8 if field == "f65521" else np.int16
    info = np.iinfo(dt)
    rng = np.random.default_rng(7)
    return layout.encode(SHAPES, [rng.integers(info.min, info.max + 1, size=s, dtype=dt) for s in SHAPES])


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
@pytest.mark.parametrize("chunk_log,world", [(14, 1), (14, 2), (12, 3)])
@pytest.mark.parametrize("given_claims", [False, True])
def test_device_shards_write_the_single_rank_proof(field, chunk_log, world, given_claims):
    bva = _bva(field)
    o_roots, o_claims, o_proof, _ = oracle.prove(SHAPES, chunk_log, 4, bva, field=field)
    fid = qf.FIELD_F65521 if field == "f65521" else qf.FIELD_KOALABEAR
    params = [qf.Parameters(SHAPES, qf.Config(chunk_log=chunk_log, packed_log=4), field=fid) for _ in range(world)]
    claims = qf.claims_from_bytes(params[0].shapes, o_claims) if given_claims else None
    group, out, errors = _Group(world), [None] * world, [None] * world

    def rank(r):
        try:
            roots, proof = params[r].prove_sharded(bva, r, world, group.gather(r), claims=claims)
            out[r] = (b"".join(roots), proof.to_bytes())
        except Exception as e:  # reported below; the others leave their barrier
            errors[r] = repr(e)
            group.barrier.abort()

    threads = [threading.Thread(target=rank, args=(r,)) for r in range(world)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(120)
    assert not any(t.is_alive() for t in threads), "a rank did not finish"
    assert errors == [None] * world, errors
    for r in range(world):
        assert out[r] == (o_roots, o_proof), f"rank {r} differs from the single-rank proof"
    assert oracle.verify(SHAPES, chunk_log, 4, o_roots, o_claims, out[0][1], field=field)

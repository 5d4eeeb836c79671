"""Block-sharded proof over gloo ranks on CPU.

Each rank holds a contiguous run of the BVA's PCS blocks and runs the
sharding layer (csrc/host/sharded.h) with the oracle's CPU shard standing in
for its device; the exchanges are an all-gather and an integer all-reduce
over torch.distributed.
Every rank must write the proof that one rank holding all blocks writes,
byte for byte, in both fields, with given and with summed benchmark claims,
with the sums taken through the gather or through an integer all-reduce,
for world sizes that split the blocks evenly and unevenly.  A rank that
leaves, or an exchange that fails, ends the proof with an error.  World
sizes up to 8 and up to 128 blocks run as threads of one process."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from parcomm_b200 import layout

SHAPES = [(300, 700), (129, 65), (1, 5000), (64, 64)]  # 228,801 active entries, 2^18 logical


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _bva(field: str) -> np.ndarray:
    rng = np.random.default_rng(7)
    lo, hi, dt = (-128, 128, np.int8) if field == "f65521" else (-32768, 32768, np.int16)
    mats = [rng.integers(lo, hi, size=(r, c), dtype=dt) for r, c in SHAPES]
    return layout.encode(SHAPES, mats)


def _all_gather(world: int):
    def gather(data: bytes) -> bytes:
        t = torch.frombuffer(bytearray(data), dtype=torch.uint8)
        parts = [torch.empty_like(t) for _ in range(world)]
        dist.all_gather(parts, t)
        return b"".join(p.numpy().tobytes() for p in parts)
    return gather


def _all_reduce(a: np.ndarray) -> None:
    """In-place integer sum over the ranks (the sums stay below 2^63)."""
    dist.all_reduce(torch.from_numpy(a.view(np.int64)), op=dist.ReduceOp.SUM)


def _rank(rank: int, world: int, port: int, field: str, cases, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bva = _bva(field)
        for key, chunk_log, claims in cases:
            calls = []
            reduce = (lambda a: (calls.append(a.size), _all_reduce(a))) if key[0] == "reduce" else None
            out[(rank, key)] = oracle.prove_sharded(SHAPES, chunk_log, 4, bva, rank, world, _all_gather(world),
                                                    claims=claims, field=field, all_reduce=reduce)
            out[(rank, key, "reduce_calls")] = len(calls)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
@pytest.mark.parametrize("world", [2, 3, 4])
def test_sharded_proof_equals_single_rank_proof(field, world):
    bva = _bva(field)
    cases, expected = [], {}
    for chunk_log in (14, 16):  # 16 and 4 blocks
        roots, claims, proof, _ = oracle.prove(SHAPES, chunk_log, 4, bva, field=field)
        cases.append((("benchmark", chunk_log), chunk_log, None))
        cases.append((("given", chunk_log), chunk_log, claims))
        cases.append((("reduce", chunk_log), chunk_log, None))  # sums through the integer all-reduce
        for kind in ("benchmark", "given", "reduce"):
            expected[(kind, chunk_log)] = (roots, claims, proof)
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.spawn(_rank, args=(world, _free_port(), field, cases, out), nprocs=world, join=True)
    for key, want in expected.items():
        for rank in range(world):
            got = out[(rank, key)]
            assert got[0] == want[0], f"rank {rank} {key}: roots differ"
            assert got[1] == want[1], f"rank {rank} {key}: claims differ"
            assert got[2] == want[2], f"rank {rank} {key}: proof bytes differ"
            assert (out[(rank, key, "reduce_calls")] > 0) == (key[0] == "reduce")
        assert oracle.verify(SHAPES, key[1], 4, want[0], want[1], out[(0, key)][2], field=field)


def test_more_ranks_than_blocks_is_an_error():
    bva = _bva("f65521")
    with pytest.raises(oracle.OracleError, match="ranks <= blocks"):
        # chunk 16 gives 4 blocks; a fifth rank would hold none.  The error is
        # raised before the first exchange, so one process can check it alone.
        oracle.prove_sharded(SHAPES, 16, 4, bva, 0, 5, lambda b: b * 5)


def test_failed_exchange_is_an_error():
    bva = _bva("f65521")
    with pytest.raises(oracle.OracleError, match="all_gather"):
        oracle.prove_sharded(SHAPES, 16, 4, bva, 0, 2, lambda b: b)  # returns one rank's bytes, not two


def _rank_with_a_lost_peer(rank: int, world: int, port: int, out):
    import datetime
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    if rank == 1:
        os._exit(0)  # leaves between steps, before its first exchange
    try:
        oracle.prove_sharded(SHAPES, 16, 4, _bva("f65521"), rank, world, _all_gather(world))
        out[rank] = "proved"
    except oracle.OracleError as e:
        out[rank] = str(e)


def test_lost_rank_ends_the_proof_with_an_error():
    """A rank that leaves before the first exchange: the survivor's gather
    fails (peer gone or the process group's timeout) and the prover returns
    an error instead of waiting."""
    world = 2
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_with_a_lost_peer, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        for p in procs:
            p.join(timeout=120)
        assert all(p.exitcode is not None for p in procs), "a rank did not end"
    finally:
        for p in procs:
            if p.is_alive():
                p.kill()
                p.join()
    assert "all_gather" in out.get(0, ""), out.get(0)


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
def test_sharded_proof_with_ranks_as_threads(field):
    """World sizes 1 to 8 as threads of one process (the same layer and CPU
    shards, an all-gather through shared memory) over 16, 64 and 128 blocks:
    every rank writes the single-rank proof.  Odd world sizes commit block by
    block, even ones all blocks at once."""
    bva = _bva(field)
    for chunk_log in (14, 12, 11):  # 16, 64 and 128 blocks
        want = oracle.prove(SHAPES, chunk_log, 4, bva, field=field)[:3]
        for world in (1, 2, 5, 7, 8):
            roots, claims, proof, same = oracle.prove_sharded_threads(SHAPES, chunk_log, 4, bva, world, field=field)
            assert same, (chunk_log, world)
            assert (roots, claims, proof) == want, (chunk_log, world)


def test_sharded_proof_at_2_24_blocks():
    """One 8B decoder layer's attention projections (4 matrices, 41.9 M
    weights) at chunk 24: four ranks, one block each, write the single-rank
    proof."""
    shapes = [(4096, 4096), (1024, 4096), (1024, 4096), (4096, 4096)]
    rng = np.random.default_rng(0)
    mats = [np.clip(np.rint(rng.normal(0, 20, r * c)), -127, 127).astype(np.int8).reshape(r, c) for r, c in shapes]
    bva = layout.encode(shapes, mats)
    want = oracle.prove(shapes, 24, 4, bva)[:3]
    roots, claims, proof, same = oracle.prove_sharded_threads(shapes, 24, 4, bva, 4)
    assert same and (roots, claims, proof) == want

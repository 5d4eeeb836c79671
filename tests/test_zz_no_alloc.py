"""qf_commit_block_noalloc (static-scratch block commitment) against qf_commit.

Two calls in a row (other inputs, other block sizes, so the shared scratch
holds the previous call's contents) must each give exactly the root that
qf_commit writes for the same block.  Collected last; needs a B200."""
import numpy as np
import pytest
import torch

import parcomm_b200 as qf
from parcomm_b200 import layout

pytestmark = pytest.mark.gpu

SHAPES = [(1024, 4096), (300, 700), (129, 65)]


def device_bva(params, seed):
    rng = np.random.default_rng(seed)
    mats = [np.clip(np.rint(rng.normal(0.0, 20.0, s.rows * s.cols)), -127, 127).astype(np.int8).reshape(s.rows, s.cols)
            for s in params.shapes]
    return torch.from_numpy(layout.encode(params.shapes, mats)).cuda()


def noalloc_roots(params, bva, blocks):
    stream = torch.cuda.current_stream().cuda_stream
    out = []
    for b in blocks:
        root = torch.zeros(32, dtype=torch.uint8, device="cuda")
        params.block_root_noalloc(bva, b, root, stream)
        torch.cuda.synchronize()
        out.append(bytes(root.cpu().numpy()))
    return out


@pytest.mark.parametrize("first_chunk,second_chunk", [(20, 16), (16, 20)])
def test_noalloc_roots_match_qf_commit_two_calls(first_chunk, second_chunk):
    torch.cuda.set_device(0)
    for call, (chunk, seed) in enumerate([(first_chunk, 11), (second_chunk, 12)]):
        p = qf.Parameters(SHAPES, qf.Config(chunk_log=chunk, packed_log=4))
        bva = device_bva(p, seed)
        c = p.commit(bva, on_device=True)
        blocks = list(range(p.blocks))[::-1] if call else list(range(p.blocks))
        got = noalloc_roots(p, bva, blocks)
        for b, r in zip(blocks, got):
            assert r == c.roots[b], f"call {call}: block {b} root differs from qf_commit"
        c.close()


def test_noalloc_allocates_no_device_memory():
    torch.cuda.set_device(0)
    p = qf.Parameters(SHAPES, qf.Config(chunk_log=20, packed_log=4))
    bva = device_bva(p, 3)
    root = torch.zeros(32, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    p.block_root_noalloc(bva, 0, root, stream)  # first call on the device: set-up
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for b in range(p.blocks):
        p.block_root_noalloc(bva, b, root, stream)
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before


def test_noalloc_rejects_blocks_beyond_the_limit():
    torch.cuda.set_device(0)
    p = qf.Parameters([(2048, 1024)], qf.Config(chunk_log=21, packed_log=4))
    bva = torch.zeros(p.active, dtype=torch.int8, device="cuda")
    root = torch.zeros(32, dtype=torch.uint8, device="cuda")
    with pytest.raises(qf.QfError) as e:
        p.block_root_noalloc(bva, 0, root)
    assert e.value.code == -9 and "exceeds the limit of 2^20" in str(e.value)


def test_noalloc_back_to_back_on_a_caller_stream():
    """Several calls queued on a caller-owned stream with no host sync in
    between, each writing its own root slot, then one sync: every root equals
    qf_commit's.  A parameter set change in the middle (chunk 16, then 20)
    re-uploads the alpha table between calls."""
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    cases = []
    for chunk, seed in ((16, 21), (20, 22)):
        p = qf.Parameters(SHAPES, qf.Config(chunk_log=chunk, packed_log=4))
        bva = device_bva(p, seed)
        c = p.commit(bva, on_device=True)
        cases.append((p, bva, list(c.roots)))
        c.close()
    slots = torch.zeros(sum(p.blocks for p, _, _ in cases), 32, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()  # the weights and the zeroed slots are complete before the caller's stream reads them
    k = 0
    for p, bva, _ in cases:
        for b in range(p.blocks):
            p.block_root_noalloc(bva, b, slots[k], stream.cuda_stream)
            k += 1
    stream.synchronize()
    got = [bytes(r) for r in slots.cpu().numpy()]
    k = 0
    for p, _, roots in cases:
        for b in range(p.blocks):
            assert got[k] == roots[b], f"chunk {p.config.chunk_log} block {b}: root differs from qf_commit"
            k += 1


def test_noalloc_rejects_host_memory():
    torch.cuda.set_device(0)
    p = qf.Parameters(SHAPES, qf.Config(chunk_log=16, packed_log=4))
    bva = device_bva(p, 4)
    host_root = torch.zeros(32, dtype=torch.uint8)
    with pytest.raises(qf.QfError) as e:
        p.block_root_noalloc(bva, 0, host_root)
    assert e.value.code == -9 and "current device" in str(e.value)

"""Byte parity at chunk_log 30, the block size of the benchmarked 8B-shape
workloads, through the C ABI against the CPU oracle.  Requires a B200.

Chunk 30 is the only size at which several parts of the prover run: the code
sequence 2^22 -> 2^17 -> 2^12 -> 2^7 -> 2^2 rows (F65521^8; 2^23 -> ... for
KoalaBear^4), the f64 query counts of that sequence, the extension-row leaf
hashing of the deepest levels, the deepest strided transform passes over
2^27-element codeword halves, and a half-live last block.  The weights are the
benchmark's own synthetic draws (bench.make_bva_on_device, same seeds): the
embedding matrix of the 8B set alone (one block), and embedding + output head
+ one MLP gate matrix (two blocks, the second partly live).  Each case compares roots, claims and
proof bytes with the oracle (qafold/f65521/src/protocol.rs:201-263; the query
counts of vendor/qafold/src/qafold.rs:75-178) and checks both verifiers.
The oracle needs about a minute per 10^9 weights on 16 host threads."""
import hashlib

import numpy as np
import pytest
import torch

import bench
import oracle
import parcomm_b200 as qf

pytestmark = pytest.mark.gpu

EMBED = (128256, 4096)


def prove_both(shapes, field, bf16):
    torch.cuda.set_device(0)
    fid = qf.FIELD_KOALABEAR if bf16 else qf.FIELD_F65521
    p = qf.Parameters(shapes, qf.Config(chunk_log=30, packed_log=4), field=fid)
    bva_dev, active = bench.make_bva_on_device(shapes, seed=0, bf16=bf16, embedding_first=bf16)
    assert active == p.active
    c = p.commit(bva_dev, on_device=True)
    claims = p.evaluate_claims(c, p.benchmark_points(c.roots))
    proof, _ = p.prove(c, claims)
    gpu = (b"".join(c.roots), qf.claims_to_bytes(claims), proof.to_bytes())
    c.close()
    bva = bva_dev.cpu().numpy()
    del bva_dev
    torch.cuda.empty_cache()
    o_roots, o_claims, o_proof, _ = oracle.prove(p.shapes, 30, 4, bva, field=field)
    assert gpu[0] == o_roots, "commitment roots differ"
    assert gpu[1] == o_claims, "claims differ"
    assert len(gpu[2]) == len(o_proof), "proof lengths differ"
    assert gpu[2] == o_proof, (f"proof bytes differ: gpu {hashlib.blake2s(gpu[2]).hexdigest()} "
                               f"oracle {hashlib.blake2s(o_proof).hexdigest()}")
    p.verify(c.roots, claims, proof)
    assert oracle.verify(p.shapes, 30, 4, o_roots, o_claims, gpu[2], field=field)
    return p


def test_f65521_embedding_one_block_chunk30():
    p = prove_both([EMBED], "f65521", False)
    assert p.blocks == 1


def test_f65521_embedding_head_and_gate_two_blocks_chunk30():
    # 1.11 G weights: two 2^30 blocks, the second about a tenth live.
    p = prove_both([EMBED, EMBED, (14336, 4096)], "f65521", False)
    assert p.blocks == 2 and p.active > (1 << 30)


def test_koalabear_embedding_one_block_chunk30():
    p = prove_both([EMBED], "koalabear", True)
    assert p.blocks == 1

"""Byte parity on the full benchmarked workloads: the 226-matrix 8B-shape set
with int8 weights (F65521^8) and with BF16 payloads (KoalaBear^4), chunk_log
30, packed_log 4, the exact weights `bench.py` times (same generator, seed
0).  The proof the GPU writes is compared byte for byte with the CPU oracle's,
and both verifiers accept it.  Requires a B200.

The oracle needs about 11 minutes per workload on 16 host threads and about
60 GB (int8) / 110 GB (BF16) of host memory, so these cases run only when
QF_PARITY_FULL=1 is set; the chunk-30 cases of test_gpu_parity_chunk30.py
run always."""
import hashlib
import os
import time

import pytest
import torch

import bench
import oracle
import parcomm_b200 as qf

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(os.environ.get("QF_PARITY_FULL") != "1",
                                 reason="full 8B-shape oracle comparison: set QF_PARITY_FULL=1")]


@pytest.mark.parametrize("workload", ["8b8", "8b16"])
def test_full_8b_shape_proof_equals_oracle(workload):
    torch.cuda.set_device(0)
    bf16 = workload == "8b16"
    field = "koalabear" if bf16 else "f65521"
    shapes = bench.shapes_8b()
    p = qf.Parameters(shapes, qf.Config(30, 4), field=qf.FIELD_KOALABEAR if bf16 else qf.FIELD_F65521)
    bva_dev, active = bench.make_bva_on_device(shapes, seed=0, bf16=bf16, embedding_first=bf16)
    c = p.commit(bva_dev, on_device=True)
    claims = p.evaluate_claims(c, p.benchmark_points(c.roots))
    proof, _ = p.prove(c, claims)
    roots, cb, pb = b"".join(c.roots), qf.claims_to_bytes(claims), proof.to_bytes()
    c.close()
    bva = bva_dev.cpu().numpy()
    del bva_dev
    torch.cuda.empty_cache()
    t0 = time.time()
    o_roots, o_claims, o_proof, _ = oracle.prove(p.shapes, 30, 4, bva, field=field)
    oracle_s = time.time() - t0
    gd, od = hashlib.blake2s(pb).hexdigest(), hashlib.blake2s(o_proof).hexdigest()
    print(f"{workload}: proof {len(pb)} bytes, gpu blake2s {gd}, oracle blake2s {od}, oracle {oracle_s:.0f} s")
    assert roots == o_roots, "commitment roots differ"
    assert cb == o_claims, "claims differ"
    assert pb == o_proof, "proof bytes differ"
    p.verify(c.roots, claims, proof)
    assert oracle.verify(p.shapes, 30, 4, o_roots, o_claims, pb, field=field)

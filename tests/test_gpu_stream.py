"""Proving from the reference's dense BVA stream on a B200: a description and
stream file for each field, read into page-locked host memory and committed
in recompute mode (streamed per pass) and in cached mode, give the oracle's
roots, claims and proof bytes; the proof verifies."""
import numpy as np
import pytest

import oracle
import parcomm_b200 as qf
from parcomm_b200 import layout, stream

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("field,dt", [("f65521", np.int8), ("koalabear", np.int16)])
def test_prove_from_a_stream_file(tmp_path, field, dt):
    shapes = [(300, 700), (129, 65), (77, 1), (9, 1)]
    rng = np.random.default_rng(21)
    info = np.iinfo(dt)
    bva = layout.encode(shapes, [rng.integers(info.min, info.max + 1, size=s).astype(dt) for s in shapes], dt)
    stream.write_stream(tmp_path / "input.json", tmp_path / "input.bva", shapes, bva)
    model = stream.open_stream(tmp_path / "input.json", tmp_path / "input.bva", qf.Config(14, 4))
    assert model.params.blocks >= 2 and np.array_equal(model.bva, bva)
    o_roots, o_claims, o_proof, _ = oracle.prove(model.params.shapes, 14, 4, bva, field=field)
    for mode in ("recompute", "cached"):
        c = model.commit(mode, resident_bytes=0)
        assert b"".join(c.roots) == o_roots
        claims = model.params.evaluate_claims(c, model.params.benchmark_points(c.roots))
        assert qf.claims_to_bytes(claims) == o_claims
        proof, _ = model.params.prove(c, claims)
        assert proof.to_bytes() == o_proof
        model.params.verify(c.roots, claims, proof)

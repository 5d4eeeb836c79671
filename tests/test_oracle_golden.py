"""The CPU oracle is pinned to the reference's own golden vectors."""
import oracle

import parcomm_b200 as qf
from parcomm_b200 import layout


def test_demo_proof_digest_matches_reference(vectors):
    digest, proof_len, json_len = oracle.demo()
    g = vectors["f65521_demo"]
    assert proof_len == g["proof_bytes"]
    assert json_len == g["public_commitment_json_bytes"]
    assert digest.hex() == g["proof_blake2s"]


def test_wire_fixture_digest_matches_reference(vectors):
    assert oracle.wire_fixture().hex() == vectors["f65521_wire_fixture"]["blake2s_root_opening_decide"]


def test_demo_layout_matches_reference(vectors):
    bs, active, logical = layout.buckets(qf.demo_shapes())
    g = vectors["f65521_demo"]
    assert (len(bs), active, logical) == (g["bucket_count"], g["active_entries"], g["logical_entries"])


def test_demo_proof_verifies_in_oracle():
    shapes = qf.demo_shapes()
    bva = layout.encode(shapes, layout.demo_matrices(shapes))
    roots, claims, proof, _ = oracle.prove(shapes, 10, 4, bva)
    assert len(roots) == 4 * 32
    assert oracle.verify(shapes, 10, 4, roots, claims, proof)

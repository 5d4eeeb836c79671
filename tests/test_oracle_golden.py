"""The CPU oracle is pinned to the reference's own golden vectors."""
import numpy as np

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


def test_koalabear_demo_proof_digest_matches_reference(vectors):
    """G2: the KoalaBear^4 / signed-i16 demo bundle (qafold/koalabear main.rs)."""
    digest, proof_len, json_len = oracle.demo("koalabear")
    g = vectors["koalabear_demo"]
    assert proof_len == g["proof_bytes"]
    assert json_len == g["public_commitment_json_bytes"]
    assert digest.hex() == g["proof_blake2s"]


def test_koalabear_demo_proof_verifies_and_tampering_is_rejected():
    shapes = qf.demo_shapes()
    bva = layout.encode(shapes, layout.demo_matrices(shapes, np.int16), np.int16)
    roots, claims, proof, _ = oracle.prove(shapes, 10, 4, bva, field="koalabear")
    assert oracle.verify(shapes, 10, 4, roots, claims, proof, field="koalabear")
    bad = bytearray(proof)
    bad[len(bad) // 2] ^= 1
    assert not oracle.verify(shapes, 10, 4, roots, claims, bytes(bad), field="koalabear")
    assert not oracle.verify(shapes, 10, 4, roots, claims, proof, field="f65521")

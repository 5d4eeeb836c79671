"""Verifier acceptance and rejection of altered proofs (end_to_end.rs:71-169),
through both the product's host verifier and the oracle's."""
import numpy as np
import pytest

import oracle
import parcomm_b200 as qf
from parcomm_b200 import layout

CFG = qf.Config(chunk_log=10, packed_log=4)


@pytest.fixture(scope="module")
def demo_bundle():
    shapes = qf.demo_shapes()
    bva = layout.encode(shapes, layout.demo_matrices(shapes))
    roots, claims, proof, _ = oracle.prove(shapes, 10, 4, bva)
    return shapes, roots, claims, proof


def product_accepts(shapes, roots, claims, proof):
    p = qf.Parameters(shapes, CFG)
    try:
        p.verify([roots[i:i + 32] for i in range(0, len(roots), 32)], qf.claims_from_bytes(p.shapes, claims), proof)
        return True
    except qf.QfError:
        return False


def test_product_verifier_accepts_oracle_proof(demo_bundle):
    assert product_accepts(*demo_bundle)


@pytest.mark.parametrize("pos", [0, 8, 200, 600, 792, 800, 820, 900, 2000, 5000, 12000, 20000, 26900, 26973])
def test_flipped_byte_rejected(demo_bundle, pos):
    shapes, roots, claims, proof = demo_bundle
    bad = bytearray(proof)
    bad[pos] ^= 0x01
    assert not product_accepts(shapes, roots, claims, bytes(bad))
    assert not oracle.verify(shapes, 10, 4, roots, claims, bytes(bad))


def test_truncated_and_extended_rejected(demo_bundle):
    shapes, roots, claims, proof = demo_bundle
    assert not product_accepts(shapes, roots, claims, proof[:-1])
    assert not product_accepts(shapes, roots, claims, proof + b"\0")


def test_wrong_claim_value_rejected(demo_bundle):
    shapes, roots, claims, proof = demo_bundle
    bad = bytearray(claims)
    bad[-16] = (bad[-16] + 1) % 251
    assert not product_accepts(shapes, roots, claims=bytes(bad), proof=proof)


def test_wrong_root_rejected(demo_bundle):
    shapes, roots, claims, proof = demo_bundle
    bad = bytearray(roots)
    bad[33] ^= 0x80
    assert not product_accepts(shapes, bytes(bad), claims, proof)

"""Verifier acceptance and rejection of altered proofs (end_to_end.rs:71-169),
through both the product's host verifier and the oracle's."""
import numpy as np
import pytest

import oracle
import parcomm_b200 as qf
from parcomm_b200 import layout

CFG = qf.Config(chunk_log=10, packed_log=4)
ROOT = __import__("pathlib").Path(__file__).resolve().parents[1]


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


# ---- field-level mutations (end_to_end.rs:70-169), both fields
_P = {"f65521": (65521, 2), "koalabear": (2130706433, 4)}


def _parse_proof(w: bytes):
    pos = 0

    def u64():
        nonlocal pos
        pos += 8
        return int.from_bytes(w[pos - 8: pos], "little")

    def el():
        nonlocal pos
        pos += 16
        return w[pos - 16: pos]

    p = {"positive": [el() for _ in range(u64())], "negative": [el() for _ in range(u64())]}
    p["rounds"] = [[el(), el()] for _ in range(u64())]
    p["value"], p["query"] = el(), el()
    p["openings"] = []
    for _ in range(u64()):
        v, n = el(), u64()
        p["openings"].append([v, w[pos: pos + n]])
        pos += n
    assert pos == len(w)
    return p


def _write_proof(p) -> bytes:
    le = lambda n: n.to_bytes(8, "little")
    out = le(len(p["positive"])) + b"".join(p["positive"]) + le(len(p["negative"])) + b"".join(p["negative"])
    out += le(len(p["rounds"])) + b"".join(a + b for a, b in p["rounds"]) + p["value"] + p["query"]
    out += le(len(p["openings"])) + b"".join(v + le(len(b)) + b for v, b in p["openings"])
    return out


def _plus_one(e: bytes, field: str) -> bytes:
    p, w = _P[field]
    c0 = (int.from_bytes(e[:w], "little") + 1) % p
    return c0.to_bytes(w, "little") + e[w:]


@pytest.fixture(scope="module", params=["f65521", "koalabear"])
def collection(request):
    field = request.param
    shapes = [(31, 37), (65, 17), (1, 7), (9, 1), (1, 1)]
    dt = np.int8 if field == "f65521" else np.int16
    bva = layout.encode(shapes, layout.demo_matrices(shapes, dtype=dt))
    roots, claims, proof, _ = oracle.prove(shapes, 10, 4, bva, field=field)
    assert len(roots) > 32
    return field, shapes, roots, claims, proof


def _accepts(field, shapes, roots, claims, proof):
    ok = oracle.verify(shapes, 10, 4, roots, claims, proof, field=field)
    p = qf.Parameters(shapes, CFG, field=qf.FIELD_F65521 if field == "f65521" else qf.FIELD_KOALABEAR)
    try:
        p.verify([roots[i:i + 32] for i in range(0, len(roots), 32)], qf.claims_from_bytes(p.shapes, claims), proof)
        product = True
    except qf.QfError:
        product = False
    assert ok == product, "the two verifiers disagree"
    return ok


def _mutations(field):
    def set_(path, fn):
        def m(p):
            cur = p
            for k in path[:-1]:
                cur = cur[k]
            cur[path[-1]] = fn(cur[path[-1]])
        return m
    inc = lambda e: _plus_one(e, field)
    return {
        "positive[0] + 1": set_(["positive", 0], inc),
        "negative[0] + 1": set_(["negative", 0], inc),
        "rounds[0][0] + 1": set_(["rounds", 0, 0], inc),
        "query + 1": set_(["query"], inc),
        "value + 1": set_(["value"], inc),
        "opening value + 1": set_(["openings", 0, 0], inc),
        "opening proof[0] ^ 1": set_(["openings", 0, 1], lambda b: bytes([b[0] ^ 1]) + b[1:]),
        "opening duplicated": lambda p: p["openings"].append(list(p["openings"][0])),
        "opening removed": lambda p: p["openings"].pop(),
        "last round removed": lambda p: p["rounds"].pop(),
        "value non-canonical": set_(["value"], lambda e: bytes([255]) * 16),
    }


@pytest.mark.parametrize("name", list(_mutations("f65521")))
def test_each_proof_field_mutation_is_rejected(collection, name):
    field, shapes, roots, claims, proof = collection
    assert _write_proof(_parse_proof(proof)) == proof
    assert _accepts(field, shapes, roots, claims, proof)
    p = _parse_proof(proof)
    _mutations(field)[name](p)
    assert not _accepts(field, shapes, roots, claims, _write_proof(p))


def test_statement_and_claim_mutations_are_rejected(collection):
    field, shapes, roots, claims, proof = collection
    swapped = roots[32:64] + roots[:32] + roots[64:]
    assert not _accepts(field, shapes, swapped, claims, proof)
    flipped = bytes([roots[0] ^ 1]) + roots[1:]
    assert not _accepts(field, shapes, flipped, claims, proof)
    # the first claim: its row point (5 elements), column point (6), value
    value_at = 16 * (5 + 6)
    bad = claims[:value_at] + _plus_one(claims[value_at:value_at + 16], field) + claims[value_at + 16:]
    assert not _accepts(field, shapes, roots, bad, proof)
    col_at = 16 * 5
    bad = claims[:col_at] + _plus_one(claims[col_at:col_at + 16], field) + claims[col_at + 16:]
    assert not _accepts(field, shapes, roots, bad, proof)
    fewer = [(30, 37)] + shapes[1:]
    assert not oracle.verify(fewer, 10, 4, roots, claims, proof, field=field)
    assert not _accepts(field, shapes, roots, claims, proof[:-1])
    assert not _accepts(field, shapes, roots, claims, proof + b"\0")


def test_fresh_process_verifies_from_public_bytes(tmp_path):
    """cli_stream.py:1-40: a process with no prover state (only the shapes,
    the config, the roots, the claims and the proof bytes on disk) accepts
    the proof, and rejects it with its last byte flipped."""
    import subprocess
    import sys
    shapes = [(32, 32)]
    mat = (np.arange(1024, dtype=np.int64) * 73 % 256).astype(np.uint8).view(np.int8).reshape(32, 32)
    bva = layout.encode(shapes, [mat])
    roots, claims, proof, _ = oracle.prove(shapes, 10, 4, bva)
    for name, data in (("roots", roots), ("claims", claims), ("proof", proof)):
        (tmp_path / name).write_bytes(data)
    script = (
        "import sys; from pathlib import Path; import parcomm_b200 as qf\n"
        "d = Path(sys.argv[1]); r = (d / 'roots').read_bytes()\n"
        "p = qf.Parameters([(32, 32)], qf.Config(chunk_log=10, packed_log=4))\n"
        "try:\n"
        "    p.verify([r[i:i + 32] for i in range(0, len(r), 32)],\n"
        "             qf.claims_from_bytes(p.shapes, (d / 'claims').read_bytes()), (d / 'proof').read_bytes())\n"
        "    print('verified')\n"
        "except qf.QfError as e:\n"
        "    print('rejected', e.code)\n")
    run = lambda: subprocess.run([sys.executable, "-c", script, str(tmp_path)], capture_output=True, text=True,
                                 cwd=str(ROOT), timeout=300)
    r = run()
    assert r.returncode == 0 and r.stdout.strip() == "verified", r.stderr
    bad = bytearray(proof)
    bad[-1] ^= 1
    (tmp_path / "proof").write_bytes(bytes(bad))
    r = run()
    assert r.returncode == 0 and r.stdout.startswith("rejected"), r.stderr

"""Claims and edge cases of the protocol, checked without the shared host code.

A claim's value is the matrix's coefficient-form polynomial at the claim's
point: sum over (r, c) of M[r, c] times the row coordinates whose bit is set
in r and the column coordinates whose bit is set in c (tbv.rs:143-185; the
reference's own independent check is end_to_end.rs:41-66).  This file
evaluates that sum in numpy, with its own extension arithmetic
(F65521[X]/(X^8 - 17), KoalaBear[X]/(X^4 - 3)), on the matrices themselves
rather than the BVA, and compares it with the oracle's claims.  It also
restates two of the reference's end-to-end cases: every packing width at
points with 0, 1 and -1 coordinates (end_to_end.rs:170-193) and a matrix with
more rows than the F65521 characteristic (end_to_end.rs:299-310)."""
import numpy as np
import pytest

import oracle
import parcomm_b200 as qf
from parcomm_b200 import layout

# field: (p, degree, X^degree =, bytes per coefficient, weight dtype)
FIELDS = {"f65521": (65521, 8, 17, 2, np.int8), "koalabear": (2130706433, 4, 3, 4, np.int16)}


def ext_mul(a, b, field):
    """Row-wise product of (n, d) and (n or 1, d) coefficient arrays."""
    p, d, nr, _, _ = FIELDS[field]
    a, b = np.atleast_2d(a), np.atleast_2d(b)
    out = np.zeros((max(a.shape[0], b.shape[0]), d), dtype=np.int64)
    for i in range(d):
        for j in range(d):
            t = (a[:, i] * b[:, j]) % p  # each factor < 2^31, so the product fits
            if i + j < d:
                out[:, i + j] = (out[:, i + j] + t) % p
            else:
                out[:, i + j - d] = (out[:, i + j - d] + nr * t) % p
    return out


def base(v, field):
    p, d, _, _, _ = FIELDS[field]
    e = np.zeros(d, dtype=np.int64)
    e[0] = v % p
    return e


def monomial_weights(point, n, field):
    """Weights of the indices 0..n-1: the product of point[k] over the bits k set."""
    w = base(1, field)[None, :]
    for c in point:
        w = np.concatenate([w, ext_mul(w, c[None, :], field)])
    return w[:n]


def claim_value(matrix, row_point, col_point, field):
    p = FIELDS[field][0]
    rows, cols = matrix.shape
    colw = monomial_weights(col_point, cols, field)
    inner = (matrix.astype(np.int64) @ colw) % p  # |entries| <= 2^15, weights < 2^31: no overflow at these sizes
    return ext_mul(inner, monomial_weights(row_point, rows, field), field).sum(axis=0) % p


def ext_to_bytes(e, field):
    w = FIELDS[field][3]
    return b"".join(int(c).to_bytes(w, "little") for c in e)


def ext_from_bytes(b, field):
    _, d, _, w, _ = FIELDS[field]
    return np.array([int.from_bytes(b[w * i: w * (i + 1)], "little") for i in range(d)], dtype=np.int64)


def parse_claims(shapes, data, field):
    out, pos = [], 0
    for r, c in shapes:
        nr, nc = (r - 1).bit_length(), (c - 1).bit_length()
        elems = [ext_from_bytes(data[pos + 16 * i: pos + 16 * (i + 1)], field) for i in range(nr + nc + 1)]
        pos += 16 * (nr + nc + 1)
        out.append((elems[:nr], elems[nr:nr + nc], elems[-1]))
    assert pos == len(data)
    return out


def random_matrices(shapes, field, seed):
    dt = FIELDS[field][4]
    info = np.iinfo(dt)
    rng = np.random.default_rng(seed)
    return [rng.integers(info.min, info.max + 1, size=s, dtype=dt) for s in shapes]


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
def test_benchmark_claims_equal_the_matrix_polynomial(field):
    shapes = [(31, 37), (65, 17), (1, 7), (9, 1), (300, 70), (1, 5000), (129, 1)]
    mats = random_matrices(shapes, field, 5)
    bva = layout.encode(shapes, mats)
    for chunk_log in (10, 14):
        roots, claims, proof, _ = oracle.prove(shapes, chunk_log, 4, bva, field=field)
        for m, (row, col, value) in zip(mats, parse_claims(shapes, claims, field)):
            assert np.array_equal(claim_value(m, row, col, field), value)
        assert oracle.verify(shapes, chunk_log, 4, roots, claims, proof, field=field)


def product_verifies(shapes, chunk_log, packed_log, roots, claims, proof, field):
    p = qf.Parameters(shapes, qf.Config(chunk_log=chunk_log, packed_log=packed_log),
                      field=qf.FIELD_F65521 if field == "f65521" else qf.FIELD_KOALABEAR)
    try:
        p.verify([roots[i:i + 32] for i in range(0, len(roots), 32)], qf.claims_from_bytes(p.shapes, claims), proof)
        return True
    except qf.QfError:
        return False


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
@pytest.mark.parametrize("packed_log", [1, 2, 3, 4, 5, 6])
def test_packing_widths_at_zero_one_minus_one_points(field, packed_log):
    """A 5 x 7 matrix of -128 at the row point (0, 1, -1) and the column point
    (1, 0, -1), with the default chunk_log (30, which the 1024-entry layout
    reduces to 10): the claim's value comes from the matrix polynomial here,
    and the oracle proves it only if the protocol agrees."""
    shapes = [(5, 7)]
    mat = np.full((5, 7), -128, dtype=FIELDS[field][4])
    row = [base(v, field) for v in (0, 1, -1)]
    col = [base(v, field) for v in (1, 0, -1)]
    value = claim_value(mat, row, col, field)
    claims = b"".join(ext_to_bytes(e, field) for e in row + col + [value])
    bva = layout.encode(shapes, [mat])
    roots, claims_out, proof, _ = oracle.prove(shapes, 30, packed_log, bva, claims=claims, field=field)
    assert claims_out == claims
    assert oracle.verify(shapes, 30, packed_log, roots, claims, proof, field=field)
    assert product_verifies(shapes, 30, packed_log, roots, claims, proof, field)
    bad = bytearray(claims)
    bad[-16] ^= 1  # another value at the same point
    assert not oracle.verify(shapes, 30, packed_log, roots, bytes(bad), proof, field=field)


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
def test_rows_above_the_characteristic_are_not_aliased(field):
    """65523 rows > 65521: row indices 65521 and 65522 must not alias 0 and 1
    (end_to_end.rs:299-310 in both crates)."""
    shapes = [(65523, 1)]
    mats = layout.demo_matrices(shapes, dtype=FIELDS[field][4])
    bva = layout.encode(shapes, mats)
    roots, claims, proof, _ = oracle.prove(shapes, 10, 4, bva, field=field)
    (row, col, value), = parse_claims(shapes, claims, field)
    assert len(row) == 16 and len(col) == 0
    assert np.array_equal(claim_value(mats[0], row, col, field), value)
    assert oracle.verify(shapes, 10, 4, roots, claims, proof, field=field)
    assert product_verifies(shapes, 10, 4, roots, claims, proof, field)


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
def test_compact_query_equals_its_dense_form(field):
    """tbv::compile's compact terms, written out densely, give the query's
    claim against the BVA, its evaluation at a point (the dense vector folded
    pair by pair) and the Laurent cross terms at stride 16 (end_to_end.rs:216-262)."""
    p = FIELDS[field][0]
    shapes = [(31, 31), (3, 2)]
    mats = layout.demo_matrices(shapes, dtype=FIELDS[field][4])
    bva = layout.encode(shapes, mats)
    _, claims, _, _ = oracle.prove(shapes, 10, 4, bva, field=field)
    dense, claim, point, evaluation, positive, negative = oracle.tbv_dense(shapes, 10, 4, bva, claims, 16, field=field)
    q = np.array([ext_from_bytes(b, field) for b in dense])
    v = np.zeros(len(dense), dtype=np.int64)
    v[: bva.size] = bva
    assert np.count_nonzero(q.any(axis=1)) >= bva.size // 2 and v.any()
    assert np.array_equal(((v[:, None] * q) % p).sum(axis=0) % p, ext_from_bytes(claim, field))
    reduced = q
    for b in point:
        reduced = (reduced[0::2] + ext_mul(reduced[1::2], ext_from_bytes(b, field)[None, :], field)) % p
    assert np.array_equal(reduced[0], ext_from_bytes(evaluation, field))
    vs, qs = v.reshape(-1, 16), q.reshape(-1, 16, q.shape[1])
    for d in range(1, 16):
        pos = ((vs[:, : 16 - d, None] * qs[:, d:, :]) % p).sum(axis=(0, 1)) % p
        neg = ((vs[:, d:, None] * qs[:, : 16 - d, :]) % p).sum(axis=(0, 1)) % p
        assert np.array_equal(pos, ext_from_bytes(positive[d - 1], field)), d
        assert np.array_equal(neg, ext_from_bytes(negative[d - 1], field)), d


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
def test_padding_is_a_proved_predicate(field):
    """protocol.rs:332-353: a nonzero entry in a bucket's padding is refused
    by the layout check and, with the check skipped, by the proof itself."""
    shapes = [(31, 31)]
    mat = np.ones((31, 31), dtype=FIELDS[field][4])
    row, col = [base(3, field)] * 5, [base(7, field)] * 5
    claims = b"".join(ext_to_bytes(e, field) for e in row + col + [claim_value(mat, row, col, field)])
    bva = layout.encode(shapes, [mat])
    _, _, proof, _ = oracle.prove(shapes, 30, 4, bva, claims=claims, field=field)
    assert oracle.prove_unchecked(shapes, 30, 4, bva, claims, field=field) == proof
    b = next(b for b in layout.buckets(shapes)[0] if b.rows > b.physical_rows or b.cols > b.physical_cols)
    index = b.offset + b.physical_cols if b.cols > b.physical_cols else b.offset + b.physical_rows * b.cols
    corrupt = bva.copy()
    corrupt[index] = 1
    with pytest.raises(oracle.OracleError, match="padding"):
        oracle.prove(shapes, 30, 4, corrupt, claims=claims, field=field)
    with pytest.raises(oracle.OracleError, match="packed reduction claim mismatch"):
        oracle.prove_unchecked(shapes, 30, 4, corrupt, claims, field=field)


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
def test_implicit_suffix_is_checked_by_the_same_relation(field):
    """protocol.rs:354-368: the entries past the active ones are zero by the
    proof's relation; a 1 in the last logical entry makes the proof fail."""
    shapes = [(3, 5)]
    mat = np.full((3, 5), 2, dtype=FIELDS[field][4])
    row, col = [base(3, field)] * 2, [base(7, field)] * 3
    claims = b"".join(ext_to_bytes(e, field) for e in row + col + [claim_value(mat, row, col, field)])
    bva = layout.encode(shapes, [mat])
    logical = layout.buckets(shapes)[2]
    full = np.zeros(logical, dtype=bva.dtype)
    full[: bva.size] = bva
    _, _, proof, _ = oracle.prove(shapes, 30, 4, bva, claims=claims, field=field)
    assert oracle.prove_unchecked(shapes, 30, 4, full, claims, field=field) == proof
    full[-1] = 1
    with pytest.raises(oracle.OracleError, match="packed reduction claim mismatch"):
        oracle.prove_unchecked(shapes, 30, 4, full, claims, field=field)

"""The single-block packed PCS against the multilinear extension of the
original base table, computed here from its definition without the packing
helpers (after vendor/qafold/tests/packed.rs:10-112): an extension-field
point, each of the eight lanes packed into one element (the last three
coordinates, most significant first), and Boolean points that select single
entries.  Each opening must claim the table's value and verify; another
value or a flipped proof byte must not."""
import numpy as np
import pytest

import oracle
from test_oracle_claims import FIELDS, ext_from_bytes, ext_mul, ext_to_bytes

SEED = bytes([91]) * 32
CTX = b"packed-pcs/integration-tests/v1"


def table(field, log_n, seed):
    return np.random.default_rng(seed).integers(0, FIELDS[field][0], size=1 << log_n, dtype=np.int64)


def ext_point(field, log_n, seed):
    """Coordinates with a nonzero coefficient above the base field."""
    p, d, _, _, _ = FIELDS[field]
    pt = np.random.default_rng(seed).integers(0, p, size=(log_n, d), dtype=np.int64)
    pt[:, 1] = np.maximum(pt[:, 1], 1)
    return pt


def base_point(field, bits):
    d = FIELDS[field][1]
    pt = np.zeros((len(bits), d), dtype=np.int64)
    pt[:, 0] = bits
    return pt


def original_mle(values, point, field):
    """Fold the table on its most significant index bit first:
    t[i] <- t[i] (1 - x) + t[half + i] x."""
    p, d, _, _, _ = FIELDS[field]
    t = np.zeros((values.size, d), dtype=np.int64)
    t[:, 0] = values % p
    one = np.zeros(d, dtype=np.int64)
    one[0] = 1
    for x in point:
        half = len(t) // 2
        t = (ext_mul(t[:half], ((one - x) % p)[None, :], field) + ext_mul(t[half:], x[None, :], field)) % p
    return t[0]


def open_and_check(field, log_n, values, point):
    pb = b"".join(ext_to_bytes(x, field) for x in point)
    root, value, proof = oracle.packed_open(log_n, 4, 32, SEED, values, pb, CTX, field=field)
    assert np.array_equal(ext_from_bytes(value, field), original_mle(values, point, field))
    assert oracle.packed_verify(log_n, 4, 32, SEED, root, pb, value, proof, CTX, field=field)
    return root, pb, value, proof


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
def test_extension_point_authenticates_the_original_table(field):
    log_n = 9
    values = table(field, log_n, 1)
    root, pb, value, proof = open_and_check(field, log_n, values, ext_point(field, log_n, 2))
    other = bytearray(value)
    other[0] ^= 1
    assert not oracle.packed_verify(log_n, 4, 32, SEED, root, pb, bytes(other), proof, CTX, field=field)
    for pos in (0, 40, len(proof) // 2, len(proof) - 1):
        bad = bytearray(proof)
        bad[pos] ^= 0x10
        assert not oracle.packed_verify(log_n, 4, 32, SEED, root, pb, value, bytes(bad), CTX, field=field)
    assert not oracle.packed_verify(log_n, 4, 32, SEED, root, pb, value, proof, CTX + b"x", field=field)


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
def test_each_lane_is_selected_by_the_last_coordinates(field):
    """An element packs 2^k adjacent entries (k = 3 for F65521^8, 2 for
    KoalaBear^4); Boolean values of the last k coordinates, most significant
    first, pick one lane."""
    log_n = 7
    lane_bits = FIELDS[field][1].bit_length() - 1
    values = table(field, log_n, 3)
    for lane in range(1 << lane_bits):
        pt = ext_point(field, log_n, 4)
        for bit in range(lane_bits):
            pt[log_n - lane_bits + bit] = base_point(field, [(lane >> (lane_bits - 1 - bit)) & 1])[0]
        open_and_check(field, log_n, values, pt)


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
def test_boolean_points_select_the_original_entry(field):
    log_n = 6
    values = table(field, log_n, 5)
    for index in (0, 1, 7, 8, (1 << log_n) - 1):
        bits = [(index >> (log_n - 1 - b)) & 1 for b in range(log_n)]
        root, pb, value, proof = open_and_check(field, log_n, values, base_point(field, bits))
        assert ext_from_bytes(value, field)[0] == values[index] and not ext_from_bytes(value, field)[1:].any()


def source(field, blocks, log_n):
    """index * 7927 + block * 65519 + 31, reduced (packed_batch_tests.rs:3-9)."""
    p = FIELDS[field][0]
    idx = np.arange(1 << log_n, dtype=np.int64)
    return np.concatenate([(idx * 7927 + b * 65519 + 31) % p for b in range(blocks)])


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
@pytest.mark.parametrize("blocks,log_n", [(2, 10), (4, 10), (8, 10), (64, 10), (2, 16)])
def test_batch_opening_equals_the_concatenated_tables_extension(field, blocks, log_n):
    """After packed_batch_tests.rs:40-140: the batch opening claims the
    multilinear extension of the blocks' tables laid end to end (the block
    coordinates first), Boolean coordinates included, and verifies; another
    context, a missing or altered root, a flipped byte in each wire section,
    and a wire one byte longer or shorter are rejected."""
    lanes = FIELDS[field][1]
    values = source(field, blocks, log_n)
    k = log_n + blocks.bit_length() - 1
    pt = ext_point(field, k, 10 * blocks + log_n)
    if blocks == 4:
        pt[0], pt[1], pt[log_n] = base_point(field, [0, 1, 1])
    pb = b"".join(ext_to_bytes(x, field) for x in pt)
    seed = bytes([0x51]) * 32
    ctx = b"batch-test"
    roots, value, wire = oracle.packed_open_batch(log_n, 32, 100, seed, blocks, values, pb, ctx, field=field)
    assert np.array_equal(ext_from_bytes(value, field), original_mle(values, pt, field))
    verify = lambda r=roots, w=wire, c=ctx: oracle.packed_verify_batch(log_n, 32, 100, seed, r, pb, value, w, c,
                                                                      field=field)
    assert verify()
    assert not verify(c=b"different-context")
    assert not verify(r=roots[:-32])
    for b in range(blocks):
        bad = bytearray(roots)
        bad[32 * b] ^= 1
        assert not verify(r=bytes(bad))
    cross = 8 + 16 + lanes * 16
    folded_root = cross + 2 * (blocks - 1) * 16
    final = folded_root + 32 + (log_n - (lanes.bit_length() - 1)) * 32
    binding = final + 16 + 8
    for offset in (0, 8, 24, cross, folded_root, final, binding, len(wire) - 1):
        bad = bytearray(wire)
        bad[offset] ^= 1
        assert not verify(w=bytes(bad)), f"accepted a flipped byte at {offset}"
    assert not verify(w=wire + b"\0")
    assert not verify(w=wire[:-1])


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
def test_fold_binding_under_other_weights_is_rejected(field):
    """packed_batch_tests.rs:142-165: a folded commitment made with the block
    weights (1, 1) binds under (1, 1) and is rejected under (1, 2)."""
    values = source(field, 2, 10)
    seed, pcs_seed = bytes([0x78]) * 32, bytes([0x51]) * 32
    assert oracle.codeword_fold_accepted(10, 32, 100, pcs_seed, 2, values, [1, 1], seed, [1, 1], field=field)
    assert not oracle.codeword_fold_accepted(10, 32, 100, pcs_seed, 2, values, [1, 1], seed, [1, 2], field=field)
    assert oracle.codeword_fold_accepted(10, 32, 100, pcs_seed, 2, values, [1, 2], seed, [1, 2], field=field)


def _plus_one(b: bytes, field) -> bytes:
    p, _, _, w, _ = FIELDS[field]
    return ((int.from_bytes(b[:w], "little") + 1) % p).to_bytes(w, "little") + b[w:16]


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
def test_single_opening_rejects_modified_statements_and_wires(field):
    """vendor/qafold/tests/packed.rs:126-262: another root, claim, point
    coordinate, context or setup; every wrapper field changed to another
    canonical value; a byte of each native payload; lengths set to 2^64 - 1;
    a non-canonical conjugate; truncations; a trailing byte; the magic.  And
    a PCS of 2^3 values is refused."""
    log_n = 9
    p, lanes, _, w, _ = FIELDS[field]
    values = table(field, log_n, 11)
    pt = ext_point(field, log_n, 12)
    pb = b"".join(ext_to_bytes(x, field) for x in pt)
    root, value, wire = oracle.packed_open(log_n, 4, 32, SEED, values, pb, CTX, field=field)
    ok = lambda r=root, q=pb, v=value, b=wire, c=CTX, s=SEED: oracle.packed_verify(log_n, 4, 32, s, r, q, v, b, c,
                                                                                   field=field)
    assert ok()
    assert not ok(r=bytes([root[0] ^ 1]) + root[1:])
    assert not ok(v=_plus_one(value, field))
    for k in (0, log_n - 1):
        assert not ok(q=pb[: 16 * k] + _plus_one(pb[16 * k: 16 * k + 16], field) + pb[16 * k + 16:])
    assert not ok(c=b"another context")
    assert not ok(s=bytes([92]) * 32)
    rd = lambda at: int.from_bytes(wire[at: at + 8], "little")
    count_at = 8 + 16 + lanes * 16
    rounds = log_n - (lanes.bit_length() - 1)
    assert rd(count_at) == rounds
    rounds_at = count_at + 8
    final_at = rounds_at + 32 * rounds
    opening_len_at = final_at + 16
    opening_at = opening_len_at + 8
    decide_len_at = opening_at + rd(opening_len_at)
    decide_at = decide_len_at + 8
    assert decide_at + rd(decide_len_at) == len(wire) and rd(opening_len_at) > 16 and rd(decide_len_at) > 16
    fields = [8, final_at] + [8 + 16 + 16 * i for i in range(lanes)] + [rounds_at + 16 * i for i in range(2 * rounds)]
    for at in fields:
        assert not ok(b=wire[:at] + _plus_one(wire[at: at + 16], field) + wire[at + 16:]), at
    for at in (opening_at + rd(opening_len_at) // 2, decide_at + rd(decide_len_at) // 2):
        assert not ok(b=wire[:at] + bytes([wire[at] ^ 1]) + wire[at + 1:]), at
    for at in (count_at, opening_len_at, decide_len_at):
        assert not ok(b=wire[:at] + b"\xff" * 8 + wire[at + 8:]), at
    assert not ok(b=wire[:24] + p.to_bytes(w, "little") + wire[24 + w:])
    for end in (0, 7, 8, count_at, final_at, opening_at, decide_at, len(wire) - 1):
        assert not ok(b=wire[:end]), end
    assert not ok(b=wire + b"\0")
    assert not ok(b=bytes([wire[0] ^ 1]) + wire[1:])
    with pytest.raises(oracle.OracleError, match="log_n"):
        oracle.packed_open(3, 4, 32, SEED, table(field, 3, 1), b"\0" * 48, CTX, field=field)


def wht(v, field):
    """Unnormalised Walsh-Hadamard transform of an (n, d) array, (a, b) -> (a + b, a - b)."""
    p = FIELDS[field][0]
    v = v.copy()
    h = 1
    while h < len(v):
        v = v.reshape(-1, 2, h, v.shape[-1])
        a, b = v[:, 0].copy(), v[:, 1].copy()
        v[:, 0], v[:, 1] = (a + b) % p, (a - b) % p
        v = v.reshape(-1, v.shape[-1])
        h *= 2
    return v


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
@pytest.mark.parametrize("log_n", [12, 16])
def test_top_code_encoding_is_the_index_two_systematic_code(field, log_n):
    """qafold_short.rs:975-1002: a column's codeword is the message followed
    by WHT(alpha (.) WHT(message)) with the code's alpha table."""
    rows = oracle.top_rows(log_n, field)
    msg = ext_point(field, rows, 20 + log_n)
    alpha, cw = oracle.encode_column(log_n, b"".join(ext_to_bytes(x, field) for x in msg), field=field)
    a = np.array([ext_from_bytes(x, field) for x in alpha])
    got = np.array([ext_from_bytes(x, field) for x in cw])
    assert np.array_equal(got[:rows], msg)
    assert np.array_equal(got[rows:], wht(ext_mul(wht(msg, field), a, field), field))


def _framed(label: bytes, data: bytes) -> bytes:
    return len(label).to_bytes(8, "little") + label + len(data).to_bytes(8, "little") + data


def _mobius(v, field):
    """high[i] -= low[i] at every level (packed.rs:708-752)."""
    p = FIELDS[field][0]
    v = v.copy()
    h = 1
    while h < len(v):
        v = v.reshape(-1, 2, h, v.shape[-1])
        v[:, 1] = (v[:, 1] - v[:, 0]) % p
        v = v.reshape(-1, v.shape[-1])
        h *= 2
    return v


def block_root(values, b, chunk_log, alpha, field):
    """A PCS block's commitment root from the definitions: pack the block's
    2^chunk_log entries into elements of `lanes` coefficients, Mobius
    transform, encode each of the 32 message columns, hash each codeword
    row (framed base-row domain, width, canonical values) and pair the
    digests under the framed inner domain (qafold_short_pc.rs:2372-2517)."""
    import hashlib
    p, lanes = FIELDS[field][0], FIELDS[field][1]
    n = 1 << chunk_log
    blk = np.zeros(n, dtype=np.int64)
    seg = values[b * n: (b + 1) * n].astype(np.int64)
    blk[: seg.size] = seg % p
    msg = _mobius(blk.reshape(-1, lanes), field)
    R = len(msg) // 32
    cols = [np.concatenate([msg[c * R:(c + 1) * R], wht(ext_mul(wht(msg[c * R:(c + 1) * R], field), alpha, field), field)])
            for c in range(32)]
    width = _framed(b"width", (32).to_bytes(8, "little"))
    dom = _framed(b"domain", b"qafold-short/base-row/v1")
    level = [hashlib.blake2s(dom + width + b"".join(ext_to_bytes(cols[c][r], field) for c in range(32))).digest()
             for r in range(2 * R)]
    inner = _framed(b"domain", b"qafold-short/merkle-inner/v1")
    while len(level) > 1:
        level = [hashlib.blake2s(inner + level[i] + level[i + 1]).digest() for i in range(0, len(level), 2)]
    return level[0]


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
def test_block_roots_from_the_definitions(field):
    """Every block root of a ragged collection, including the zero blocks past
    the active entries, recomputed in numpy and hashlib equals the oracle's."""
    from parcomm_b200 import layout
    dt = FIELDS[field][4]
    shapes = [(31, 37), (65, 17), (1, 7), (9, 1), (300, 40)]
    info = np.iinfo(dt)
    rng = np.random.default_rng(30)
    bva = layout.encode(shapes, [rng.integers(info.min, info.max + 1, size=s, dtype=dt) for s in shapes])
    for chunk_log in (10, 13):
        roots = oracle.commit_roots(shapes, chunk_log, 4, bva, field=field)
        rows = oracle.top_rows(chunk_log, field)
        alpha, _ = oracle.encode_column(chunk_log, bytes(16 * rows), field=field)
        a = np.array([ext_from_bytes(x, field) for x in alpha])
        blocks = layout.buckets(shapes)[2] >> chunk_log
        assert blocks >= 2
        for b in range(blocks):
            assert block_root(bva, b, chunk_log, a, field) == roots[32 * b: 32 * (b + 1)], (chunk_log, b)

"""Field known-answer tests (after vendor/qafold/tests/full_extension.rs:43-180
and the KoalaBear field's tests), from the definitions rather than the host
code: both moduli are prime; X^8 - 17 and X^4 - 3 are irreducible; the
Frobenius constants in the host headers are the powers they must be; and the
host field's product, inverse and Frobenius step (through the oracle library)
agree with a numpy restatement on random and extreme operands.  The device
field is checked against the host field by test_device_field.py."""
import re
from pathlib import Path

import numpy as np
import pytest

import oracle
from test_oracle_claims import FIELDS, ext_from_bytes, ext_mul, ext_to_bytes

ROOT = Path(__file__).resolve().parents[1]


def is_prime(n: int) -> bool:
    """Miller-Rabin with bases 2, 3, 5, 7: deterministic below 3,215,031,751."""
    if n < 2:
        return False
    for q in (2, 3, 5, 7):
        if n % q == 0:
            return n == q
    d, s = n - 1, 0
    while d % 2 == 0:
        d, s = d // 2, s + 1
    for a in (2, 3, 5, 7):
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
def test_modulus_prime_and_extension_irreducible(field):
    """X^n - a with n a power of two is irreducible over F_p when a is not a
    square and -4 is a square (Capelli: a lies in no K^2 and not in
    -4 K^4, which sits inside the squares when -4 is one)."""
    p, d, nr, _, _ = FIELDS[field]
    assert p < 3_215_031_751 and is_prime(p)
    assert (p - 1) % d == 0
    assert pow(nr, (p - 1) // 2, p) == p - 1
    assert pow(-4 % p, (p - 1) // 2, p) == 1


def test_frobenius_constants_in_the_headers():
    """X^p = X * a^((p-1)/n): the step multiplies coefficient i by (a^((p-1)/n))^i."""
    text = (ROOT / "parcomm_b200" / "csrc" / "host" / "field65521.h").read_text()
    omega = pow(17, (65521 - 1) // 8, 65521)
    assert omega == 57852 and pow(omega, 4, 65521) == 65520
    assert re.search(r"kFrobRoot\[8\] = \{1, %d," % omega, text)
    text = (ROOT / "parcomm_b200" / "csrc" / "host" / "fieldkb.h").read_text()
    p = 2130706433
    g = pow(3, (p - 1) // 4, p)
    phases = [pow(g, k, p) for k in range(4)]
    assert re.search(r"phases\[4\] = \{%s\}" % ", ".join(f"{v}u" for v in phases), text)


def operands(field, n, seed):
    p, d, _, _, _ = FIELDS[field]
    rng = np.random.default_rng(seed)
    a = rng.integers(0, p, size=(n, d), dtype=np.int64)
    extremes = [np.zeros(d, np.int64), np.eye(d, dtype=np.int64)[0], np.full(d, p - 1, np.int64)]
    for i in range(d):
        e = np.zeros(d, np.int64)
        e[i] = p - 1
        extremes += [e, np.eye(d, dtype=np.int64)[i]]
    return np.concatenate([np.array(extremes), a])


def ext_pow(a, e, field):
    r = np.zeros_like(a)
    r[:, 0] = 1
    while e:
        if e & 1:
            r = ext_mul(r, a, field)
        a = ext_mul(a, a, field)
        e >>= 1
    return r


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
def test_host_field_matches_the_definitions(field):
    p, d, _, _, _ = FIELDS[field]
    a = operands(field, 3000, 1)
    b = operands(field, 3000, 2)[::-1].copy()
    blob = lambda x: b"".join(ext_to_bytes(e, field) for e in x)
    prod, inv, frob = oracle.field_ops(blob(a), blob(b), field=field)
    split = lambda raw: np.array([ext_from_bytes(raw[16 * i: 16 * (i + 1)], field) for i in range(len(a))])
    prod, inv, frob = split(prod), split(inv), split(frob)
    assert np.array_equal(prod, ext_mul(a, b, field))
    nonzero = a.any(axis=1)
    one = np.zeros(d, np.int64)
    one[0] = 1
    assert (ext_mul(a[nonzero], inv[nonzero], field) == one).all()
    assert not inv[~nonzero].any()
    assert np.array_equal(frob, ext_pow(a.copy(), p, field))


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
def test_non_canonical_encoding_rejected(field):
    """full_extension.rs:181-218: a coefficient at or above p in any lane is
    refused (every such 16-bit value for F65521; p, p + 1 and 2^32 - 1 for
    KoalaBear), while p - 1 in every lane, an integer above the field's size,
    is a valid element."""
    p, d, _, w, _ = FIELDS[field]
    good = ext_to_bytes(np.ones(d, np.int64), field)
    invalid = range(p, 1 << 16) if w == 2 else (p, p + 1, (1 << 32) - 1)
    for i in range(d):
        for v in invalid:
            bad = bytearray(good)
            bad[w * i: w * (i + 1)] = v.to_bytes(w, "little")
            with pytest.raises(oracle.OracleError, match="non-canonical"):
                oracle.field_ops(bytes(bad), good, field=field)
    top = ext_to_bytes(np.full(d, p - 1, np.int64), field)
    assert oracle.field_ops(top, good, field=field)[0]


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
def test_products_of_edge_coefficients(field):
    """full_extension.rs:118-137: every pair of edge coefficient values, with
    one lane (or all) of the left factor set and the rest at p - 1."""
    p, d, _, _, _ = FIELDS[field]
    edge = [0, 1, 15, 32_760, 32_761, 65_519, 65_520] if field == "f65521" else [0, 1, 15, p // 2, p // 2 + 1, p - 2, p - 1]
    a, b = [], []
    for left in edge:
        for right in edge:
            for lane in range(d + 1):
                a.append([left if lane == d or i == lane else p - 1 for i in range(d)])
                b.append([right] * d)
    a, b = np.array(a, dtype=np.int64), np.array(b, dtype=np.int64)
    blob = lambda x: b"".join(ext_to_bytes(e, field) for e in x)
    prod, _, _ = oracle.field_ops(blob(a), blob(b), field=field)
    got = np.array([ext_from_bytes(prod[16 * i: 16 * (i + 1)], field) for i in range(len(a))])
    assert np.array_equal(got, ext_mul(a, b, field))

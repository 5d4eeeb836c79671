"""LogUp range audit on the CPU: the oracle against a pure-Python restatement
(hashlib BLAKE2s for alpha, big-integer field arithmetic, a Fermat
inversion), the identity on edge-value multisets, rejection of altered
multiplicities, the library's host table sum (batched inversion) against
the direct sum, and the C ABI's argument checks without a device."""
import ctypes
import hashlib
import struct

import numpy as np
import pytest

import oracle
import parcomm_b200 as qf

DOMAIN = b"parcomm-b200/logup-range-audit/v1"
FIELDS = {
    # name: (p, degree, X^d = w, entry dtype, field name, coefficient bytes)
    "f65521": (65521, 8, 17, np.int8, b"FullPrime65521Ext8/X^8-17/v1", 2),
    "koalabear": (2130706433, 4, 3, np.int16, b"FullKoalaBearExt4/X^4-3/scalar/v1", 4),
}


def frame(label: bytes, data: bytes) -> bytes:
    return struct.pack("<Q", len(label)) + label + struct.pack("<Q", len(data)) + data


class Ext:
    """F_p[X] / (X^d - w) with coefficient lists."""

    def __init__(self, p, d, w):
        self.p, self.d, self.w = p, d, w

    def mul(self, a, b):
        r = [0] * self.d
        for i, x in enumerate(a):
            for j, y in enumerate(b):
                if i + j < self.d:
                    r[i + j] += x * y
                else:
                    r[i + j - self.d] += self.w * x * y
        return [v % self.p for v in r]

    def add(self, a, b):
        return [(x + y) % self.p for x, y in zip(a, b)]

    def base(self, v):
        return [v % self.p] + [0] * (self.d - 1)

    def inv(self, a):
        e, r, b = self.p ** self.d - 2, self.base(1), list(a)
        while e:
            if e & 1:
                r = self.mul(r, b)
            b = self.mul(b, b)
            e >>= 1
        return r


def to_bytes(a, cb):
    return b"".join(int(v).to_bytes(cb, "little") for v in a)


def alpha_of(seed, field):
    p, d, _, _, name, cb = FIELDS[field]
    for counter in range(1000):
        h = hashlib.blake2s(frame(b"domain", DOMAIN) + frame(b"field", name) + frame(b"seed", seed)
                            + frame(b"counter", struct.pack("<Q", counter))).digest()
        words = [int.from_bytes(h[cb * i: cb * i + cb], "little") for i in range(d)]
        if cb == 4:
            words = [w & 0x7FFFFFFF for w in words]
        if all(w < p for w in words) and any(words[1:]):
            return words
    raise AssertionError("no alpha")


def restated(values, seed, field):
    p, d, w, dt, _, cb = FIELDS[field]
    E = Ext(p, d, w)
    a = alpha_of(seed, field)
    lo = -128 if dt == np.int8 else -32768
    mult = np.bincount(np.asarray(values, dtype=np.int64) - lo, minlength=256 if dt == np.int8 else 65536)
    lhs = E.base(0)
    for v in values:  # per value, as the definition reads
        lhs = E.add(lhs, E.inv(E.add(a, E.base(-int(v)))))
    rhs = E.base(0)
    for k in np.nonzero(mult)[0]:
        rhs = E.add(rhs, E.mul(E.base(int(mult[k])), E.inv(E.add(a, E.base(-(int(k) + lo))))))
    return mult.astype(np.uint64), to_bytes(a, cb), to_bytes(lhs, cb), to_bytes(rhs, cb)


def sample(field, n, seed):
    rng = np.random.default_rng(seed)
    dt = FIELDS[field][3]
    info = np.iinfo(dt)
    v = rng.integers(info.min, info.max + 1, size=n).astype(dt)
    v[:4] = [info.min, info.max, 0, -1]  # the table's ends and the wrap points
    return v


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
def test_oracle_matches_the_python_restatement(field):
    values = sample(field, 40, 3)
    seed = hashlib.blake2s(b"range-audit-pin-" + field.encode()).digest()
    mult, a, l, r = oracle.range_audit(values, seed, field)
    pm, pa, pl, pr = restated(values, seed, field)
    assert np.array_equal(mult, pm)
    assert (a, l, r) == (pa, pl, pr)
    assert l == r


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
def test_identity_on_edge_multisets(field):
    dt = FIELDS[field][3]
    info = np.iinfo(dt)
    seed = bytes(range(32))
    cases = [
        np.zeros(0, dtype=dt),                            # no values
        np.zeros(1000, dtype=dt),                         # one bin only
        np.full(70000, info.min, dtype=dt),               # a count above 2^16 in one bin
        np.arange(info.min, info.max + 1, dtype=np.int64).astype(dt),  # every table value once
        sample(field, 4099, 11),                          # a ragged length
    ]
    for v in cases:
        mult, _, l, r = oracle.range_audit(v, seed, field)
        assert int(mult.sum()) == v.size
        assert l == r


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
def test_altered_multiplicities_break_the_identity(field):
    """Moving one count to a neighbouring bin (the multiset of a value outside
    the data) changes the table side; the value side stays, so they differ."""
    p, d, w, dt, _, cb = FIELDS[field]
    E = Ext(p, d, w)
    values = sample(field, 25, 5)
    seed = b"\x07" * 32
    mult, a_b, l_b, _ = oracle.range_audit(values, seed, field)
    lo = -128 if dt == np.int8 else -32768
    a = [int.from_bytes(a_b[cb * i: cb * i + cb], "little") for i in range(d)]
    k = int(np.nonzero(mult)[0][0])
    bad = mult.copy()
    bad[k] -= 1
    bad[(k + 1) % bad.size] += 1
    rhs = E.base(0)
    for j in np.nonzero(bad)[0]:
        rhs = E.add(rhs, E.mul(E.base(int(bad[j])), E.inv(E.add(a, E.base(-(int(j) + lo))))))
    assert to_bytes(rhs, cb) != l_b


def test_capi_checks_arguments_without_a_device():
    L = qf.lib()
    holds = ctypes.c_int(7)
    rc = L.qf_range_audit(None, None, b"\x00" * 32, None, 0, None, None, None, ctypes.byref(holds))
    assert rc == qf.QF_E_ARGUMENT and holds.value == 7


def test_host_table_sum_batched_inversion(tmp_path):
    """The library's host table sum (one batched inversion) against the direct
    per-term sum, both fields, compiled with the host compiler."""
    import json
    import subprocess
    from pathlib import Path
    src = Path(__file__).resolve().parent / "range_audit_check.cpp"
    exe = tmp_path / "range_audit_check"
    subprocess.run(["/usr/bin/g++", "-std=c++17", "-O2", str(src), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert r.returncode == 0 and out["mismatches"] == 0 and out["checked"] == 48, out

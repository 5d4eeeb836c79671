"""The host BLAKE2s-256 (transcripts, Merkle leaves and nodes, setup
digests) against Python's hashlib.blake2s (RFC 7693): every length around
the 64-byte block boundaries, long inputs, and the same data fed in pieces
of every size pattern; the SSSE3 and scalar compressions agree on random
states and blocks, last-block flag set and clear."""
import hashlib
import platform

import numpy as np
import pytest

import oracle


def test_lengths_around_block_boundaries():
    rng = np.random.default_rng(1)
    for n in list(range(0, 260)) + [511, 512, 513, 1000, 4095, 4096, 4097, 65537, (1 << 20) + 3]:
        data = rng.integers(0, 256, size=n, dtype=np.uint8).tobytes()
        assert oracle.blake2s_stream(data) == hashlib.blake2s(data).digest(), n


def test_pieces_of_any_size_give_the_same_digest():
    rng = np.random.default_rng(2)
    data = rng.integers(0, 256, size=5000, dtype=np.uint8).tobytes()
    want = hashlib.blake2s(data).digest()
    for pattern in ([64] * 78, [1] * 200, [63, 65] * 30, [128, 0, 0, 64], [4999], [0, 5000]):
        cuts = np.cumsum(pattern)
        cuts = cuts[cuts <= len(data)]
        assert oracle.blake2s_stream(data, cuts) == want, pattern
    for _ in range(50):
        cuts = np.sort(rng.integers(0, len(data) + 1, size=int(rng.integers(1, 40))))
        assert oracle.blake2s_stream(data, cuts) == want


@pytest.mark.skipif(platform.machine() not in ("x86_64", "AMD64"), reason="SSSE3 is an x86-64 path")
def test_ssse3_and_scalar_compressions_agree():
    rng = np.random.default_rng(3)
    for i in range(500):
        h = rng.integers(0, 1 << 32, size=8, dtype=np.uint64).astype(np.uint32)
        block = rng.integers(0, 256, size=64, dtype=np.uint8).tobytes()
        t = int(rng.integers(0, 1 << 62)) if i % 2 else int(rng.integers(1, 1 << 16))
        last = bool(i % 3 == 0)
        a = oracle.blake2s_compress(h, block, t, last, ssse3=False)
        b = oracle.blake2s_compress(h, block, t, last, ssse3=True)
        assert np.array_equal(a, b), i
        assert not np.array_equal(a, h)

"""The setup's generator, rand 0.8's StdRng, restated in Python from the
published algorithms and compared with the host C++ generator.

- ChaCha with 12 rounds (rand_chacha 0.3): the constants, the 256-bit key,
  a 64-bit block counter in words 12-13 and a zero stream id in words 14-15.
  The Python block function is checked at 20 rounds against the
  `cryptography` package's ChaCha20 first.
- rand_core 0.6's block buffer: next_u32 takes the next output word,
  next_u64 the next two (low word first), and fill_bytes(n) the next
  ceil(n / 4) words, of which the first n bytes are written.
- seed_from_u64: PCG32 output words fill the 32-byte seed.
The setup seed draw (StdRng::from_seed([0x51; 32]).fill_bytes of 32 bytes)
and the wire fixture's seed_from_u64 generator are among the cases."""
import struct

import numpy as np
import pytest
from cryptography.hazmat.primitives.ciphers import Cipher, algorithms

import oracle

M32 = 0xFFFFFFFF


def _rotl(x, n):
    return ((x << n) | (x >> (32 - n))) & M32


def chacha_block(key_words, counter, rounds):
    s = [0x61707865, 0x3320646E, 0x79622D32, 0x6B206574] + list(key_words) + [counter & M32, counter >> 32, 0, 0]
    x = list(s)

    def qr(a, b, c, d):
        x[a] = (x[a] + x[b]) & M32; x[d] = _rotl(x[d] ^ x[a], 16)
        x[c] = (x[c] + x[d]) & M32; x[b] = _rotl(x[b] ^ x[c], 12)
        x[a] = (x[a] + x[b]) & M32; x[d] = _rotl(x[d] ^ x[a], 8)
        x[c] = (x[c] + x[d]) & M32; x[b] = _rotl(x[b] ^ x[c], 7)

    for _ in range(rounds // 2):
        qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15)
        qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14)
    return [(a + b) & M32 for a, b in zip(x, s)]


def pcg32_seed(state):
    out = b""
    for _ in range(8):
        state = (state * 6364136223846793005 + 11634580027462260723) % (1 << 64)
        xorshifted = (((state >> 18) ^ state) >> 27) & M32
        rot = state >> 59
        out += (((xorshifted >> rot) | (xorshifted << ((32 - rot) & 31))) & M32).to_bytes(4, "little")
    return out


class PyStdRng:
    def __init__(self, seed: bytes):
        self.key = struct.unpack("<8I", seed)
        self.words, self.counter = [], 0

    def _word(self):
        if not self.words:
            self.words = chacha_block(self.key, self.counter, 12)
            self.counter += 1
        return self.words.pop(0)

    def draw(self, op):
        if op == -1:
            return self._word().to_bytes(4, "little")
        if op == -2:
            lo = self._word()
            return (lo | (self._word() << 32)).to_bytes(8, "little")
        return b"".join(self._word().to_bytes(4, "little") for _ in range((op + 3) // 4))[:op]


def test_python_chacha_matches_cryptography_chacha20():
    key = bytes(range(7, 39))
    kw = struct.unpack("<8I", key)
    for counter in (0, 1, 5, 1000):
        nonce = counter.to_bytes(4, "little") + bytes(12)
        stream = Cipher(algorithms.ChaCha20(key, nonce), mode=None).encryptor().update(bytes(64))
        assert struct.pack("<16I", *chacha_block(kw, counter, 20)) == stream


@pytest.mark.parametrize("seed_kind", ["setup", "random", "u64"])
def test_host_stdrng_matches_the_restatement(seed_kind):
    rng = np.random.default_rng(4)
    ops = [int(v) for v in rng.choice([-1, -2, 1, 3, 4, 7, 32, 61, 64, 255, 256, 300], size=400)]
    ops = [32] + ops  # the setup draw first
    if seed_kind == "u64":
        u = 0x706172616C6C656C  # the wire fixture's seed (qafold_short_pc.rs:3605-3614)
        host = oracle.stdrng(ops, seed_u64=u)
        py = PyStdRng(pcg32_seed(u))
    else:
        seed = bytes([0x51]) * 32 if seed_kind == "setup" else rng.integers(0, 256, 32, dtype=np.uint8).tobytes()
        host = oracle.stdrng(ops, seed=seed)
        py = PyStdRng(seed)
    assert host == b"".join(py.draw(op) for op in ops)

"""Julia-compatible random stream: SHA-256 known answers (FIPS 180-4 via
hashlib), seeding and the xoshiro256++ stream against the oracle restatement."""
import hashlib

import numpy as np
import pytest

from acgpu._lib import lib
from julia_rng import JuliaRng, make_seed


@pytest.mark.parametrize("msg", [b"", b"abc", b"\x01\x00\x00\x00", bytes(range(64)), bytes(range(200)) * 3])
def test_sha256_known_answers(msg):
    out = np.zeros(32, np.uint8)
    buf = np.frombuffer(msg, dtype=np.uint8).copy() if msg else np.zeros(1, np.uint8)
    assert lib().acg_sha256(buf, len(msg), out) == 0
    assert bytes(out) == hashlib.sha256(msg).digest()


def test_make_seed_limbs():
    assert make_seed(1) == b"\x01\x00\x00\x00"
    assert make_seed(2 ** 32 + 5) == b"\x05\x00\x00\x00\x01\x00\x00\x00"


@pytest.mark.parametrize("seed", [0, 1, 42, 2 ** 32 + 7, 2 ** 63 + 11])
def test_stream_matches_restatement(seed):
    st = np.zeros(4, np.uint64)
    assert lib().acg_rng_seed(seed, st) == 0
    ref = JuliaRng(seed)
    assert [int(x) for x in st] == ref.s
    out = np.zeros(1000)
    assert lib().acg_rng_rand(st, out, out.size) == 0
    exp = np.array([ref.rand() for _ in range(1000)])
    assert np.array_equal(out, exp)
    assert np.all((out >= 0) & (out < 1))

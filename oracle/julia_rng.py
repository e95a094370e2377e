"""ORACLE — test infrastructure only (checker, never shipped or measured).

Pure-Python restatement of Julia 1.8's default random stream (stdlib Random,
pinned by the reference's Manifest.toml julia_version = 1.8.5), independent of
the product's C++ one:
  * `Random.seed!(k)`: `make_seed(k)` = k as 32-bit little-endian limbs,
    SHA-256 of those bytes (hashlib here), digest read as 4 LE UInt64 words;
  * xoshiro256++ step;  * `rand()` = (next >> 11) * 2^-53.
Used by the approxChol restatement (src/approxChol.jl:917 calls rand()).
"""
from __future__ import annotations

import hashlib
import struct

MASK = (1 << 64) - 1


def make_seed(k: int) -> bytes:
    if k < 0:
        raise ValueError("seed must be non-negative")
    out = b""
    while True:
        out += struct.pack("<I", k & 0xFFFFFFFF)
        k >>= 32
        if k == 0:
            return out


class JuliaRng:
    def __init__(self, seed: int | None = None, state=None):
        if state is not None:
            self.s = [int(x) & MASK for x in state]
        else:
            self.seed(0 if seed is None else seed)

    def seed(self, k: int):
        dig = hashlib.sha256(make_seed(k)).digest()
        self.s = list(struct.unpack("<4Q", dig))

    def next_u64(self) -> int:
        s0, s1, s2, s3 = self.s
        tmp = (s0 + s3) & MASK
        res = ((((tmp << 23) | (tmp >> 41)) & MASK) + s0) & MASK
        t = (s1 << 17) & MASK
        s2 ^= s0
        s3 ^= s1
        s1 ^= s2
        s0 ^= s3
        s2 ^= t
        s3 = ((s3 << 45) | (s3 >> 19)) & MASK
        self.s = [s0, s1, s2, s3]
        return res

    def rand(self) -> float:
        return float(self.next_u64() >> 11) * (2.0 ** -53)

// Julia-compatible global random stream used by the host elimination.
//
// The reference draws its samples with Julia's global `rand()`
// (src/approxChol.jl:917), i.e. the task-local Xoshiro256++ generator of the
// Julia 1.8 `Random` stdlib (Manifest.toml julia_version 1.8.5), seeded by
// `Random.seed!(k)`.  This header restates that generator so that the same
// seed drives the same stream of doubles:
//   * seed!(k::Integer): the seed is split into 32-bit little-endian limbs
//     (`make_seed`), hashed with SHA-256, and the 32-byte digest is read as
//     four little-endian UInt64 words s0..s3.
//   * next UInt64: xoshiro256++ (Blackman & Vigna), res = rotl(s0+s3,23)+s0.
//   * rand() :: Float64 in [0,1): (next >> 11) * 2^-53.
#pragma once
#include <cstdint>
#include <cstddef>

namespace acg {

struct JuliaRng {
  uint64_t s[4];
};

// SHA-256 of `len` bytes (FIPS 180-4), digest written to out[32].
void sha256(const uint8_t* data, size_t len, uint8_t out[32]);

// Random.seed!(rng, seed) for a non-negative integer seed.
void julia_seed(JuliaRng* rng, uint64_t seed);

inline uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

inline uint64_t julia_next_u64(JuliaRng* r) {
  uint64_t s0 = r->s[0], s1 = r->s[1], s2 = r->s[2], s3 = r->s[3];
  uint64_t res = rotl64(s0 + s3, 23) + s0;
  uint64_t t = s1 << 17;
  s2 ^= s0;
  s3 ^= s1;
  s1 ^= s2;
  s0 ^= s3;
  s2 ^= t;
  s3 = rotl64(s3, 45);
  r->s[0] = s0; r->s[1] = s1; r->s[2] = s2; r->s[3] = s3;
  return res;
}

inline double julia_rand(JuliaRng* r) {
  return (double)(julia_next_u64(r) >> 11) * 0x1.0p-53;
}

}  // namespace acg

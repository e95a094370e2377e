// SHA-256 (FIPS 180-4) and the Julia 1.8 `Random.seed!` restatement.
#include "acg_rng.h"

#include <cstring>
#include <vector>

namespace acg {

namespace {

const uint32_t kRoundK[64] = {
    0x428a2f98u, 0x71374491u, 0xb5c0fbcfu, 0xe9b5dba5u, 0x3956c25bu, 0x59f111f1u, 0x923f82a4u,
    0xab1c5ed5u, 0xd807aa98u, 0x12835b01u, 0x243185beu, 0x550c7dc3u, 0x72be5d74u, 0x80deb1feu,
    0x9bdc06a7u, 0xc19bf174u, 0xe49b69c1u, 0xefbe4786u, 0x0fc19dc6u, 0x240ca1ccu, 0x2de92c6fu,
    0x4a7484aau, 0x5cb0a9dcu, 0x76f988dau, 0x983e5152u, 0xa831c66du, 0xb00327c8u, 0xbf597fc7u,
    0xc6e00bf3u, 0xd5a79147u, 0x06ca6351u, 0x14292967u, 0x27b70a85u, 0x2e1b2138u, 0x4d2c6dfcu,
    0x53380d13u, 0x650a7354u, 0x766a0abbu, 0x81c2c92eu, 0x92722c85u, 0xa2bfe8a1u, 0xa81a664bu,
    0xc24b8b70u, 0xc76c51a3u, 0xd192e819u, 0xd6990624u, 0xf40e3585u, 0x106aa070u, 0x19a4c116u,
    0x1e376c08u, 0x2748774cu, 0x34b0bcb5u, 0x391c0cb3u, 0x4ed8aa4au, 0x5b9cca4fu, 0x682e6ff3u,
    0x748f82eeu, 0x78a5636fu, 0x84c87814u, 0x8cc70208u, 0x90befffau, 0xa4506cebu, 0xbef9a3f7u,
    0xc67178f2u};

inline uint32_t rotr32(uint32_t x, int k) { return (x >> k) | (x << (32 - k)); }

void compress_block(uint32_t h[8], const uint8_t* blk) {
  uint32_t w[64];
  for (int t = 0; t < 16; ++t)
    w[t] = (uint32_t)blk[4 * t] << 24 | (uint32_t)blk[4 * t + 1] << 16 |
           (uint32_t)blk[4 * t + 2] << 8 | (uint32_t)blk[4 * t + 3];
  for (int t = 16; t < 64; ++t) {
    uint32_t s0 = rotr32(w[t - 15], 7) ^ rotr32(w[t - 15], 18) ^ (w[t - 15] >> 3);
    uint32_t s1 = rotr32(w[t - 2], 17) ^ rotr32(w[t - 2], 19) ^ (w[t - 2] >> 10);
    w[t] = w[t - 16] + s0 + w[t - 7] + s1;
  }
  uint32_t a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], hh = h[7];
  for (int t = 0; t < 64; ++t) {
    uint32_t S1 = rotr32(e, 6) ^ rotr32(e, 11) ^ rotr32(e, 25);
    uint32_t ch = (e & f) ^ (~e & g);
    uint32_t t1 = hh + S1 + ch + kRoundK[t] + w[t];
    uint32_t S0 = rotr32(a, 2) ^ rotr32(a, 13) ^ rotr32(a, 22);
    uint32_t mj = (a & b) ^ (a & c) ^ (b & c);
    uint32_t t2 = S0 + mj;
    hh = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + t2;
  }
  h[0] += a; h[1] += b; h[2] += c; h[3] += d; h[4] += e; h[5] += f; h[6] += g; h[7] += hh;
}

}  // namespace

void sha256(const uint8_t* data, size_t len, uint8_t out[32]) {
  uint32_t h[8] = {0x6a09e667u, 0xbb67ae85u, 0x3c6ef372u, 0xa54ff53au,
                   0x510e527fu, 0x9b05688cu, 0x1f83d9abu, 0x5be0cd19u};
  size_t full = len / 64;
  for (size_t b = 0; b < full; ++b) compress_block(h, data + 64 * b);
  // Padding: 0x80, zeros, 64-bit big-endian bit length.
  uint8_t tail[128];
  size_t rem = len - 64 * full;
  std::memset(tail, 0, sizeof(tail));
  if (rem) std::memcpy(tail, data + 64 * full, rem);
  tail[rem] = 0x80;
  size_t tail_len = (rem + 1 + 8 <= 64) ? 64 : 128;
  uint64_t bits = (uint64_t)len * 8u;
  for (int k = 0; k < 8; ++k) tail[tail_len - 1 - k] = (uint8_t)(bits >> (8 * k));
  compress_block(h, tail);
  if (tail_len == 128) compress_block(h, tail + 64);
  for (int k = 0; k < 8; ++k) {
    out[4 * k] = (uint8_t)(h[k] >> 24);
    out[4 * k + 1] = (uint8_t)(h[k] >> 16);
    out[4 * k + 2] = (uint8_t)(h[k] >> 8);
    out[4 * k + 3] = (uint8_t)h[k];
  }
}

void julia_seed(JuliaRng* rng, uint64_t seed) {
  // make_seed: 32-bit limbs, least significant first, at least one limb.
  std::vector<uint8_t> bytes;
  uint64_t v = seed;
  do {
    uint32_t limb = (uint32_t)(v & 0xffffffffu);
    for (int k = 0; k < 4; ++k) bytes.push_back((uint8_t)(limb >> (8 * k)));
    v >>= 32;
  } while (v != 0);
  uint8_t dig[32];
  sha256(bytes.data(), bytes.size(), dig);
  for (int w = 0; w < 4; ++w) {
    uint64_t x = 0;
    for (int k = 0; k < 8; ++k) x |= (uint64_t)dig[8 * w + k] << (8 * k);
    rng->s[w] = x;
  }
}

}  // namespace acg

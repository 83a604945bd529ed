// oracle/chacha.hpp — ChaCha12 first-output restatement of rand 0.8 StdRng.
//
// TEST INFRASTRUCTURE ONLY (part of the oracle; never linked into the product).
//
// rand 0.8.5 StdRng = rand_chacha 0.3.1 ChaCha12Rng (pinned in
// stark-stir-swarm/Cargo.lock, not vendored). from_seed(seed) uses the 32 seed
// bytes as the key (8 LE words), a 64-bit block counter starting at 0 in state
// words 12-13 and a zero 64-bit stream id in words 14-15 (D. J. Bernstein's
// ChaCha layout, 6 double rounds). gen::<u64>() on a fresh generator returns
// word0 | word1 << 32 of block 0. Call site: fri.rs:1044-1051 (index_from_seed).
// Pinned only by the golden proofs' raw_query_index fields.
#pragma once
#include <cstdint>
#include <cstring>

namespace orc {

inline uint32_t rotl32(uint32_t x, unsigned r) { return (x << r) | (x >> (32 - r)); }

inline void chacha_block(const uint32_t key[8], uint64_t counter, uint64_t stream, int rounds,
                         uint32_t out[16]) {
  uint32_t s[16] = {0x61707865u, 0x3320646eu, 0x79622d32u, 0x6b206574u, key[0], key[1], key[2], key[3],
                    key[4],      key[5],      key[6],      key[7],      (uint32_t)counter,
                    (uint32_t)(counter >> 32), (uint32_t)stream, (uint32_t)(stream >> 32)};
  uint32_t x[16];
  memcpy(x, s, sizeof x);
#define ORC_QR(a, b, c, d)            \
  x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 16); \
  x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 12); \
  x[a] += x[b]; x[d] = rotl32(x[d] ^ x[a], 8);  \
  x[c] += x[d]; x[b] = rotl32(x[b] ^ x[c], 7);
  for (int r = 0; r < rounds; r += 2) {
    ORC_QR(0, 4, 8, 12) ORC_QR(1, 5, 9, 13) ORC_QR(2, 6, 10, 14) ORC_QR(3, 7, 11, 15)
    ORC_QR(0, 5, 10, 15) ORC_QR(1, 6, 11, 12) ORC_QR(2, 7, 8, 13) ORC_QR(3, 4, 9, 14)
  }
#undef ORC_QR
  for (int i = 0; i < 16; ++i) out[i] = x[i] + s[i];
}

// StdRng::from_seed(seed).gen::<u64>()
inline uint64_t stdrng_first_u64(const uint8_t seed[32]) {
  uint32_t key[8];
  for (int i = 0; i < 8; ++i) memcpy(&key[i], seed + 4 * i, 4);
  uint32_t out[16];
  chacha_block(key, 0, 0, 12, out);
  return (uint64_t)out[0] | ((uint64_t)out[1] << 32);
}

}  // namespace orc

// oracle/keccak.hpp — CPU Keccak-f[1600] and streaming SHA3-256/384/512.
//
// TEST INFRASTRUCTURE ONLY (part of the oracle; never linked into the product).
//
// sha3 0.10.8 / keccak 0.1.6 (pinned in stark-stir-swarm/Cargo.lock, not vendored)
// implement FIPS 202; this restates FIPS 202 directly: rate 200 - 2d bytes for
// a d-byte digest (136 for SHA3-256), domain padding 0x06 ... 0x80. Callers in the reference:
// merkle/src/lib.rs:197-216,232-237 (tree nodes), transcript/src/lib.rs:158-213
// (Fiat-Shamir), fri.rs:1035-1066 (tree-domain hashes). Pinned by
// hashlib.sha3_256 in tests and by the golden proofs.
#pragma once
#include <cstdint>
#include <cstring>

namespace orc {

inline uint64_t rotl64(uint64_t x, unsigned r) { return r ? (x << r) | (x >> (64 - r)) : x; }

inline void keccak_f1600(uint64_t s[25]) {
  static const uint64_t RC[24] = {
      0x0000000000000001ull, 0x0000000000008082ull, 0x800000000000808Aull, 0x8000000080008000ull,
      0x000000000000808Bull, 0x0000000080000001ull, 0x8000000080008081ull, 0x8000000000008009ull,
      0x000000000000008Aull, 0x0000000000000088ull, 0x0000000080008009ull, 0x000000008000000Aull,
      0x000000008000808Bull, 0x800000000000008Bull, 0x8000000000008089ull, 0x8000000000008003ull,
      0x8000000000008002ull, 0x8000000000000080ull, 0x000000000000800Aull, 0x800000008000000Aull,
      0x8000000080008081ull, 0x8000000000008080ull, 0x0000000080000001ull, 0x8000000080008008ull};
  // rotation offsets r[x][y] for lane index x + 5y
  static const unsigned ROT[25] = {0, 1, 62, 28, 27, 36, 44, 6, 55, 20, 3, 10, 43,
                                   25, 39, 41, 45, 15, 21, 8, 18, 2, 61, 56, 14};
  for (int round = 0; round < 24; ++round) {
    uint64_t C[5], D[5], B[25];
    for (int x = 0; x < 5; ++x) C[x] = s[x] ^ s[x + 5] ^ s[x + 10] ^ s[x + 15] ^ s[x + 20];
    for (int x = 0; x < 5; ++x) D[x] = C[(x + 4) % 5] ^ rotl64(C[(x + 1) % 5], 1);
    for (int i = 0; i < 25; ++i) s[i] ^= D[i % 5];
    // rho + pi: B[y, 2x+3y] = rot(A[x,y], r[x,y])
    for (int x = 0; x < 5; ++x)
      for (int y = 0; y < 5; ++y) B[y + 5 * ((2 * x + 3 * y) % 5)] = rotl64(s[x + 5 * y], ROT[x + 5 * y]);
    // chi
    for (int x = 0; x < 5; ++x)
      for (int y = 0; y < 5; ++y)
        s[x + 5 * y] = B[x + 5 * y] ^ (~B[(x + 1) % 5 + 5 * y] & B[(x + 2) % 5 + 5 * y]);
    s[0] ^= RC[round];
  }
}

// Streaming SHA3 with an OUT-byte digest (rate 200 - 2 OUT bytes); copyable,
// since the transcript clones it to squeeze.
template <int OUT>
struct Sha3 {
  static constexpr int RATE = 200 - 2 * OUT;
  uint64_t st[25];
  uint8_t buf[RATE];
  size_t fill;
  Sha3() { reset(); }
  void reset() {
    memset(st, 0, sizeof st);
    fill = 0;
  }
  void absorb_block(const uint8_t* blk) {
    for (int i = 0; i < RATE / 8; ++i) {
      uint64_t w;
      memcpy(&w, blk + 8 * i, 8);  // little-endian host assumed (x86-64)
      st[i] ^= w;
    }
    keccak_f1600(st);
  }
  void update(const void* data, size_t len) {
    const uint8_t* p = (const uint8_t*)data;
    while (len) {
      size_t take = RATE - fill;
      if (take > len) take = len;
      memcpy(buf + fill, p, take);
      fill += take;
      p += take;
      len -= take;
      if (fill == (size_t)RATE) {
        absorb_block(buf);
        fill = 0;
      }
    }
  }
  void finalize(uint8_t out[OUT]) const {
    Sha3 c = *this;
    memset(c.buf + c.fill, 0, RATE - c.fill);
    c.buf[c.fill] ^= 0x06;
    c.buf[RATE - 1] ^= 0x80;
    c.absorb_block(c.buf);
    memcpy(out, c.st, OUT);
  }
};
using Sha3_256 = Sha3<32>;

// The hash profile of the Merkle channel and the Fiat-Shamir transcript: the
// reference picks it at compile time (hash/src/selected.rs:8-48, HASH_BYTES 32 /
// 48 / 64 for the sha3-256 / sha3-384 / sha3-512 features); so does this build.
#ifndef ORC_HASH_BYTES
#define ORC_HASH_BYTES 32
#endif
static_assert(ORC_HASH_BYTES == 32 || ORC_HASH_BYTES == 48 || ORC_HASH_BYTES == 64, "SHA3-256/384/512 only");
constexpr int HASH_BYTES = ORC_HASH_BYTES;
using SelectedHasher = Sha3<HASH_BYTES>;

inline void sha3_256(const void* data, size_t len, uint8_t out[32]) {
  Sha3_256 h;
  h.update(data, len);
  h.finalize(out);
}

}  // namespace orc

// keccak.cuh — Keccak-f[1600] and SHA3-256/384/512 (FIPS 202) for host and device.
//
// The reference hashes every Merkle leaf/node, its transcript and its tree
// domain tags with the hasher its hash feature selects at compile time
// (hash/src/selected.rs:8-48: Sha3_256, Sha3_384 or Sha3_512 from sha3 0.10.8;
// merkle/src/lib.rs:185-238, transcript/src/lib.rs:162-212). This library does
// the same with SG_HASH_BYTES (32, the default, 48 or 64): a d-byte SHA3 absorbs
// 200 - 2d byte blocks (17, 13 or 9 lanes) and pads with 0x06 .. 0x80. DNS record
// hashing and the pi_hash recipes use SHA3-256 in every build
// (swarm-dns/src/dns.rs:17, prover.rs:207).
//
// On the device the 25-lane state lives in registers; each 64-bit XOR/rotate
// lowers to 32-bit LOP3/SHF pairs, except half of the rho rotations, which are
// written as IMAD products (4 % more permutations per second on B200). Messages in this library are built from
// whole 64-bit lanes (32-byte labels, 8-byte field elements, whole-lane digests),
// so lane-granular absorption is all the kernels need.
#pragma once
#include <cstdint>
#include <cstring>

#if defined(__CUDACC__)
#define KC_HD __host__ __device__ __forceinline__
#else
#define KC_HD inline
#endif

#ifndef SG_HASH_BYTES
#define SG_HASH_BYTES 32
#endif
static_assert(SG_HASH_BYTES == 32 || SG_HASH_BYTES == 48 || SG_HASH_BYTES == 64, "SHA3-256, -384 or -512");

namespace kc {

// The Merkle / transcript hash profile of this build.
constexpr int kHashBytes = SG_HASH_BYTES;
constexpr int kDigestLanes = kHashBytes / 8;
constexpr int kRateLanes = (200 - 2 * kHashBytes) / 8;

KC_HD uint64_t rotl(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }

#if defined(__CUDACC__)
__constant__ static const uint64_t kRC_dev[24] = {
#else
static const uint64_t kRC_dev[24] = {
#endif
    0x0000000000000001ull, 0x0000000000008082ull, 0x800000000000808Aull, 0x8000000080008000ull,
    0x000000000000808Bull, 0x0000000080000001ull, 0x8000000080008081ull, 0x8000000000008009ull,
    0x000000000000008Aull, 0x0000000000000088ull, 0x0000000080008009ull, 0x000000008000000Aull,
    0x000000008000808Bull, 0x800000000000008Bull, 0x8000000000008089ull, 0x8000000000008003ull,
    0x8000000000008002ull, 0x8000000000000080ull, 0x000000000000800Aull, 0x800000008000000Aull,
    0x8000000080008081ull, 0x8000000000008080ull, 0x0000000080000001ull, 0x8000000080008008ull};

static const uint64_t kRC_host[24] = {
    0x0000000000000001ull, 0x0000000000008082ull, 0x800000000000808Aull, 0x8000000080008000ull,
    0x000000000000808Bull, 0x0000000080000001ull, 0x8000000080008081ull, 0x8000000000008009ull,
    0x000000000000008Aull, 0x0000000000000088ull, 0x0000000080008009ull, 0x000000008000000Aull,
    0x000000008000808Bull, 0x800000000000008Bull, 0x8000000000008089ull, 0x8000000000008003ull,
    0x8000000000008002ull, 0x8000000000000080ull, 0x000000000000800Aull, 0x800000008000000Aull,
    0x8000000080008081ull, 0x8000000000008080ull, 0x0000000080000001ull, 0x8000000080008008ull};

#if defined(__CUDACC__)
// 2^r (r < 32) in constant memory, opaque to the compiler, so that a rotation
// written as products stays on the FMA pipe (four IMADs) instead of the ALU pipe
// (two funnel shifts). Half of the rho rotations take this form: the ALU pipe is
// the bottleneck of the permutation and the FMA pipe is otherwise idle.
__constant__ static const uint32_t kRotMul[32] = {
    1u << 0,  1u << 1,  1u << 2,  1u << 3,  1u << 4,  1u << 5,  1u << 6,  1u << 7,
    1u << 8,  1u << 9,  1u << 10, 1u << 11, 1u << 12, 1u << 13, 1u << 14, 1u << 15,
    1u << 16, 1u << 17, 1u << 18, 1u << 19, 1u << 20, 1u << 21, 1u << 22, 1u << 23,
    1u << 24, 1u << 25, 1u << 26, 1u << 27, 1u << 28, 1u << 29, 1u << 30, 1u << 31};
template <int R>
__device__ __forceinline__ uint64_t rotl_fma(uint64_t x) {
  uint32_t lo = (uint32_t)x, hi = (uint32_t)(x >> 32);
  if constexpr (R >= 32) {
    const uint32_t t = lo;
    lo = hi;
    hi = t;
  }
  constexpr int r = R & 31;
  if constexpr (r == 0) {
    return (uint64_t)hi << 32 | lo;
  } else {
    uint32_t nlo, nhi;
    asm("{\n\t.reg .u32 t0, t1;\n\t"
        "mul.hi.u32 t0, %3, %4;\n\tmad.lo.u32 %0, %2, %4, t0;\n\t"
        "mul.hi.u32 t1, %2, %4;\n\tmad.lo.u32 %1, %3, %4, t1;\n\t}"
        : "=r"(nlo), "=r"(nhi)
        : "r"(lo), "r"(hi), "r"(kRotMul[r]));
    return (uint64_t)nhi << 32 | nlo;
  }
}
#endif
#if defined(__CUDA_ARCH__)
#define KC_ROT_B(x, R) kc::rotl_fma<R>(x)
#else
#define KC_ROT_B(x, R) kc::rotl(x, R)
#endif

// a ^ b ^ c. On the device each 32-bit half is one three-input LOP3, so theta's
// "A[x][y] ^= C[x-1] ^ rot(C[x+1], 1)" costs one instruction per half and lane
// (the two-step form, D[x] first, costs 10 more per round).
KC_HD uint64_t xor3(uint64_t a, uint64_t b, uint64_t c) {
#if defined(__CUDA_ARCH__)
  uint32_t lo, hi;
  asm("lop3.b32 %0, %1, %2, %3, 0x96;" : "=r"(lo) : "r"((uint32_t)a), "r"((uint32_t)b), "r"((uint32_t)c));
  asm("lop3.b32 %0, %1, %2, %3, 0x96;"
      : "=r"(hi)
      : "r"((uint32_t)(a >> 32)), "r"((uint32_t)(b >> 32)), "r"((uint32_t)(c >> 32)));
  return (uint64_t)hi << 32 | lo;
#else
  return a ^ b ^ c;
#endif
}

// a ^ (~b & c), Keccak's chi, as one LOP3 per 32-bit half on the device.
KC_HD uint64_t chi(uint64_t a, uint64_t b, uint64_t c) {
#if defined(__CUDA_ARCH__)
  uint32_t lo, hi;
  asm("lop3.b32 %0, %1, %2, %3, 0xD2;" : "=r"(lo) : "r"((uint32_t)a), "r"((uint32_t)b), "r"((uint32_t)c));
  asm("lop3.b32 %0, %1, %2, %3, 0xD2;"
      : "=r"(hi)
      : "r"((uint32_t)(a >> 32)), "r"((uint32_t)(b >> 32)), "r"((uint32_t)(c >> 32)));
  return (uint64_t)hi << 32 | lo;
#else
  return a ^ (~b & c);
#endif
}

// One round on a register-resident state (theta, rho+pi, chi, iota). With
// R[x] = rot(C[x], 1), theta's D[x] = C[x-1] ^ R[x+1] is folded into each lane's
// update as xor3(A, C[x-1], R[x+1]). The rho rotations of B2, B4, ..., B24 go
// through KC_ROT_B (see above).
#define KC_ROUND(A, rc)                                                         \
  {                                                                             \
    uint64_t C0 = kc::xor3(kc::xor3(A[0], A[5], A[10]), A[15], A[20]);          \
    uint64_t C1 = kc::xor3(kc::xor3(A[1], A[6], A[11]), A[16], A[21]);          \
    uint64_t C2 = kc::xor3(kc::xor3(A[2], A[7], A[12]), A[17], A[22]);          \
    uint64_t C3 = kc::xor3(kc::xor3(A[3], A[8], A[13]), A[18], A[23]);          \
    uint64_t C4 = kc::xor3(kc::xor3(A[4], A[9], A[14]), A[19], A[24]);          \
    uint64_t R0 = kc::rotl(C0, 1), R1 = kc::rotl(C1, 1), R2 = kc::rotl(C2, 1);  \
    uint64_t R3 = kc::rotl(C3, 1), R4 = kc::rotl(C4, 1);                        \
    uint64_t B0 = kc::xor3(A[0], C4, R1);                                       \
    uint64_t B1 = kc::rotl(kc::xor3(A[6], C0, R2), 44);                         \
    uint64_t B2 = KC_ROT_B(kc::xor3(A[12], C1, R3), 43);                        \
    uint64_t B3 = kc::rotl(kc::xor3(A[18], C2, R4), 21);                        \
    uint64_t B4 = KC_ROT_B(kc::xor3(A[24], C3, R0), 14);                        \
    uint64_t B5 = kc::rotl(kc::xor3(A[3], C2, R4), 28);                         \
    uint64_t B6 = KC_ROT_B(kc::xor3(A[9], C3, R0), 20);                         \
    uint64_t B7 = kc::rotl(kc::xor3(A[10], C4, R1), 3);                         \
    uint64_t B8 = KC_ROT_B(kc::xor3(A[16], C0, R2), 45);                        \
    uint64_t B9 = kc::rotl(kc::xor3(A[22], C1, R3), 61);                        \
    uint64_t B10 = KC_ROT_B(kc::xor3(A[1], C0, R2), 1);                         \
    uint64_t B11 = kc::rotl(kc::xor3(A[7], C1, R3), 6);                         \
    uint64_t B12 = KC_ROT_B(kc::xor3(A[13], C2, R4), 25);                       \
    uint64_t B13 = kc::rotl(kc::xor3(A[19], C3, R0), 8);                        \
    uint64_t B14 = KC_ROT_B(kc::xor3(A[20], C4, R1), 18);                       \
    uint64_t B15 = kc::rotl(kc::xor3(A[4], C3, R0), 27);                        \
    uint64_t B16 = KC_ROT_B(kc::xor3(A[5], C4, R1), 36);                        \
    uint64_t B17 = kc::rotl(kc::xor3(A[11], C0, R2), 10);                       \
    uint64_t B18 = KC_ROT_B(kc::xor3(A[17], C1, R3), 15);                       \
    uint64_t B19 = kc::rotl(kc::xor3(A[23], C2, R4), 56);                       \
    uint64_t B20 = KC_ROT_B(kc::xor3(A[2], C1, R3), 62);                        \
    uint64_t B21 = kc::rotl(kc::xor3(A[8], C2, R4), 55);                        \
    uint64_t B22 = KC_ROT_B(kc::xor3(A[14], C3, R0), 39);                       \
    uint64_t B23 = kc::rotl(kc::xor3(A[15], C4, R1), 41);                       \
    uint64_t B24 = KC_ROT_B(kc::xor3(A[21], C0, R2), 2);                        \
    A[0] = kc::chi(B0, B1, B2) ^ (rc);                                          \
    A[1] = kc::chi(B1, B2, B3);                                                 \
    A[2] = kc::chi(B2, B3, B4);                                                 \
    A[3] = kc::chi(B3, B4, B0);                                                 \
    A[4] = kc::chi(B4, B0, B1);                                                 \
    A[5] = kc::chi(B5, B6, B7);                                                 \
    A[6] = kc::chi(B6, B7, B8);                                                 \
    A[7] = kc::chi(B7, B8, B9);                                                 \
    A[8] = kc::chi(B8, B9, B5);                                                 \
    A[9] = kc::chi(B9, B5, B6);                                                 \
    A[10] = kc::chi(B10, B11, B12);                                             \
    A[11] = kc::chi(B11, B12, B13);                                             \
    A[12] = kc::chi(B12, B13, B14);                                             \
    A[13] = kc::chi(B13, B14, B10);                                             \
    A[14] = kc::chi(B14, B10, B11);                                             \
    A[15] = kc::chi(B15, B16, B17);                                             \
    A[16] = kc::chi(B16, B17, B18);                                             \
    A[17] = kc::chi(B17, B18, B19);                                             \
    A[18] = kc::chi(B18, B19, B15);                                             \
    A[19] = kc::chi(B19, B15, B16);                                             \
    A[20] = kc::chi(B20, B21, B22);                                             \
    A[21] = kc::chi(B21, B22, B23);                                             \
    A[22] = kc::chi(B22, B23, B24);                                             \
    A[23] = kc::chi(B23, B24, B20);                                             \
    A[24] = kc::chi(B24, B20, B21);                                             \
  }

KC_HD void keccak_f(uint64_t A[25]) {
#if defined(__CUDA_ARCH__)
#pragma unroll 2
  for (int r = 0; r < 24; ++r) KC_ROUND(A, kRC_dev[r]);
#else
  for (int r = 0; r < 24; ++r) KC_ROUND(A, kRC_host[r]);
#endif
}

// Lane-granular sponge of the build's profile: absorb whole 64-bit lanes, squeeze
// kDigestLanes lanes.
// The state is only ever indexed by constants (a switch on the block
// position), so it stays in registers; when the caller's loop is unrolled the
// position is a compile-time constant and the switch disappears.
struct LaneSponge {
  uint64_t s[25];
  int pos;  // lanes absorbed into the current block (0 .. kRateLanes-1)
  KC_HD void init() {
#pragma unroll
    for (int i = 0; i < 25; ++i) s[i] = 0;
    pos = 0;
  }
  KC_HD void xor_at(int p, uint64_t w) {
    switch (p) {
      case 0: s[0] ^= w; break;
      case 1: s[1] ^= w; break;
      case 2: s[2] ^= w; break;
      case 3: s[3] ^= w; break;
      case 4: s[4] ^= w; break;
      case 5: s[5] ^= w; break;
      case 6: s[6] ^= w; break;
      case 7: s[7] ^= w; break;
      case 8: s[8] ^= w; break;
      case 9: s[9] ^= w; break;
      case 10: s[10] ^= w; break;
      case 11: s[11] ^= w; break;
      case 12: s[12] ^= w; break;
      case 13: s[13] ^= w; break;
      case 14: s[14] ^= w; break;
      case 15: s[15] ^= w; break;
      default: s[16] ^= w; break;
    }
  }
  KC_HD void lane(uint64_t w) {
    xor_at(pos, w);
    if (++pos == kRateLanes) {
      keccak_f(s);
      pos = 0;
    }
  }
  KC_HD void finish(uint64_t out[kDigestLanes]) {
    xor_at(pos, 0x06ull);
    s[kRateLanes - 1] ^= 0x8000000000000000ull;
    keccak_f(s);
#pragma unroll
    for (int i = 0; i < kDigestLanes; ++i) out[i] = s[i];
  }
};

// Byte-granular streaming SHA3 with an OUT-byte digest for host code
// (transcript, domain tags, record hashing).
template <int OUT>
struct Sha3T {
  static constexpr int RATE = 200 - 2 * OUT;
  uint64_t st[25];
  uint8_t buf[RATE];
  size_t fill;
  Sha3T() { reset(); }
  void reset() {
    memset(st, 0, sizeof st);
    fill = 0;
  }
  void block(const uint8_t* b) {
    for (int i = 0; i < RATE / 8; ++i) {
      uint64_t w;
      memcpy(&w, b + 8 * i, 8);
      st[i] ^= w;
    }
    keccak_f(st);
  }
  void update(const void* data, size_t len) {
    const uint8_t* p = (const uint8_t*)data;
    while (len) {
      size_t take = RATE - fill < len ? RATE - fill : len;
      memcpy(buf + fill, p, take);
      fill += take;
      p += take;
      len -= take;
      if (fill == (size_t)RATE) {
        block(buf);
        fill = 0;
      }
    }
  }
  void finalize(uint8_t out[OUT]) const {
    Sha3T c = *this;
    memset(c.buf + c.fill, 0, RATE - c.fill);
    c.buf[c.fill] ^= 0x06;
    c.buf[RATE - 1] ^= 0x80;
    c.block(c.buf);
    memcpy(out, c.st, OUT);
  }
};
using Sha3 = Sha3T<32>;             // SHA3-256: records, pi_hash recipes
using Sha3Sel = Sha3T<kHashBytes>;  // the profile: Merkle channel and transcript

}  // namespace kc

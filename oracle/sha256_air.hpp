// oracle/sha256_air.hpp — CPU restatement of the SHA-256 AIR (756 columns, 766 constraints).
//
// TEST INFRASTRUCTURE ONLY (part of the oracle; never linked into the product).
//
// Follows deep_ali/src/sha256_air.rs:
//   :140-248   column layout (blocks A..O), WIDTH = 756
//   :255-278   K and IV (FIPS 180-4 §4.2.2, §5.3.3)
//   :399-410   FIPS padding;  :429-472 build_sha256_trace_multi (128 rows per block,
//              height next_pow2, last useful row replicated)
//   :648-937   fill_block
//   :956-1294  eval_sha256_constraints: the constraint ORDER below is the reference's,
//              because the merge combines them with lambda_j = j + 1.
#pragma once
#include <cstdint>
#include <vector>

#include "gl.hpp"

namespace orc {
namespace sha {

enum : size_t {
  A_a = 0, A_b, A_c, A_d, A_e, A_f, A_g, A_h,
  BIT_A = 8, BIT_B = 40, BIT_C = 72, BIT_E = 104, BIT_F = 136, BIT_G = 168,
  S0_T = 200, S0_BIT = 232, S0_W = 264,
  S1_T = 265, S1_BIT = 297, S1_W = 329,
  CH_BIT = 330, CH_W = 362,
  MAJ_AB = 363, MAJ_AC = 395, MAJ_BC = 427, MAJ_U = 459, MAJ_BIT = 491, MAJ_W = 523,
  W_ = 524,
  T1_LO = 525, T1_C0 = 526, T1_C1 = 527, T1_C2 = 528, T1_CW = 529,
  T2_LO = 530, T2_C0 = 531, T2_C1 = 532, T2_CW = 533,
  H0 = 534,
  WW0 = 542,
  BIT_WW14 = 557, BIT_WW1 = 589,
  SS0_T = 621, SS0_BIT = 653, SS0_W = 685,
  SS1_T = 686, SS1_BIT = 718, SS1_W = 750,
  WS_C0 = 751, WS_C1 = 752, WS_CW = 753,
  NA_C = 754, NE_C = 755,
  WIDTH = 756, NUM_CONSTRAINTS = 766, ROWS_PER_BLOCK = 128
};

static const uint32_t K[64] = {
    0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
    0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
    0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
    0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
    0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
    0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
    0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
    0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};
static const uint32_t IV[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                               0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};

inline uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }
inline uint32_t bs0(uint32_t x) { return rotr(x, 2) ^ rotr(x, 13) ^ rotr(x, 22); }
inline uint32_t bs1(uint32_t x) { return rotr(x, 6) ^ rotr(x, 11) ^ rotr(x, 25); }
inline uint32_t ss0(uint32_t x) { return rotr(x, 7) ^ rotr(x, 18) ^ (x >> 3); }
inline uint32_t ss1(uint32_t x) { return rotr(x, 17) ^ rotr(x, 19) ^ (x >> 10); }
inline uint32_t ch(uint32_t x, uint32_t y, uint32_t z) { return (x & y) ^ (~x & z); }
inline uint32_t maj(uint32_t x, uint32_t y, uint32_t z) { return (x & y) ^ (x & z) ^ (y & z); }
inline uint32_t bitof(uint32_t x, int i) { return (x >> i) & 1; }

inline std::vector<std::vector<uint8_t>> pad_blocks(const uint8_t* msg, size_t len) {
  std::vector<uint8_t> buf(msg, msg + len);
  buf.push_back(0x80);
  while (buf.size() % 64 != 56) buf.push_back(0);
  uint64_t bits = (uint64_t)len * 8;
  for (int i = 7; i >= 0; --i) buf.push_back((uint8_t)(bits >> (8 * i)));
  std::vector<std::vector<uint8_t>> out;
  for (size_t o = 0; o < buf.size(); o += 64) out.emplace_back(buf.begin() + o, buf.begin() + o + 64);
  return out;
}

inline void schedule(const uint8_t* block, uint32_t w[64]) {
  for (int i = 0; i < 16; ++i)
    w[i] = ((uint32_t)block[4 * i] << 24) | ((uint32_t)block[4 * i + 1] << 16) | ((uint32_t)block[4 * i + 2] << 8) |
           block[4 * i + 3];
  for (int t = 16; t < 64; ++t) w[t] = ss1(w[t - 2]) + w[t - 7] + ss0(w[t - 15]) + w[t - 16];
}

// trace: WIDTH columns of `height` rows, column-major (tr[c*height + r])
inline void fill_block(Fp* tr, size_t height, size_t base, const uint8_t* block, const uint32_t iv[8]) {
  auto at = [&](size_t c, size_t r) -> Fp& { return tr[c * height + r]; };
  auto fu = [](uint64_t x) { return Fp(x); };
  uint32_t w[64];
  schedule(block, w);
  uint32_t st[65][8];
  for (int k = 0; k < 8; ++k) st[0][k] = iv[k];
  for (int t = 0; t < 64; ++t) {
    const uint32_t* s = st[t];
    uint32_t t1 = s[7] + bs1(s[4]) + ch(s[4], s[5], s[6]) + K[t] + w[t];
    uint32_t t2 = bs0(s[0]) + maj(s[0], s[1], s[2]);
    uint32_t n[8] = {t1 + t2, s[0], s[1], s[2], s[3] + t1, s[4], s[5], s[6]};
    for (int k = 0; k < 8; ++k) st[t + 1][k] = n[k];
  }
  uint32_t digest[8];
  for (int k = 0; k < 8; ++k) digest[k] = iv[k] + st[64][k];
  auto wat = [&](long idx) -> uint32_t { return (idx >= 0 && idx < 64) ? w[idx] : 0; };
  for (size_t br = 0; br < ROWS_PER_BLOCK; ++br) {
    size_t row = base + br;
    const uint32_t* s = st[br <= 64 ? br : 64];
    uint32_t a = s[0], b = s[1], c = s[2], d = s[3], e = s[4], f = s[5], g = s[6], h = s[7];
    for (int k = 0; k < 8; ++k) at(A_a + k, row) = fu(s[k]);
    for (int i = 0; i < 32; ++i) {
      at(BIT_A + i, row) = fu(bitof(a, i));
      at(BIT_B + i, row) = fu(bitof(b, i));
      at(BIT_C + i, row) = fu(bitof(c, i));
      at(BIT_E + i, row) = fu(bitof(e, i));
      at(BIT_F + i, row) = fu(bitof(f, i));
      at(BIT_G + i, row) = fu(bitof(g, i));
    }
    for (int i = 0; i < 32; ++i) {
      uint32_t p = bitof(a, (i + 2) % 32), q = bitof(a, (i + 13) % 32), r = bitof(a, (i + 22) % 32);
      at(S0_T + i, row) = fu(p ^ q);
      at(S0_BIT + i, row) = fu(p ^ q ^ r);
    }
    at(S0_W, row) = fu(bs0(a));
    for (int i = 0; i < 32; ++i) {
      uint32_t p = bitof(e, (i + 6) % 32), q = bitof(e, (i + 11) % 32), r = bitof(e, (i + 25) % 32);
      at(S1_T + i, row) = fu(p ^ q);
      at(S1_BIT + i, row) = fu(p ^ q ^ r);
    }
    at(S1_W, row) = fu(bs1(e));
    uint32_t chw = ch(e, f, g);
    for (int i = 0; i < 32; ++i) at(CH_BIT + i, row) = fu(bitof(chw, i));
    at(CH_W, row) = fu(chw);
    for (int i = 0; i < 32; ++i) {
      uint32_t ai = bitof(a, i), bi = bitof(b, i), ci = bitof(c, i);
      uint32_t ab = ai & bi, ac = ai & ci, bc = bi & ci, u = ab ^ ac;
      at(MAJ_AB + i, row) = fu(ab);
      at(MAJ_AC + i, row) = fu(ac);
      at(MAJ_BC + i, row) = fu(bc);
      at(MAJ_U + i, row) = fu(u);
      at(MAJ_BIT + i, row) = fu(u ^ bc);
    }
    at(MAJ_W, row) = fu(maj(a, b, c));
    uint32_t wt = br < 64 ? w[br] : 0, kt = br < 64 ? K[br] : 0;
    at(W_, row) = fu(wt);
    uint64_t t1 = (uint64_t)h + bs1(e) + chw + kt + wt;
    uint32_t t1c = (uint32_t)(t1 >> 32);
    at(T1_LO, row) = fu(t1 & 0xFFFFFFFFu);
    at(T1_C0, row) = fu(t1c & 1);
    at(T1_C1, row) = fu((t1c >> 1) & 1);
    at(T1_C2, row) = fu((t1c >> 2) & 1);
    at(T1_CW, row) = fu(t1c);
    uint64_t t2 = (uint64_t)bs0(a) + maj(a, b, c);
    uint32_t t2c = (uint32_t)(t2 >> 32);
    at(T2_LO, row) = fu(t2 & 0xFFFFFFFFu);
    at(T2_C0, row) = fu(t2c & 1);
    at(T2_C1, row) = fu((t2c >> 1) & 1);
    at(T2_CW, row) = fu(t2c);
    for (int k = 0; k < 8; ++k) at(H0 + k, row) = fu(br <= 64 ? iv[k] : digest[k]);
    for (int k = 0; k < 15; ++k) at(WW0 + k, row) = fu(wat((long)br - 15 + k));
    uint32_t ww14 = wat((long)br - 1), ww1 = wat((long)br - 14);
    for (int i = 0; i < 32; ++i) {
      at(BIT_WW14 + i, row) = fu(bitof(ww14, i));
      at(BIT_WW1 + i, row) = fu(bitof(ww1, i));
    }
    for (int i = 0; i < 32; ++i) {
      uint32_t p = bitof(ww1, (i + 7) % 32), q = bitof(ww1, (i + 18) % 32), r = i + 3 < 32 ? bitof(ww1, i + 3) : 0;
      at(SS0_T + i, row) = fu(p ^ q);
      at(SS0_BIT + i, row) = fu(p ^ q ^ r);
    }
    at(SS0_W, row) = fu(ss0(ww1));
    for (int i = 0; i < 32; ++i) {
      uint32_t p = bitof(ww14, (i + 17) % 32), q = bitof(ww14, (i + 19) % 32),
               r = i + 10 < 32 ? bitof(ww14, i + 10) : 0;
      at(SS1_T + i, row) = fu(p ^ q);
      at(SS1_BIT + i, row) = fu(p ^ q ^ r);
    }
    at(SS1_W, row) = fu(ss1(ww14));
    uint64_t sum = (uint64_t)wat((long)br - 15) + ss0(ww1) + wat((long)br - 6) + ss1(ww14);
    uint32_t sc = (uint32_t)(sum >> 32);
    at(WS_C0, row) = fu(sc & 1);
    at(WS_C1, row) = fu((sc >> 1) & 1);
    at(WS_CW, row) = fu(sc);
    if (br < 64) {
      uint64_t t1lo = t1 & 0xFFFFFFFFu, t2lo = t2 & 0xFFFFFFFFu;
      at(NA_C, row) = fu((t1lo + t2lo) >> 32);
      at(NE_C, row) = fu(((uint64_t)d + t1lo) >> 32);
    }
  }
}

// build_sha256_trace_multi: returns height, fills `tr` (resized to WIDTH*height) and n_blocks.
inline size_t build_trace_multi(const uint8_t* msg, size_t len, std::vector<Fp>* tr, size_t* n_blocks) {
  auto blocks = pad_blocks(msg, len);
  *n_blocks = blocks.size();
  size_t useful = ROWS_PER_BLOCK * blocks.size();
  size_t height = ROWS_PER_BLOCK;
  while (height < useful) height <<= 1;
  tr->assign(WIDTH * height, Fp());
  uint32_t iv[8];
  for (int k = 0; k < 8; ++k) iv[k] = IV[k];
  for (size_t b = 0; b < blocks.size(); ++b) {
    fill_block(tr->data(), height, b * ROWS_PER_BLOCK, blocks[b].data(), iv);
    // next IV = iv + post-compression state
    uint32_t w[64];
    schedule(blocks[b].data(), w);
    uint32_t s[8];
    for (int k = 0; k < 8; ++k) s[k] = iv[k];
    for (int t = 0; t < 64; ++t) {
      uint32_t t1 = s[7] + bs1(s[4]) + ch(s[4], s[5], s[6]) + K[t] + w[t];
      uint32_t t2 = bs0(s[0]) + maj(s[0], s[1], s[2]);
      uint32_t n[8] = {t1 + t2, s[0], s[1], s[2], s[3] + t1, s[4], s[5], s[6]};
      for (int k = 0; k < 8; ++k) s[k] = n[k];
    }
    for (int k = 0; k < 8; ++k) iv[k] += s[k];
  }
  for (size_t r = useful; r < height; ++r)
    for (size_t c = 0; c < WIDTH; ++c) (*tr)[c * height + r] = (*tr)[c * height + useful - 1];
  return height;
}

// eval_sha256_constraints (sha256_air.rs:956-1294); out has NUM_CONSTRAINTS entries.
inline void eval(const Fp* cur, const Fp* nxt, size_t row, size_t n_blocks, Fp* out) {
  size_t o = 0;
  auto push = [&](Fp v) { out[o++] = v; };
  const Fp one = Fp::raw(1), two = Fp::raw(2), four = Fp::raw(4), p32 = Fp::raw(1ull << 32);
  auto xr = [&](Fp x, Fp y) { return x + y - two * x * y; };
  const size_t blk = row / ROWS_PER_BLOCK, br = row % ROWS_PER_BLOCK;
  const bool past = blk >= n_blocks;
  const bool comp = !past && br < 64, fin = !past && br == 64, sched = !past && br >= 15 && br <= 62;
  const size_t bool_offs[8] = {BIT_A, BIT_B, BIT_C, BIT_E, BIT_F, BIT_G, BIT_WW14, BIT_WW1};
  for (size_t off : bool_offs)
    for (int i = 0; i < 32; ++i) push(cur[off + i] * (one - cur[off + i]));
  auto pack = [&](size_t off) {
    Fp s;
    for (int i = 0; i < 32; ++i) s = s + Fp::raw(1ull << i) * cur[off + i];
    return s;
  };
  push(cur[A_a] - pack(BIT_A));
  push(cur[A_b] - pack(BIT_B));
  push(cur[A_c] - pack(BIT_C));
  push(cur[A_e] - pack(BIT_E));
  push(cur[A_f] - pack(BIT_F));
  push(cur[A_g] - pack(BIT_G));
  push(cur[WW0 + 14] - pack(BIT_WW14));
  push(cur[WW0 + 1] - pack(BIT_WW1));
  auto sigma_block = [&](size_t bits, size_t toff, size_t boff, size_t woff, int r1, int r2, int r3, bool shift) {
    for (int i = 0; i < 32; ++i) push(cur[toff + i] - xr(cur[bits + (i + r1) % 32], cur[bits + (i + r2) % 32]));
    for (int i = 0; i < 32; ++i) {
      Fp r = shift ? (i + r3 < 32 ? cur[bits + i + r3] : Fp()) : cur[bits + (i + r3) % 32];
      push(cur[boff + i] - xr(cur[toff + i], r));
    }
    push(cur[woff] - pack(boff));
  };
  sigma_block(BIT_A, S0_T, S0_BIT, S0_W, 2, 13, 22, false);
  sigma_block(BIT_E, S1_T, S1_BIT, S1_W, 6, 11, 25, false);
  sigma_block(BIT_WW1, SS0_T, SS0_BIT, SS0_W, 7, 18, 3, true);
  sigma_block(BIT_WW14, SS1_T, SS1_BIT, SS1_W, 17, 19, 10, true);
  for (int i = 0; i < 32; ++i) {
    Fp e = cur[BIT_E + i], f = cur[BIT_F + i], g = cur[BIT_G + i];
    push(cur[CH_BIT + i] - (e * f + g - e * g));
  }
  push(cur[CH_W] - pack(CH_BIT));
  for (int i = 0; i < 32; ++i) {
    Fp a = cur[BIT_A + i], b = cur[BIT_B + i], c = cur[BIT_C + i];
    push(cur[MAJ_AB + i] - a * b);
    push(cur[MAJ_AC + i] - a * c);
    push(cur[MAJ_BC + i] - b * c);
  }
  for (int i = 0; i < 32; ++i) push(cur[MAJ_U + i] - xr(cur[MAJ_AB + i], cur[MAJ_AC + i]));
  for (int i = 0; i < 32; ++i) push(cur[MAJ_BIT + i] - xr(cur[MAJ_U + i], cur[MAJ_BC + i]));
  push(cur[MAJ_W] - pack(MAJ_BIT));
  Fp krow = comp ? Fp(K[br]) : Fp();
  push(cur[T1_LO] + p32 * cur[T1_CW] - (cur[A_h] + cur[S1_W] + cur[CH_W] + krow + cur[W_]));
  for (size_t off : {(size_t)T1_C0, (size_t)T1_C1, (size_t)T1_C2}) push(cur[off] * (one - cur[off]));
  push(cur[T1_CW] - cur[T1_C0] - two * cur[T1_C1] - four * cur[T1_C2]);
  push(cur[T2_LO] + p32 * cur[T2_CW] - (cur[S0_W] + cur[MAJ_W]));
  for (size_t off : {(size_t)T2_C0, (size_t)T2_C1}) push(cur[off] * (one - cur[off]));
  push(cur[T2_CW] - cur[T2_C0] - two * cur[T2_C1]);
  push(comp ? nxt[A_b] - cur[A_a] : Fp());
  push(comp ? nxt[A_c] - cur[A_b] : Fp());
  push(comp ? nxt[A_d] - cur[A_c] : Fp());
  push(comp ? nxt[A_f] - cur[A_e] : Fp());
  push(comp ? nxt[A_g] - cur[A_f] : Fp());
  push(comp ? nxt[A_h] - cur[A_g] : Fp());
  if (comp) {
    push(nxt[A_a] + p32 * cur[NA_C] - cur[T1_LO] - cur[T2_LO]);
    push(cur[NA_C] * (one - cur[NA_C]));
    push(nxt[A_e] + p32 * cur[NE_C] - cur[A_d] - cur[T1_LO]);
    push(cur[NE_C] * (one - cur[NE_C]));
    push(Fp());
    push(Fp());
  } else {
    for (int i = 0; i < 6; ++i) push(Fp());
  }
  for (int k = 0; k < 8; ++k) {
    if (fin) {
      Fp delta = cur[H0 + k] + cur[A_a + k] - nxt[H0 + k];
      push(delta * (delta - p32));
    } else {
      push(nxt[H0 + k] - cur[H0 + k]);
    }
  }
  for (int k = 0; k < 14; ++k) push(nxt[WW0 + k] - cur[WW0 + k + 1]);
  push(nxt[WW0 + 14] - cur[W_]);
  if (sched) {
    Fp sum = cur[WW0] + cur[SS0_W] + cur[WW0 + 9] + cur[SS1_W];
    push(nxt[W_] + p32 * cur[WS_CW] - sum);
    push(cur[WS_C0] * (one - cur[WS_C0]));
    push(cur[WS_C1] * (one - cur[WS_C1]));
    push(cur[WS_CW] - cur[WS_C0] - two * cur[WS_C1]);
  } else {
    for (int i = 0; i < 4; ++i) push(Fp());
  }
}

}  // namespace sha
}  // namespace orc

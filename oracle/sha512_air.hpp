// oracle/sha512_air.hpp — CPU restatement of the SHA-512 AIR (1510 columns, 1526 constraints).
//
// TEST INFRASTRUCTURE ONLY (part of the oracle; never linked into the product).
//
// Follows deep_ali/src/sha512_air.rs:
//   :147-162   IV, 80 rounds, 128-byte blocks, 128 rows per block
//   :218-236   FIPS 180-4 §5.1.2 padding (0x80, zeros to 112 mod 128, 128-bit length)
//   :313-471   column layout, WIDTH = 1510: every 64-bit word is two 32-bit limbs
//   :551-578   build_sha512_trace_multi (height next_pow2, last useful row replicated)
//   :585-896   fill_block: rows 0..79 rounds, row 80 post-compression state, rows >= 81
//              idle; H-state = IV on rows <= 80, block digest on rows >= 81
//   :909-1270  eval_sha512_constraints: the constraint ORDER below is the reference's,
//              because the merge combines them with lambda_j.
// K and IV are the FIPS 180-4 §4.2.3 / §5.3.5 constants (first 64 bits of the
// fractional parts of the cube / square roots of the first primes).
#pragma once
#include <cstdint>
#include <vector>

#include "gl.hpp"

namespace orc {
namespace sha512 {

enum : size_t {
  A_LO = 0,  // word k of {a..h}: lo limb at 2k, hi limb at 2k + 1
  BIT_A = 16, BIT_B = 80, BIT_C = 144, BIT_E = 208, BIT_F = 272, BIT_G = 336,
  S0_T = 400, S0_BIT = 464, S0_LO = 528, S0_HI = 529,
  S1_T = 530, S1_BIT = 594, S1_LO = 658, S1_HI = 659,
  CH_BIT = 660, CH_LO = 724, CH_HI = 725,
  MAJ_AB = 726, MAJ_AC = 790, MAJ_BC = 854, MAJ_U = 918, MAJ_BIT = 982, MAJ_LO = 1046, MAJ_HI = 1047,
  W_LO = 1048, W_HI = 1049,
  T1_LO_LO = 1050, T1_LO_C0, T1_LO_C1, T1_LO_C2, T1_LO_CW,
  T1_HI_LO = 1055, T1_HI_C0, T1_HI_C1, T1_HI_C2, T1_HI_CW,
  T2_LO_LO = 1060, T2_LO_C0, T2_LO_CW, T2_HI_LO, T2_HI_C0, T2_HI_CW,
  H0_LO = 1066,   // H_k: lo at 1066 + 2k, hi at 1067 + 2k
  WW0_LO = 1082,  // W_win[k]: lo at 1082 + 2k, hi at 1083 + 2k (k < 15)
  BIT_WW14 = 1112, BIT_WW1 = 1176,
  SS0_T = 1240, SS0_BIT = 1304, SS0_LO = 1368, SS0_HI = 1369,
  SS1_T = 1370, SS1_BIT = 1434, SS1_LO = 1498, SS1_HI = 1499,
  WS_LO_C0 = 1500, WS_LO_C1, WS_LO_CW, WS_HI_C0, WS_HI_C1, WS_HI_CW,
  NA_LO_C = 1506, NA_HI_C, NE_LO_C, NE_HI_C,
  WIDTH = 1510, NUM_CONSTRAINTS = 1526, ROWS_PER_BLOCK = 128, ROUNDS = 80
};

static const uint64_t K[80] = {
0x428a2f98d728ae22ull, 0x7137449123ef65cdull, 0xb5c0fbcfec4d3b2full, 0xe9b5dba58189dbbcull,
0x3956c25bf348b538ull, 0x59f111f1b605d019ull, 0x923f82a4af194f9bull, 0xab1c5ed5da6d8118ull,
0xd807aa98a3030242ull, 0x12835b0145706fbeull, 0x243185be4ee4b28cull, 0x550c7dc3d5ffb4e2ull,
0x72be5d74f27b896full, 0x80deb1fe3b1696b1ull, 0x9bdc06a725c71235ull, 0xc19bf174cf692694ull,
0xe49b69c19ef14ad2ull, 0xefbe4786384f25e3ull, 0x0fc19dc68b8cd5b5ull, 0x240ca1cc77ac9c65ull,
0x2de92c6f592b0275ull, 0x4a7484aa6ea6e483ull, 0x5cb0a9dcbd41fbd4ull, 0x76f988da831153b5ull,
0x983e5152ee66dfabull, 0xa831c66d2db43210ull, 0xb00327c898fb213full, 0xbf597fc7beef0ee4ull,
0xc6e00bf33da88fc2ull, 0xd5a79147930aa725ull, 0x06ca6351e003826full, 0x142929670a0e6e70ull,
0x27b70a8546d22ffcull, 0x2e1b21385c26c926ull, 0x4d2c6dfc5ac42aedull, 0x53380d139d95b3dfull,
0x650a73548baf63deull, 0x766a0abb3c77b2a8ull, 0x81c2c92e47edaee6ull, 0x92722c851482353bull,
0xa2bfe8a14cf10364ull, 0xa81a664bbc423001ull, 0xc24b8b70d0f89791ull, 0xc76c51a30654be30ull,
0xd192e819d6ef5218ull, 0xd69906245565a910ull, 0xf40e35855771202aull, 0x106aa07032bbd1b8ull,
0x19a4c116b8d2d0c8ull, 0x1e376c085141ab53ull, 0x2748774cdf8eeb99ull, 0x34b0bcb5e19b48a8ull,
0x391c0cb3c5c95a63ull, 0x4ed8aa4ae3418acbull, 0x5b9cca4f7763e373ull, 0x682e6ff3d6b2b8a3ull,
0x748f82ee5defb2fcull, 0x78a5636f43172f60ull, 0x84c87814a1f0ab72ull, 0x8cc702081a6439ecull,
0x90befffa23631e28ull, 0xa4506cebde82bde9ull, 0xbef9a3f7b2c67915ull, 0xc67178f2e372532bull,
0xca273eceea26619cull, 0xd186b8c721c0c207ull, 0xeada7dd6cde0eb1eull, 0xf57d4f7fee6ed178ull,
0x06f067aa72176fbaull, 0x0a637dc5a2c898a6ull, 0x113f9804bef90daeull, 0x1b710b35131c471bull,
0x28db77f523047d84ull, 0x32caab7b40c72493ull, 0x3c9ebe0a15c9bebcull, 0x431d67c49c100d4cull,
0x4cc5d4becb3e42b6ull, 0x597f299cfc657e2aull, 0x5fcb6fab3ad6faecull, 0x6c44198c4a475817ull};
static const uint64_t IV[8] = {
0x6a09e667f3bcc908ull, 0xbb67ae8584caa73bull, 0x3c6ef372fe94f82bull, 0xa54ff53a5f1d36f1ull,
0x510e527fade682d1ull, 0x9b05688c2b3e6c1full, 0x1f83d9abfb41bd6bull, 0x5be0cd19137e2179ull};

inline uint64_t rotr(uint64_t x, int n) { return (x >> n) | (x << (64 - n)); }
inline uint64_t bs0(uint64_t x) { return rotr(x, 28) ^ rotr(x, 34) ^ rotr(x, 39); }
inline uint64_t bs1(uint64_t x) { return rotr(x, 14) ^ rotr(x, 18) ^ rotr(x, 41); }
inline uint64_t ss0(uint64_t x) { return rotr(x, 1) ^ rotr(x, 8) ^ (x >> 7); }
inline uint64_t ss1(uint64_t x) { return rotr(x, 19) ^ rotr(x, 61) ^ (x >> 6); }
inline uint64_t ch(uint64_t x, uint64_t y, uint64_t z) { return (x & y) ^ (~x & z); }
inline uint64_t maj(uint64_t x, uint64_t y, uint64_t z) { return (x & y) ^ (x & z) ^ (y & z); }
inline uint64_t bitof(uint64_t x, int i) { return (x >> i) & 1; }
inline uint64_t lo32(uint64_t x) { return x & 0xFFFFFFFFull; }
inline uint64_t hi32(uint64_t x) { return x >> 32; }

inline std::vector<std::vector<uint8_t>> pad_blocks(const uint8_t* msg, size_t len) {
  std::vector<uint8_t> buf(msg, msg + len);
  buf.push_back(0x80);
  while (buf.size() % 128 != 112) buf.push_back(0);
  for (int i = 0; i < 8; ++i) buf.push_back(0);  // upper 64 bits of the 128-bit length
  const uint64_t bits = (uint64_t)len * 8;
  for (int i = 7; i >= 0; --i) buf.push_back((uint8_t)(bits >> (8 * i)));
  std::vector<std::vector<uint8_t>> out;
  for (size_t o = 0; o < buf.size(); o += 128) out.emplace_back(buf.begin() + o, buf.begin() + o + 128);
  return out;
}

inline void schedule(const uint8_t* block, uint64_t w[80]) {
  for (int i = 0; i < 16; ++i) {
    uint64_t v = 0;
    for (int b = 0; b < 8; ++b) v = (v << 8) | block[8 * i + b];
    w[i] = v;
  }
  for (int t = 16; t < 80; ++t) w[t] = ss1(w[t - 2]) + w[t - 7] + ss0(w[t - 15]) + w[t - 16];
}

// st[t] = (a..h) at the start of round t; st[80] = post-compression state
inline void rounds(const uint64_t w[80], const uint64_t iv[8], uint64_t st[81][8]) {
  for (int k = 0; k < 8; ++k) st[0][k] = iv[k];
  for (int t = 0; t < 80; ++t) {
    const uint64_t* s = st[t];
    const uint64_t t1 = s[7] + bs1(s[4]) + ch(s[4], s[5], s[6]) + K[t] + w[t];
    const uint64_t t2 = bs0(s[0]) + maj(s[0], s[1], s[2]);
    const uint64_t n[8] = {t1 + t2, s[0], s[1], s[2], s[3] + t1, s[4], s[5], s[6]};
    for (int k = 0; k < 8; ++k) st[t + 1][k] = n[k];
  }
}

// trace: WIDTH columns of `height` rows, column-major (tr[c*height + r])
inline void fill_block(Fp* tr, size_t height, size_t base, const uint8_t* block, const uint64_t iv[8]) {
  auto put = [&](size_t c, size_t r, uint64_t v) { tr[c * height + r] = Fp(v); };
  uint64_t w[80], st[81][8], digest[8];
  schedule(block, w);
  rounds(w, iv, st);
  for (int k = 0; k < 8; ++k) digest[k] = iv[k] + st[80][k];
  auto wat = [&](long idx) -> uint64_t { return (idx >= 0 && idx < 80) ? w[idx] : 0; };
  for (size_t br = 0; br < ROWS_PER_BLOCK; ++br) {
    const size_t row = base + br;
    const uint64_t* s = st[br <= 80 ? br : 80];
    const uint64_t a = s[0], b = s[1], c = s[2], d = s[3], e = s[4], f = s[5], g = s[6], h = s[7];
    for (int k = 0; k < 8; ++k) {
      put(A_LO + 2 * k, row, lo32(s[k]));
      put(A_LO + 2 * k + 1, row, hi32(s[k]));
    }
    for (int i = 0; i < 64; ++i) {
      put(BIT_A + i, row, bitof(a, i));
      put(BIT_B + i, row, bitof(b, i));
      put(BIT_C + i, row, bitof(c, i));
      put(BIT_E + i, row, bitof(e, i));
      put(BIT_F + i, row, bitof(f, i));
      put(BIT_G + i, row, bitof(g, i));
    }
    for (int i = 0; i < 64; ++i) {
      const uint64_t p = bitof(a, (i + 28) % 64), q = bitof(a, (i + 34) % 64), r = bitof(a, (i + 39) % 64);
      put(S0_T + i, row, p ^ q);
      put(S0_BIT + i, row, p ^ q ^ r);
    }
    put(S0_LO, row, lo32(bs0(a)));
    put(S0_HI, row, hi32(bs0(a)));
    for (int i = 0; i < 64; ++i) {
      const uint64_t p = bitof(e, (i + 14) % 64), q = bitof(e, (i + 18) % 64), r = bitof(e, (i + 41) % 64);
      put(S1_T + i, row, p ^ q);
      put(S1_BIT + i, row, p ^ q ^ r);
    }
    put(S1_LO, row, lo32(bs1(e)));
    put(S1_HI, row, hi32(bs1(e)));
    const uint64_t chw = ch(e, f, g);
    for (int i = 0; i < 64; ++i) put(CH_BIT + i, row, bitof(chw, i));
    put(CH_LO, row, lo32(chw));
    put(CH_HI, row, hi32(chw));
    for (int i = 0; i < 64; ++i) {
      const uint64_t ai = bitof(a, i), bi = bitof(b, i), ci = bitof(c, i);
      const uint64_t ab = ai & bi, ac = ai & ci, bc = bi & ci, u = ab ^ ac;
      put(MAJ_AB + i, row, ab);
      put(MAJ_AC + i, row, ac);
      put(MAJ_BC + i, row, bc);
      put(MAJ_U + i, row, u);
      put(MAJ_BIT + i, row, u ^ bc);
    }
    const uint64_t mjw = maj(a, b, c);
    put(MAJ_LO, row, lo32(mjw));
    put(MAJ_HI, row, hi32(mjw));
    const uint64_t wt = br < 80 ? w[br] : 0, kt = br < 80 ? K[br] : 0;
    put(W_LO, row, lo32(wt));
    put(W_HI, row, hi32(wt));
    // T1, T2 per-limb carry decompositions
    const uint64_t t1l = lo32(h) + lo32(bs1(e)) + lo32(chw) + lo32(kt) + lo32(wt);
    const uint64_t t1lc = t1l >> 32;
    const uint64_t t1h = hi32(h) + hi32(bs1(e)) + hi32(chw) + hi32(kt) + hi32(wt) + t1lc;
    const uint64_t t1hc = t1h >> 32;
    put(T1_LO_LO, row, lo32(t1l));
    put(T1_LO_C0, row, t1lc & 1);
    put(T1_LO_C1, row, (t1lc >> 1) & 1);
    put(T1_LO_C2, row, (t1lc >> 2) & 1);
    put(T1_LO_CW, row, t1lc);
    put(T1_HI_LO, row, lo32(t1h));
    put(T1_HI_C0, row, t1hc & 1);
    put(T1_HI_C1, row, (t1hc >> 1) & 1);
    put(T1_HI_C2, row, (t1hc >> 2) & 1);
    put(T1_HI_CW, row, t1hc);
    const uint64_t t2l = lo32(bs0(a)) + lo32(mjw), t2lc = t2l >> 32;
    const uint64_t t2h = hi32(bs0(a)) + hi32(mjw) + t2lc, t2hc = t2h >> 32;
    put(T2_LO_LO, row, lo32(t2l));
    put(T2_LO_C0, row, t2lc & 1);
    put(T2_LO_CW, row, t2lc);
    put(T2_HI_LO, row, lo32(t2h));
    put(T2_HI_C0, row, t2hc & 1);
    put(T2_HI_CW, row, t2hc);
    for (int k = 0; k < 8; ++k) {
      const uint64_t hv = br <= 80 ? iv[k] : digest[k];
      put(H0_LO + 2 * k, row, lo32(hv));
      put(H0_LO + 2 * k + 1, row, hi32(hv));
    }
    for (int k = 0; k < 15; ++k) {
      const uint64_t v = wat((long)br - 15 + k);
      put(WW0_LO + 2 * k, row, lo32(v));
      put(WW0_LO + 2 * k + 1, row, hi32(v));
    }
    const uint64_t ww14 = wat((long)br - 1), ww1 = wat((long)br - 14);
    for (int i = 0; i < 64; ++i) put(BIT_WW14 + i, row, bitof(ww14, i));
    for (int i = 0; i < 64; ++i) put(BIT_WW1 + i, row, bitof(ww1, i));
    for (int i = 0; i < 64; ++i) {
      const uint64_t p = bitof(ww1, (i + 1) % 64), q = bitof(ww1, (i + 8) % 64), r = i + 7 < 64 ? bitof(ww1, i + 7) : 0;
      put(SS0_T + i, row, p ^ q);
      put(SS0_BIT + i, row, p ^ q ^ r);
    }
    put(SS0_LO, row, lo32(ss0(ww1)));
    put(SS0_HI, row, hi32(ss0(ww1)));
    for (int i = 0; i < 64; ++i) {
      const uint64_t p = bitof(ww14, (i + 19) % 64), q = bitof(ww14, (i + 61) % 64),
                     r = i + 6 < 64 ? bitof(ww14, i + 6) : 0;
      put(SS1_T + i, row, p ^ q);
      put(SS1_BIT + i, row, p ^ q ^ r);
    }
    put(SS1_LO, row, lo32(ss1(ww14)));
    put(SS1_HI, row, hi32(ss1(ww14)));
    const uint64_t w0 = wat((long)br - 15), w9 = wat((long)br - 6);
    const uint64_t wsl = lo32(w0) + lo32(ss0(ww1)) + lo32(w9) + lo32(ss1(ww14)), wslc = wsl >> 32;
    const uint64_t wsh = hi32(w0) + hi32(ss0(ww1)) + hi32(w9) + hi32(ss1(ww14)) + wslc, wshc = wsh >> 32;
    put(WS_LO_C0, row, wslc & 1);
    put(WS_LO_C1, row, (wslc >> 1) & 1);
    put(WS_LO_CW, row, wslc);
    put(WS_HI_C0, row, wshc & 1);
    put(WS_HI_C1, row, (wshc >> 1) & 1);
    put(WS_HI_CW, row, wshc);
    if (br < 80) {
      const uint64_t nal = lo32(t1l) + lo32(t2l), nalc = nal >> 32;
      const uint64_t nah = lo32(t1h) + lo32(t2h) + nalc;
      const uint64_t nel = lo32(d) + lo32(t1l), nelc = nel >> 32;
      const uint64_t neh = hi32(d) + lo32(t1h) + nelc;
      put(NA_LO_C, row, nalc);
      put(NA_HI_C, row, nah >> 32);
      put(NE_LO_C, row, nelc);
      put(NE_HI_C, row, neh >> 32);
    }
  }
}

// build_sha512_trace_multi: returns height, fills `tr` (WIDTH*height) and n_blocks.
inline size_t build_trace_multi(const uint8_t* msg, size_t len, std::vector<Fp>* tr, size_t* n_blocks) {
  auto blocks = pad_blocks(msg, len);
  *n_blocks = blocks.size();
  const size_t useful = ROWS_PER_BLOCK * blocks.size();
  size_t height = ROWS_PER_BLOCK;
  while (height < useful) height <<= 1;
  tr->assign(WIDTH * height, Fp());
  uint64_t iv[8];
  for (int k = 0; k < 8; ++k) iv[k] = IV[k];
  for (size_t b = 0; b < blocks.size(); ++b) {
    fill_block(tr->data(), height, b * ROWS_PER_BLOCK, blocks[b].data(), iv);
    uint64_t w[80], st[81][8];
    schedule(blocks[b].data(), w);
    rounds(w, iv, st);
    for (int k = 0; k < 8; ++k) iv[k] += st[80][k];
  }
  for (size_t r = useful; r < height; ++r)
    for (size_t c = 0; c < WIDTH; ++c) (*tr)[c * height + r] = (*tr)[c * height + useful - 1];
  return height;
}

// eval_sha512_constraints (sha512_air.rs:909-1270); out has NUM_CONSTRAINTS entries.
inline void eval(const Fp* cur, const Fp* nxt, size_t row, size_t n_blocks, Fp* out) {
  size_t o = 0;
  auto push = [&](Fp v) { out[o++] = v; };
  const Fp one = Fp::raw(1), two = Fp::raw(2), four = Fp::raw(4), p32 = Fp::raw(1ull << 32);
  auto xr = [&](Fp x, Fp y) { return x + y - two * x * y; };
  const size_t blk = row / ROWS_PER_BLOCK, br = row % ROWS_PER_BLOCK;
  const bool past = blk >= n_blocks;
  const bool comp = !past && br < ROUNDS, fin = !past && br == ROUNDS, sched = !past && br >= 15 && br <= 78;
  const size_t bool_offs[8] = {BIT_A, BIT_B, BIT_C, BIT_E, BIT_F, BIT_G, BIT_WW14, BIT_WW1};
  for (size_t off : bool_offs)
    for (int i = 0; i < 64; ++i) push(cur[off + i] * (one - cur[off + i]));
  auto pack = [&](size_t off) {  // sum_{i<32} 2^i cur[off + i]
    Fp s;
    for (int i = 0; i < 32; ++i) s = s + Fp::raw(1ull << i) * cur[off + i];
    return s;
  };
  const size_t words[6][2] = {{0, BIT_A}, {1, BIT_B}, {2, BIT_C}, {4, BIT_E}, {5, BIT_F}, {6, BIT_G}};
  for (auto& wb : words) {
    push(cur[A_LO + 2 * wb[0]] - pack(wb[1]));
    push(cur[A_LO + 2 * wb[0] + 1] - pack(wb[1] + 32));
  }
  push(cur[WW0_LO + 28] - pack(BIT_WW14));
  push(cur[WW0_LO + 29] - pack(BIT_WW14 + 32));
  push(cur[WW0_LO + 2] - pack(BIT_WW1));
  push(cur[WW0_LO + 3] - pack(BIT_WW1 + 32));
  auto sigma_block = [&](size_t bits, size_t toff, size_t boff, size_t lo, int r1, int r2, int r3, bool shift) {
    for (int i = 0; i < 64; ++i) push(cur[toff + i] - xr(cur[bits + (i + r1) % 64], cur[bits + (i + r2) % 64]));
    for (int i = 0; i < 64; ++i) {
      Fp r = shift ? (i + r3 < 64 ? cur[bits + i + r3] : Fp()) : cur[bits + (i + r3) % 64];
      push(cur[boff + i] - xr(cur[toff + i], r));
    }
    push(cur[lo] - pack(boff));
    push(cur[lo + 1] - pack(boff + 32));
  };
  sigma_block(BIT_A, S0_T, S0_BIT, S0_LO, 28, 34, 39, false);
  sigma_block(BIT_E, S1_T, S1_BIT, S1_LO, 14, 18, 41, false);
  sigma_block(BIT_WW1, SS0_T, SS0_BIT, SS0_LO, 1, 8, 7, true);
  sigma_block(BIT_WW14, SS1_T, SS1_BIT, SS1_LO, 19, 61, 6, true);
  for (int i = 0; i < 64; ++i) {
    Fp e = cur[BIT_E + i], f = cur[BIT_F + i], g = cur[BIT_G + i];
    push(cur[CH_BIT + i] - (e * f + g - e * g));
  }
  push(cur[CH_LO] - pack(CH_BIT));
  push(cur[CH_HI] - pack(CH_BIT + 32));
  for (int i = 0; i < 64; ++i) {
    Fp a = cur[BIT_A + i], b = cur[BIT_B + i], c = cur[BIT_C + i];
    push(cur[MAJ_AB + i] - a * b);
    push(cur[MAJ_AC + i] - a * c);
    push(cur[MAJ_BC + i] - b * c);
  }
  for (int i = 0; i < 64; ++i) push(cur[MAJ_U + i] - xr(cur[MAJ_AB + i], cur[MAJ_AC + i]));
  for (int i = 0; i < 64; ++i) push(cur[MAJ_BIT + i] - xr(cur[MAJ_U + i], cur[MAJ_BC + i]));
  push(cur[MAJ_LO] - pack(MAJ_BIT));
  push(cur[MAJ_HI] - pack(MAJ_BIT + 32));
  const uint64_t kt = comp ? K[br] : 0;
  const Fp klo(lo32(kt)), khi(hi32(kt));
  push(cur[T1_LO_LO] + p32 * cur[T1_LO_CW] - (cur[A_LO + 14] + cur[S1_LO] + cur[CH_LO] + klo + cur[W_LO]));
  for (size_t off : {(size_t)T1_LO_C0, (size_t)T1_LO_C1, (size_t)T1_LO_C2}) push(cur[off] * (one - cur[off]));
  push(cur[T1_LO_CW] - cur[T1_LO_C0] - two * cur[T1_LO_C1] - four * cur[T1_LO_C2]);
  push(cur[T1_HI_LO] + p32 * cur[T1_HI_CW] -
       (cur[A_LO + 15] + cur[S1_HI] + cur[CH_HI] + khi + cur[W_HI] + cur[T1_LO_CW]));
  for (size_t off : {(size_t)T1_HI_C0, (size_t)T1_HI_C1, (size_t)T1_HI_C2}) push(cur[off] * (one - cur[off]));
  push(cur[T1_HI_CW] - cur[T1_HI_C0] - two * cur[T1_HI_C1] - four * cur[T1_HI_C2]);
  push(cur[T2_LO_LO] + p32 * cur[T2_LO_CW] - (cur[S0_LO] + cur[MAJ_LO]));
  push(cur[T2_LO_C0] * (one - cur[T2_LO_C0]));
  push(cur[T2_LO_CW] - cur[T2_LO_C0]);
  push(cur[T2_HI_LO] + p32 * cur[T2_HI_CW] - (cur[S0_HI] + cur[MAJ_HI] + cur[T2_LO_CW]));
  push(cur[T2_HI_C0] * (one - cur[T2_HI_C0]));
  push(cur[T2_HI_CW] - cur[T2_HI_C0]);
  // working-register shifts b<-a, c<-b, d<-c, f<-e, g<-f, h<-g (lo, hi)
  const int shifts[6][2] = {{1, 0}, {2, 1}, {3, 2}, {5, 4}, {6, 5}, {7, 6}};
  for (auto& sh : shifts) {
    push(comp ? nxt[A_LO + 2 * sh[0]] - cur[A_LO + 2 * sh[1]] : Fp());
    push(comp ? nxt[A_LO + 2 * sh[0] + 1] - cur[A_LO + 2 * sh[1] + 1] : Fp());
  }
  if (comp) {
    push(nxt[A_LO] + p32 * cur[NA_LO_C] - cur[T1_LO_LO] - cur[T2_LO_LO]);
    push(cur[NA_LO_C] * (one - cur[NA_LO_C]));
    push(nxt[A_LO + 1] + p32 * cur[NA_HI_C] - cur[T1_HI_LO] - cur[T2_HI_LO] - cur[NA_LO_C]);
    push(cur[NA_HI_C] * (one - cur[NA_HI_C]));
    push(nxt[A_LO + 8] + p32 * cur[NE_LO_C] - cur[A_LO + 6] - cur[T1_LO_LO]);
    push(cur[NE_LO_C] * (one - cur[NE_LO_C]));
    push(nxt[A_LO + 9] + p32 * cur[NE_HI_C] - cur[A_LO + 7] - cur[T1_HI_LO] - cur[NE_LO_C]);
    push(cur[NE_HI_C] * (one - cur[NE_HI_C]));
  } else {
    for (int i = 0; i < 8; ++i) push(Fp());
  }
  static const Fp inv32 = inv(Fp::raw(1ull << 32));
  for (int k = 0; k < 8; ++k) {
    const size_t hl = H0_LO + 2 * k, al = A_LO + 2 * k;
    if (fin) {
      const Fp dlo = cur[hl] + cur[al] - nxt[hl];
      const Fp dhi = cur[hl + 1] + cur[al + 1] + dlo * inv32 - nxt[hl + 1];
      push(dlo * (dlo - p32));
      push(dhi * (dhi - p32));
    } else {
      push(nxt[hl] - cur[hl]);
      push(nxt[hl + 1] - cur[hl + 1]);
    }
  }
  for (int k = 0; k < 14; ++k) {
    push(nxt[WW0_LO + 2 * k] - cur[WW0_LO + 2 * (k + 1)]);
    push(nxt[WW0_LO + 2 * k + 1] - cur[WW0_LO + 2 * (k + 1) + 1]);
  }
  push(nxt[WW0_LO + 28] - cur[W_LO]);
  push(nxt[WW0_LO + 29] - cur[W_HI]);
  if (sched) {
    push(nxt[W_LO] + p32 * cur[WS_LO_CW] - (cur[WW0_LO] + cur[SS0_LO] + cur[WW0_LO + 18] + cur[SS1_LO]));
    push(cur[WS_LO_C0] * (one - cur[WS_LO_C0]));
    push(cur[WS_LO_C1] * (one - cur[WS_LO_C1]));
    push(cur[WS_LO_CW] - cur[WS_LO_C0] - two * cur[WS_LO_C1]);
    push(nxt[W_HI] + p32 * cur[WS_HI_CW] -
         (cur[WW0_LO + 1] + cur[SS0_HI] + cur[WW0_LO + 19] + cur[SS1_HI] + cur[WS_LO_CW]));
    push(cur[WS_HI_C0] * (one - cur[WS_HI_C0]));
    push(cur[WS_HI_C1] * (one - cur[WS_HI_C1]));
    push(cur[WS_HI_CW] - cur[WS_HI_C0] - two * cur[WS_HI_C1]);
  } else {
    for (int i = 0; i < 8; ++i) push(Fp());
  }
}

}  // namespace sha512
}  // namespace orc

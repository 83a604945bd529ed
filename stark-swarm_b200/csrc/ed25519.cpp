// ed25519.cpp — host side of the Ed25519 verify AIR: arithmetic mod 2^255 - 19 and
// on Edwards25519, the v16 layout, the constraint program and the trace witness.
//
// Every cell of the reference's trace is a canonical limb, a bit of one, a carry
// (0/1, -1/0/1 as a pos/neg pair, or a signed value biased into 36 or 24 bits),
// a constant, or a SHA-512 cell. The values are fixed by exact integer arithmetic
// (the reference fills each gadget from canonicalised inputs and its canonical
// output, ed25519_group_air.rs:251-321, ed25519_field_air.rs:330-996), so this
// builder computes them with 256-bit integers mod p and replays each carry chain
// from the integer relation it encodes.
#include "ed25519.hpp"

#include <algorithm>
#include <map>
#include <cstring>
#include <atomic>
#include <exception>
#include <thread>

#include "bigint.hpp"
#include "context.hpp"
#include "keccak.cuh"

namespace sg {
namespace ed25519 {
namespace {

// ------------------------------------------------------------------ F_p, p = 2^255 - 19
struct F {
  uint64_t v[4] = {0, 0, 0, 0};  // canonical, little-endian words
};
constexpr uint64_t P0 = 0xFFFFFFFFFFFFFFEDull, P1 = ~0ull, P2 = ~0ull, P3 = 0x7FFFFFFFFFFFFFFFull;

bool geq_p(const uint64_t a[4]) {
  if (a[3] != P3) return a[3] > P3;
  if (a[2] != P2) return a[2] > P2;
  if (a[1] != P1) return a[1] > P1;
  return a[0] >= P0;
}
void sub_p(uint64_t a[4]) {
  const uint64_t p[4] = {P0, P1, P2, P3};
  unsigned __int128 br = 0;
  for (int i = 0; i < 4; ++i) {
    const unsigned __int128 t = (unsigned __int128)a[i] - p[i] - br;
    a[i] = (uint64_t)t;
    br = (t >> 64) & 1;
  }
}
// a value below 2^256 to canonical form
F canon(const uint64_t a[4]) {
  F r;
  memcpy(r.v, a, 32);
  while (geq_p(r.v)) sub_p(r.v);
  return r;
}
F fe(uint64_t x) {
  F r;
  r.v[0] = x;
  return r;
}
bool eq(const F& a, const F& b) { return memcmp(a.v, b.v, 32) == 0; }
bool is_zero(const F& a) { return !(a.v[0] | a.v[1] | a.v[2] | a.v[3]); }
F add(const F& a, const F& b) {
  uint64_t s[4];
  unsigned __int128 c = 0;
  for (int i = 0; i < 4; ++i) {
    c += (unsigned __int128)a.v[i] + b.v[i];
    s[i] = (uint64_t)c;
    c >>= 64;
  }
  // a + b < 2p < 2^256: no carry out
  return canon(s);
}
F neg(const F& a) {
  if (is_zero(a)) return a;
  const uint64_t p[4] = {P0, P1, P2, P3};
  F r;
  unsigned __int128 br = 0;
  for (int i = 0; i < 4; ++i) {
    const unsigned __int128 t = (unsigned __int128)p[i] - a.v[i] - br;
    r.v[i] = (uint64_t)t;
    br = (t >> 64) & 1;
  }
  return r;
}
F sub(const F& a, const F& b) { return add(a, neg(b)); }
F mul(const F& a, const F& b) {
  uint64_t t[8] = {0};
  for (int i = 0; i < 4; ++i) {
    unsigned __int128 c = 0;
    for (int j = 0; j < 4; ++j) {
      c += (unsigned __int128)a.v[i] * b.v[j] + t[i + j];
      t[i + j] = (uint64_t)c;
      c >>= 64;
    }
    t[i + 4] = (uint64_t)c;
  }
  // 2^256 = 38 (mod p): fold the high half twice, then at most one more small carry
  uint64_t r[4];
  unsigned __int128 c = 0;
  for (int i = 0; i < 4; ++i) {
    c += (unsigned __int128)t[i] + (unsigned __int128)t[i + 4] * 38;
    r[i] = (uint64_t)c;
    c >>= 64;
  }
  uint64_t top = (uint64_t)c;
  while (top) {
    unsigned __int128 d = (unsigned __int128)top * 38;
    top = 0;
    for (int i = 0; i < 4; ++i) {
      d += r[i];
      r[i] = (uint64_t)d;
      d >>= 64;
    }
    top = (uint64_t)d;
  }
  return canon(r);
}
F pow(F a, const uint64_t e[4]) {
  F r = fe(1);
  for (int w = 3; w >= 0; --w)
    for (int b = 63; b >= 0; --b) {
      r = mul(r, r);
      if ((e[w] >> b) & 1) r = mul(r, a);
    }
  return r;
}
F inv(const F& a) {
  const uint64_t e[4] = {P0 - 2, P1, P2, P3};
  return pow(a, e);
}
// the value mod p of 10 non-negative limbs below 2^32 (canonical ones, or the
// doubled limbs of 2d)
F pack(const uint32_t l[NL]) {
  uint64_t acc[5] = {0};
  for (int i = 0; i < NL; ++i) {
    const unsigned w = LOFF[i] / 64, s = LOFF[i] % 64;
    const unsigned __int128 v = (unsigned __int128)l[i] << s;
    unsigned __int128 c = (unsigned __int128)acc[w] + (uint64_t)v;
    acc[w] = (uint64_t)c;
    c = (c >> 64) + (uint64_t)(v >> 64);
    for (unsigned j = w + 1; j < 5 && c; ++j) {
      c += acc[j];
      acc[j] = (uint64_t)c;
      c >>= 64;
    }
  }
  // 2^256 = 38 (mod p)
  unsigned __int128 c = (unsigned __int128)acc[4] * 38;
  for (int i = 0; i < 4; ++i) {
    c += acc[i];
    acc[i] = (uint64_t)c;
    c >>= 64;
  }
  if (c) {  // one more small fold
    unsigned __int128 d = (unsigned __int128)(uint64_t)c * 38;
    for (int i = 0; i < 4; ++i) {
      d += acc[i];
      acc[i] = (uint64_t)d;
      d >>= 64;
    }
  }
  return canon(acc);
}
void limbs_of(const F& x, uint32_t out[NL]) {
  for (int i = 0; i < NL; ++i) {
    const unsigned o = LOFF[i], w = o / 64, s = o % 64;
    uint64_t v = x.v[w] >> s;
    if (s + LW[i] > 64 && w + 1 < 4) v |= x.v[w + 1] << (64 - s);
    out[i] = (uint32_t)(v & ((1ull << LW[i]) - 1));
  }
}
F from_bytes_le(const uint8_t b[32], bool* canonical) {
  uint64_t a[4];
  memcpy(a, b, 32);
  a[3] &= 0x7FFFFFFFFFFFFFFFull;
  if (canonical) *canonical = !geq_p(a);
  return canon(a);
}

F d_const() {  // d = -121665 / 121666
  return mul(neg(fe(121665)), inv(fe(121666)));
}
F sqrt_m1() {  // 2^((p-1)/4)
  const uint64_t e[4] = {0xFFFFFFFFFFFFFFFBull, ~0ull, ~0ull, 0x1FFFFFFFFFFFFFFFull};
  return pow(fe(2), e);
}

// ------------------------------------------------------------------ Edwards25519
struct Pt {
  F X, Y, Z, T;
};
Pt identity() { return {fe(0), fe(1), fe(1), fe(0)}; }
const F& D() {
  static const F d = d_const();
  return d;
}
const F& D2() {
  static const F d2 = add(D(), D());
  return d2;
}
// EdwardsPoint::add (ed25519_group.rs:101-126)
Pt padd(const Pt& p, const Pt& q) {
  const F a = mul(sub(p.Y, p.X), sub(q.Y, q.X)), b = mul(add(p.Y, p.X), add(q.Y, q.X));
  const F c = mul(mul(p.T, q.T), D2()), d = add(mul(p.Z, q.Z), mul(p.Z, q.Z));
  const F e = sub(b, a), f = sub(d, c), g = add(d, c), h = add(b, a);
  return {mul(e, f), mul(g, h), mul(f, g), mul(e, h)};
}
// EdwardsPoint::double (ed25519_group.rs:147-165)
Pt pdbl(const Pt& p) {
  const F a = mul(p.X, p.X), b = mul(p.Y, p.Y), zz = mul(p.Z, p.Z), c = add(zz, zz), h = add(a, b);
  const F xy = add(p.X, p.Y), e = sub(h, mul(xy, xy)), g = sub(a, b), f = add(c, g);
  return {mul(e, f), mul(g, h), mul(f, g), mul(e, h)};
}
Pt pneg(const Pt& p) { return {neg(p.X), p.Y, p.Z, neg(p.T)}; }
// EdwardsPoint::decompress (ed25519_group.rs:204-232): x^2 = (y^2 - 1)/(d y^2 + 1),
// the root of the encoded parity. false for y >= p, a non-square, or x = 0 with the sign set.
bool decompress(const uint8_t b[32], Pt* out, F* y_out, int* sign_out) {
  bool canonical = false;
  const F y = from_bytes_le(b, &canonical);
  const int sign = b[31] >> 7;
  if (!canonical) return false;
  const F yy = mul(y, y), u = sub(yy, fe(1)), v = add(mul(D(), yy), fe(1));
  const F x2 = mul(u, inv(v));
  const uint64_t e[4] = {0xFFFFFFFFFFFFFFFEull, ~0ull, ~0ull, 0x0FFFFFFFFFFFFFFFull};  // (p + 3) / 8
  F x = pow(x2, e);
  if (!eq(mul(x, x), x2)) x = mul(x, sqrt_m1());
  if (!eq(mul(x, x), x2)) return false;
  if ((int)(x.v[0] & 1) != sign) {
    if (is_zero(x)) return false;
    x = neg(x);
  }
  *out = {x, y, fe(1), mul(x, y)};
  if (y_out) *y_out = y;
  if (sign_out) *sign_out = sign;
  return true;
}
const Pt& basepoint() {
  static const Pt b = [] {
    uint8_t enc[32];
    enc[0] = 0x58;
    memset(enc + 1, 0x66, 31);
    Pt p;
    decompress(enc, &p, nullptr, nullptr);
    return p;
  }();
  return b;
}
Pt ladder(const Pt& base, const uint8_t* bits, uint32_t k) {
  Pt acc = identity();
  for (uint32_t i = 0; i < k; ++i) {
    acc = pdbl(acc);
    if (bits[i]) acc = padd(acc, base);
  }
  return acc;
}
bool is_identity(const Pt& p) { return is_zero(p.X) && eq(p.Y, p.Z) && !is_zero(p.Z); }

// L = 2^252 + 27742317777372353535851937790883648493 as 32-bit words
constexpr uint32_t L32[8] = {0x5cf5d3ed, 0x5812631a, 0xa2f79cd6, 0x14def9de, 0, 0, 0, 0x10000000};
// x (nw 32-bit words, little-endian) mod L, and the quotient (nq words)
void divmod_L(const uint32_t* x, int nw, uint32_t r[8], uint32_t* q, int nq) {
  std::vector<uint32_t> qq(nw - 8 + 1), rr(8);
  bn::divmod(x, nw, L32, 8, qq.data(), rr.data());
  memcpy(r, rr.data(), 32);
  if (q) {
    memset(q, 0, 4 * nq);
    memcpy(q, qq.data(), 4 * std::min<int>(nq, (int)qq.size()));
  }
}
bool scalar_canonical(const uint8_t s[32]) {
  uint32_t w[8];
  memcpy(w, s, 32);
  return bn::cmp(w, L32, 8) < 0;
}
// the k low bits of a little-endian 256-bit scalar, most significant first
// (s_bits_for_ladder, swarm-dns/src/prover.rs:829-839; r_thread_bits_for_kA, ed25519_verify_air.rs:1881-1893)
void ladder_bits(const uint8_t s[32], uint32_t k, uint8_t* out) {
  for (uint32_t i = 0; i < k; ++i) {
    const uint32_t b = k - 1 - i;
    out[i] = (s[b / 8] >> (b % 8)) & 1;
  }
}

// ------------------------------------------------------------------ layout
struct Alloc {
  uint32_t next;
  uint32_t take(uint32_t n) {
    const uint32_t r = next;
    next += n;
    return r;
  }
  GSub sub(uint32_t a, uint32_t b) {
    GSub g{a, b, 0, 0, 0, 0};
    g.c = take(NL);
    g.bits = take(255);
    g.pos = take(NL);
    g.neg = take(NL);
    return g;
  }
  GAdd add(uint32_t a, uint32_t b) {
    GAdd g{a, b, 0, 0, 0};
    g.c = take(NL);
    g.bits = take(255);
    g.carries = take(NL);
    return g;
  }
  GMul mul(uint32_t a, uint32_t b) {
    GMul g{a, b, 0, 0, 0};
    g.c = take(NL);
    g.bits = take(255);
    g.carry = take(MUL_CB * NL);
    return g;
  }
};

PAdd point_add_layout(uint32_t base, const uint32_t p1[4], const uint32_t p2[4]) {
  Alloc al{base};
  PAdd g;
  memcpy(g.p1, p1, 16);
  memcpy(g.p2, p2, 16);
  g.d2 = al.take(NL);
  g.sub_ym1 = al.sub(p1[1], p1[0]);
  g.sub_ym2 = al.sub(p2[1], p2[0]);
  g.add_yp1 = al.add(p1[1], p1[0]);
  g.add_yp2 = al.add(p2[1], p2[0]);
  g.mul_A = al.mul(g.sub_ym1.c, g.sub_ym2.c);
  g.mul_B = al.mul(g.add_yp1.c, g.add_yp2.c);
  g.mul_tt = al.mul(p1[3], p2[3]);
  g.mul_C = al.mul(g.mul_tt.c, g.d2);
  g.mul_zz = al.mul(p1[2], p2[2]);
  g.add_D = al.add(g.mul_zz.c, g.mul_zz.c);
  g.sub_E = al.sub(g.mul_B.c, g.mul_A.c);
  g.sub_F = al.sub(g.add_D.c, g.mul_C.c);
  g.add_G = al.add(g.add_D.c, g.mul_C.c);
  g.add_H = al.add(g.mul_B.c, g.mul_A.c);
  g.mul_X3 = al.mul(g.sub_E.c, g.sub_F.c);
  g.mul_Y3 = al.mul(g.add_G.c, g.add_H.c);
  g.mul_T3 = al.mul(g.sub_E.c, g.add_H.c);
  g.mul_Z3 = al.mul(g.sub_F.c, g.add_G.c);
  g.out[0] = g.mul_X3.c;
  g.out[1] = g.mul_Y3.c;
  g.out[2] = g.mul_Z3.c;
  g.out[3] = g.mul_T3.c;
  g.end = al.next;
  return g;
}

PDbl point_double_layout(uint32_t base, uint32_t x, uint32_t y, uint32_t z) {
  Alloc al{base};
  PDbl g;
  g.p1[0] = x;
  g.p1[1] = y;
  g.p1[2] = z;
  g.sq_A = al.mul(x, x);
  g.sq_B = al.mul(y, y);
  g.sq_zz = al.mul(z, z);
  g.add_C = al.add(g.sq_zz.c, g.sq_zz.c);
  g.add_H = al.add(g.sq_A.c, g.sq_B.c);
  g.add_xy = al.add(x, y);
  g.sq_xy = al.mul(g.add_xy.c, g.add_xy.c);
  g.sub_E = al.sub(g.add_H.c, g.sq_xy.c);
  g.sub_G = al.sub(g.sq_A.c, g.sq_B.c);
  g.add_F = al.add(g.add_C.c, g.sub_G.c);
  g.mul_X3 = al.mul(g.sub_E.c, g.add_F.c);
  g.mul_Y3 = al.mul(g.sub_G.c, g.add_H.c);
  g.mul_T3 = al.mul(g.sub_E.c, g.add_H.c);
  g.mul_Z3 = al.mul(g.add_F.c, g.sub_G.c);
  g.out[0] = g.mul_X3.c;
  g.out[1] = g.mul_Y3.c;
  g.out[2] = g.mul_Z3.c;
  g.out[3] = g.mul_T3.c;
  g.end = al.next;
  return g;
}

CAdd cond_add_layout(uint32_t base, const uint32_t acc[4], const uint32_t bp[4]) {
  Alloc al{base};
  CAdd g;
  g.bit = al.take(1);
  for (int q = 0; q < 4; ++q) g.out[q] = al.take(NL);
  g.add = point_add_layout(al.next, acc, bp);
  al.next = g.add.end;
  for (int q = 0; q < 4; ++q) g.sel[q] = GSel{acc[q], g.add.out[q], g.bit, g.out[q]};
  g.end = al.next;
  return g;
}

Decomp decompress_layout(uint32_t base, uint32_t y, uint32_t sign) {
  Alloc al{base};
  Decomp g;
  g.y = y;
  g.sign = sign;
  g.d = al.take(NL);
  g.x = al.take(NL);
  g.x_bits = al.take(255);
  g.sq_x = al.mul(g.x, g.x);
  g.sq_y = al.mul(y, y);
  g.mul_dx2 = al.mul(g.d, g.sq_x.c);
  g.mul_dxy = al.mul(g.mul_dx2.c, g.sq_y.c);
  g.one = al.take(NL);
  g.sub_y2m1 = al.sub(g.sq_y.c, g.one);
  g.sub_lhs = al.sub(g.sub_y2m1.c, g.sq_x.c);
  g.sub_eq = al.sub(g.sub_lhs.c, g.mul_dxy.c);
  g.sign_match = al.take(1);
  g.end = al.next;
  return g;
}

uint32_t next_pow2(uint32_t x) {
  uint32_t h = 1;
  while (h < x) h <<= 1;
  return h;
}

}  // namespace

uint32_t n_constraints(uint32_t k) {
  const uint32_t PA_K = NL + 4 * SUB_K + 5 * ADD_K + 9 * MUL_K, DBL_K = 8 * MUL_K + 4 * ADD_K + 2 * SUB_K;
  const uint32_t DECOMP_K = NL + ELEM + 4 * MUL_K + 3 * SUB_K + NL + 2;
  const uint32_t fixed = SHA_K + REDUCE_K + FORMAT_K + 2 * DECOMP_K + 2 * (DBL_K + PA_K + 4 * SEL_K + 80 + 40) + 80 +
                         22 + 2 + (NL + 3 * SUB_K + 3 * NL) + DBL_K + 30 + 40 + 4 * 40 + 40 + 10 + MUL_K + 40 +
                         (NL + 2 * SUB_K + PA_K) + (2 * SUB_K + PA_K) + 30;
  return fixed + 7 * k - 2;
}

Layout make_layout(uint64_t sha_len, uint32_t k) {
  require(k >= 2 && k <= K_FULL, "ed25519: k_scalar must be in [2, 256]");
  Layout L;
  L.k = k;
  L.n_blocks = (uint32_t)((sha_len + 1 + 16 + 127) / 128);
  require(L.n_blocks <= (1u << 14), "ed25519: message too long");
  L.k_hash = next_pow2(std::max<uint32_t>(128, 128 * L.n_blocks));
  L.reduce_row = L.k_hash;
  L.decomp_R_row = L.k_hash + 1;
  L.decomp_A_row = L.k_hash + 2;
  L.sB_first = L.k_hash + 3;
  L.sB_last = L.sB_first + k - 1;
  L.kA_first = L.sB_first + k;
  L.kA_last = L.kA_first + k - 1;
  L.residual_row = L.kA_last + 1;
  for (int i = 0; i < 3; ++i) L.dbl_row[i] = L.kA_last + 2 + i;
  L.result_row = L.kA_last + 5;
  // v0: the reduction at columns 0.. of its row
  uint32_t nx = RED_IN;
  L.red.input = 0;
  L.red.q = nx, nx += RED_Q;
  L.red.q_bits = nx, nx += RED_Q * RED_LB;
  L.red.r = nx, nx += RED_R;
  L.red.r_bits = nx, nx += RED_R * RED_LB;
  L.red.slack = nx, nx += RED_R;
  L.red.slack_bits = nx, nx += RED_R * RED_LB;
  L.red.carry_bits = nx;
  L.digest_bits = SHA_W;  // v1
  L.decomp = decompress_layout(NL + 1, 0, NL);  // v2
  // the ladder row (ed25519_scalar_mult_air.rs:93-131)
  for (int q = 0; q < 4; ++q) {
    L.base[q] = q * NL;
    L.acc[q] = 40 + q * NL;
  }
  L.mdbl = point_double_layout(80, L.acc[0], L.acc[1], L.acc[2]);
  L.cadd = cond_add_layout(L.mdbl.end, L.mdbl.out, L.base);
  const uint32_t w3 = L.cadd.end;  // 14941
  L.sblock_sB = w3;  // v6
  L.sblock_kA = w3 + k;
  L.r_thread = w3 + 2 * k;  // v7
  nx = w3 + 3 * k;
  for (int q = 0; q < 4; ++q) L.result[q] = nx + q * NL;  // v10
  nx += 4 * NL;
  L.zero_const = nx;
  nx += NL;
  Alloc al{nx};
  L.sub_X = al.sub(L.result[0], L.zero_const);
  L.sub_T = al.sub(L.result[3], L.zero_const);
  L.sub_YZ = al.sub(L.result[1], L.result[2]);
  for (int q = 0; q < 3; ++q) L.dbl_in[q] = al.take(NL);
  L.dbl = point_double_layout(al.next, L.dbl_in[0], L.dbl_in[1], L.dbl_in[2]);
  nx = L.dbl.end;
  for (int q = 0; q < 4; ++q) L.thr_sB[q] = nx + q * NL;  // v11
  nx += 4 * NL;
  for (int q = 0; q < 4; ++q) L.thr_kA[q] = nx + q * NL;  // v12
  nx += 4 * NL;
  for (int q = 0; q < 4; ++q) L.thr_R[q] = nx + q * NL;  // v13
  nx += 4 * NL;
  L.one_R = nx;
  nx += NL;
  al = Alloc{nx};
  L.mul_RT = al.mul(L.thr_R[0], L.thr_R[1]);
  L.zero_R1 = al.take(NL);  // v14
  L.sub_negR_X = al.sub(L.zero_R1, L.thr_R[0]);
  L.sub_negR_T = al.sub(L.zero_R1, L.thr_R[3]);
  const uint32_t negR[4] = {L.sub_negR_X.c, L.thr_R[1], L.thr_R[2], L.sub_negR_T.c};
  L.pa_R1 = point_add_layout(al.next, L.thr_sB, negR);
  al = Alloc{L.pa_R1.end};  // v15
  L.sub_negkA_X = al.sub(L.zero_R1, L.thr_kA[0]);
  L.sub_negkA_T = al.sub(L.zero_R1, L.thr_kA[3]);
  const uint32_t negkA[4] = {L.sub_negkA_X.c, L.thr_kA[1], L.thr_kA[2], L.sub_negkA_T.c};
  L.pa_R2 = point_add_layout(al.next, L.pa_R1.out, negkA);
  L.width = L.pa_R2.end;
  // heights of v3, v10 and v14 (ed25519_verify_air.rs:915,2774,3997)
  uint32_t h = next_pow2(L.kA_last + 1);
  if (h < L.kA_last + 6) h = next_pow2(L.kA_last + 5);
  if (h < L.kA_last + 7) h = next_pow2(L.kA_last + 6);
  L.height = h;
  L.n_constraints = n_constraints(k);
  return L;
}

namespace {

// ------------------------------------------------------------------ program
struct ProgBuilder {
  Program& P;
  void blk(uint32_t gate, uint32_t g0, uint32_t g1, uint32_t g2, uint32_t kind, std::initializer_list<uint32_t> ps,
           uint32_t count) {
    Block b{};
    b.gate = gate;
    b.g[0] = g0;
    b.g[1] = g1;
    b.g[2] = g2;
    b.kind = kind;
    int i = 0;
    for (uint32_t p : ps) b.p[i++] = p;
    b.lam = P.n_constraints;
    b.count = count;
    P.blocks.push_back(b);
    P.n_constraints += count;
  }
  struct Gate {
    uint32_t kind, g0 = ~0u, g1 = ~0u, g2 = ~0u;
  };
  void gadget(const Gate& G, const GMul& g) {
    blk(G.kind, G.g0, G.g1, G.g2, B_MUL, {g.a, g.b, g.c, g.bits, g.carry}, MUL_K);
  }
  void gadget(const Gate& G, const GAdd& g) {
    blk(G.kind, G.g0, G.g1, G.g2, B_ADD, {g.a, g.b, g.c, g.bits, g.carries}, ADD_K);
  }
  void gadget(const Gate& G, const GSub& g) {
    blk(G.kind, G.g0, G.g1, G.g2, B_SUB, {g.a, g.b, g.c, g.bits, g.pos, g.neg}, SUB_K);
  }
  void gadget(const Gate& G, const GSel& g) { blk(G.kind, G.g0, G.g1, G.g2, B_SEL, {g.a, g.b, g.bit, g.c}, SEL_K); }
  // pairs: (src, cell) - (src, cell or constant)
  std::vector<uint64_t> items;
  void pr(uint64_t sa, uint64_t a, uint64_t sb, uint64_t b) {
    items.push_back(sa << 62 | a);
    items.push_back(sb << 62 | b);
  }
  void flush(const Gate& G) {
    const uint32_t off = (uint32_t)(P.pairs.size() / 2), cnt = (uint32_t)(items.size() / 2);
    P.pairs.insert(P.pairs.end(), items.begin(), items.end());
    items.clear();
    blk(G.kind, G.g0, G.g1, G.g2, B_PAIRS, {off, cnt}, cnt);
  }
  void point_add(const Gate& G, const PAdd& g, const uint32_t d2[NL]) {
    for (int k = 0; k < NL; ++k) pr(SRC_CUR, g.d2 + k, SRC_CONST, d2[k]);
    flush(G);
    gadget(G, g.sub_ym1);
    gadget(G, g.sub_ym2);
    gadget(G, g.add_yp1);
    gadget(G, g.add_yp2);
    gadget(G, g.mul_A);
    gadget(G, g.mul_B);
    gadget(G, g.mul_tt);
    gadget(G, g.mul_C);
    gadget(G, g.mul_zz);
    gadget(G, g.add_D);
    gadget(G, g.sub_E);
    gadget(G, g.sub_F);
    gadget(G, g.add_G);
    gadget(G, g.add_H);
    gadget(G, g.mul_X3);
    gadget(G, g.mul_Y3);
    gadget(G, g.mul_T3);
    gadget(G, g.mul_Z3);
  }
  void point_double(const Gate& G, const PDbl& g) {
    gadget(G, g.sq_A);
    gadget(G, g.sq_B);
    gadget(G, g.sq_zz);
    gadget(G, g.add_C);
    gadget(G, g.add_H);
    gadget(G, g.add_xy);
    gadget(G, g.sq_xy);
    gadget(G, g.sub_E);
    gadget(G, g.sub_G);
    gadget(G, g.add_F);
    gadget(G, g.mul_X3);
    gadget(G, g.mul_Y3);
    gadget(G, g.mul_T3);
    gadget(G, g.mul_Z3);
  }
  void decompress(const Gate& G, const Decomp& g, const uint32_t d[NL]) {
    for (int k = 0; k < NL; ++k) pr(SRC_CUR, g.d + k, SRC_CONST, d[k]);
    flush(G);
    blk(G.kind, G.g0, G.g1, G.g2, B_RANGE, {g.x, g.x_bits}, ELEM);
    gadget(G, g.sq_x);
    gadget(G, g.sq_y);
    gadget(G, g.mul_dx2);
    gadget(G, g.mul_dxy);
    gadget(G, g.sub_y2m1);
    gadget(G, g.sub_lhs);
    gadget(G, g.sub_eq);
    for (int k = 0; k < NL; ++k) pr(SRC_CUR, g.sub_eq.c + k, SRC_CONST, 0);
    flush(G);
    blk(G.kind, G.g0, G.g1, G.g2, B_SIGN, {g.sign, g.x_bits}, 2);
  }
};

// eval_verify_air_v16_per_row (ed25519_verify_air.rs:4870-4960) as blocks, through the
// v15 .. v0 evaluators it delegates to (v10 builds on v7 directly: v8 and v9's own
// blocks are not part of v16).
Program make_program(const Layout& L, const uint8_t* s_bits, const uint8_t* k_bits, const F& r_y, int r_sign,
                     const F& a_y, int a_sign, const Pt& A) {
  using G = ProgBuilder::Gate;
  Program P;
  ProgBuilder b{P};
  const uint32_t K = L.k;
  uint32_t d[NL], d2[NL], one[NL];
  limbs_of(D(), d);
  for (int i = 0; i < NL; ++i) d2[i] = 2 * d[i];  // ed25519_field.rs:609: D.add(&D), limb-wise, not reduced
  limbs_of(fe(1), one);
  // v3 with v0 .. v2 inside
  b.blk(GATE_RANGE, 0, L.k_hash - 1, ~0u, B_SHA512, {L.n_blocks}, SHA_K);
  b.blk(GATE_EQ, L.reduce_row, ~0u, ~0u, B_REDUCE,
        {L.red.input, L.red.q, L.red.q_bits, L.red.r, L.red.r_bits, L.red.slack, L.red.slack_bits,
         L.red.carry_bits},
        REDUCE_K);
  b.blk(GATE_EQ, L.k_hash - 1, ~0u, ~0u, B_FORMAT, {L.digest_bits, L.red.input, SHA_H0_LO}, FORMAT_K);
  b.decompress(G{GATE_EQ, L.decomp_R_row}, L.decomp, d);
  b.decompress(G{GATE_EQ, L.decomp_A_row}, L.decomp, d);
  for (int ph = 0; ph < 2; ++ph) {
    const uint32_t first = ph ? L.kA_first : L.sB_first, last = ph ? L.kA_last : L.sB_last;
    const G rows{GATE_RANGE, first, last + 1};
    b.point_double(rows, L.mdbl);
    b.point_add(rows, L.cadd.add, d2);
    for (int q = 0; q < 4; ++q) b.gadget(rows, L.cadd.sel[q]);
    for (int k = 0; k < NL; ++k)
      for (int q = 0; q < 4; ++q) b.pr(SRC_NXT, L.base[q] + k, SRC_CUR, L.base[q] + k);
    for (int k = 0; k < NL; ++k)
      for (int q = 0; q < 4; ++q) b.pr(SRC_NXT, L.acc[q] + k, SRC_CUR, L.cadd.out[q] + k);
    b.flush(G{GATE_RANGE, first, last});
    for (int k = 0; k < NL; ++k)
      for (int q = 0; q < 4; ++q) b.pr(SRC_CUR, L.acc[q] + k, SRC_CONST, (q == 1 || q == 2) && k == 0 ? 1 : 0);
    b.flush(G{GATE_EQ, first});
  }
  // v4: the ladders' bases
  {
    const Pt& B = basepoint();
    const F* bc[4] = {&B.X, &B.Y, &B.Z, &B.T};
    const F* ac[4] = {&A.X, &A.Y, &A.Z, &A.T};
    for (int which = 0; which < 2; ++which) {
      for (int q = 0; q < 4; ++q) {
        uint32_t l[NL];
        limbs_of(which ? *ac[q] : *bc[q], l);
        for (int k = 0; k < NL; ++k) b.pr(SRC_CUR, L.base[q] + k, SRC_CONST, l[k]);
      }
      b.flush(G{GATE_EQ, which ? L.kA_first : L.sB_first});
    }
  }
  // v5: the decompressions' inputs
  for (int which = 0; which < 2; ++which) {
    uint32_t l[NL];
    limbs_of(which ? a_y : r_y, l);
    for (int k = 0; k < NL; ++k) b.pr(SRC_CUR, L.decomp.y + k, SRC_CONST, l[k]);
    b.pr(SRC_CUR, L.decomp.sign, SRC_CONST, (uint32_t)(which ? a_sign : r_sign));
    b.flush(G{GATE_EQ, which ? L.decomp_A_row : L.decomp_R_row});
  }
  // v6: scalar shift chains
  for (int which = 0; which < 2; ++which) {
    const uint32_t first = which ? L.kA_first : L.sB_first, last = which ? L.kA_last : L.sB_last;
    const uint32_t base = which ? L.sblock_kA : L.sblock_sB;
    const uint8_t* bits = which ? k_bits : s_bits;
    for (uint32_t i = 0; i < K; ++i) b.pr(SRC_CUR, base + i, SRC_CONST, bits[i]);
    b.flush(G{GATE_EQ, first});
    b.pr(SRC_CUR, L.cadd.bit, SRC_CUR, base);
    b.flush(G{GATE_RANGE, first, last + 1});
    for (uint32_t i = 0; i + 1 < K; ++i) b.pr(SRC_NXT, base + i, SRC_CUR, base + i + 1);
    b.flush(G{GATE_RANGE, first, last});
  }
  // v7: the r thread
  for (uint32_t i = 0; i < K; ++i) b.pr(SRC_CUR, L.r_thread + i, SRC_CUR, L.red.r_bits + K - 1 - i);
  b.flush(G{GATE_EQ, L.reduce_row});
  for (uint32_t i = 0; i < K; ++i) b.pr(SRC_NXT, L.r_thread + i, SRC_CUR, L.r_thread + i);
  b.flush(G{GATE_ALWAYS});
  for (uint32_t i = 0; i < K; ++i) b.pr(SRC_CUR, L.sblock_kA + i, SRC_CUR, L.r_thread + i);
  b.flush(G{GATE_EQ, L.kA_first});
  // v10: verdict, doubling chain, result binding
  {
    const G res{GATE_EQ, L.result_row};
    for (int i = 0; i < NL; ++i) b.pr(SRC_CUR, L.zero_const + i, SRC_CONST, 0);
    b.flush(res);
    b.gadget(res, L.sub_X);
    b.gadget(res, L.sub_T);
    b.gadget(res, L.sub_YZ);
    for (const GSub* g : {&L.sub_X, &L.sub_T, &L.sub_YZ})
      for (int i = 0; i < NL; ++i) b.pr(SRC_CUR, g->c + i, SRC_CONST, 0);
    b.flush(res);
    b.point_double(G{GATE_SET, L.dbl_row[0], L.dbl_row[1], L.dbl_row[2]}, L.dbl);
    for (int q = 0; q < 3; ++q)
      for (int i = 0; i < NL; ++i) b.pr(SRC_NXT, L.dbl_in[q] + i, SRC_CUR, L.dbl.out[q] + i);
    b.flush(G{GATE_SET, L.dbl_row[0], L.dbl_row[1], ~0u});
    for (int q = 0; q < 4; ++q)
      for (int i = 0; i < NL; ++i) b.pr(SRC_NXT, L.result[q] + i, SRC_CUR, L.dbl.out[q] + i);
    b.flush(G{GATE_EQ, L.dbl_row[2]});
  }
  // v11, v12: the ladders' output threads
  for (int which = 0; which < 2; ++which) {
    const uint32_t* thr = which ? L.thr_kA : L.thr_sB;
    for (int q = 0; q < 4; ++q)
      for (int i = 0; i < NL; ++i) b.pr(SRC_CUR, thr[q] + i, SRC_CUR, L.cadd.out[q] + i);
    b.flush(G{GATE_EQ, which ? L.kA_last : L.sB_last});
    for (int q = 0; q < 4; ++q)
      for (int i = 0; i < NL; ++i) b.pr(SRC_NXT, thr[q] + i, SRC_CUR, thr[q] + i);
    b.flush(G{GATE_ALWAYS});
  }
  // v13: the R thread with T = X Y in the circuit
  {
    const G rr{GATE_EQ, L.decomp_R_row};
    const uint32_t src[4] = {L.decomp.x, L.decomp.y, L.one_R, L.mul_RT.c};
    for (int q = 0; q < 4; ++q)
      for (int i = 0; i < NL; ++i) b.pr(SRC_CUR, L.thr_R[q] + i, SRC_CUR, src[q] + i);
    b.flush(rr);
    for (int i = 0; i < NL; ++i) b.pr(SRC_CUR, L.one_R + i, SRC_CONST, one[i]);
    b.flush(rr);
    b.gadget(rr, L.mul_RT);
    for (int q = 0; q < 4; ++q)
      for (int i = 0; i < NL; ++i) b.pr(SRC_NXT, L.thr_R[q] + i, SRC_CUR, L.thr_R[q] + i);
    b.flush(G{GATE_ALWAYS});
  }
  // v14, v15: the residual row; v16: residual_2 into the doubling chain
  {
    const G rs{GATE_EQ, L.residual_row};
    for (int i = 0; i < NL; ++i) b.pr(SRC_CUR, L.zero_R1 + i, SRC_CONST, 0);
    b.flush(rs);
    b.gadget(rs, L.sub_negR_X);
    b.gadget(rs, L.sub_negR_T);
    b.point_add(rs, L.pa_R1, d2);
    b.gadget(rs, L.sub_negkA_X);
    b.gadget(rs, L.sub_negkA_T);
    b.point_add(rs, L.pa_R2, d2);
    for (int q = 0; q < 3; ++q)
      for (int i = 0; i < NL; ++i) b.pr(SRC_NXT, L.dbl_in[q] + i, SRC_CUR, L.pa_R2.out[q] + i);
    b.flush(rs);
  }
  require(P.n_constraints == L.n_constraints, "ed25519: constraint count");
  return P;
}

// ------------------------------------------------------------------ witness emission
// Cells of one row: each value that cells are read from becomes a word; the codes
// of the row's phase are recorded on the phase's first row (every row of a phase
// emits the same cells in the same order).
struct Emit {
  std::vector<uint64_t>& words;
  uint32_t* codes;  // this phase's width codes, or null once recorded
  uint32_t nw = 0;
  uint32_t word(uint64_t v) {
    words.push_back(v);
    return nw++;
  }
  void set(uint32_t col, uint32_t c) {
    if (codes) codes[col] = c;
  }
  void value(uint32_t col, uint64_t v) { set(col, code(OP_WORD, word(v))); }
  void limbs(uint32_t base, const uint32_t l[NL]) {
    for (int i = 0; i < NL; ++i) value(base + i, l[i]);
  }
  // the nb bit cells of word w at col (codes of the phase's first row only)
  void bits(uint32_t col, uint32_t w, uint32_t nb) {
    if (codes)
      for (uint32_t b = 0; b < nb; ++b) codes[col + b] = code(OP_BIT, w, b);
  }
  // limbs and their 255 range bits
  void elem(uint32_t c, uint32_t bit_cells, const uint32_t l[NL]) {
    uint32_t off = 0;
    for (int i = 0; i < NL; ++i) {
      const uint32_t w = word(l[i]);
      set(c + i, code(OP_WORD, w));
      bits(bit_cells + off, w, LW[i]);
      off += LW[i];
    }
  }
};

inline int64_t lval(const uint32_t l[NL], int i) { return (int64_t)l[i]; }

// fill_add_gadget (ed25519_field_air.rs:330-418): c = a + b mod p, c = a + b - carry[9] p
F fill_add(Emit& e, const GAdd& g, const uint32_t a[NL], const uint32_t b[NL]) {
  const F av = pack(a), bv = pack(b), c = add(av, bv);
  uint32_t cl[NL];
  limbs_of(c, cl);
  e.elem(g.c, g.bits, cl);
  // a + b >= p exactly when the canonical sum wrapped
  uint64_t s[5] = {0};
  {
    unsigned __int128 cc = 0;
    for (int i = 0; i < 4; ++i) {
      cc += (unsigned __int128)av.v[i] + bv.v[i];
      s[i] = (uint64_t)cc;
      cc >>= 64;
    }
  }
  const int64_t top = geq_p(s) ? 1 : 0;
  int64_t prev = 19 * top;
  for (int k = 0; k < NL; ++k) {
    const int64_t d = lval(a, k) + lval(b, k) + prev - cl[k];
    const int64_t cy = d >> LW[k];
    require(cy * (1ll << LW[k]) == d && (cy == 0 || cy == 1), "ed25519 witness: add carry");
    e.value(g.carries + k, (uint64_t)cy);
    prev = cy;
  }
  require(prev == top, "ed25519 witness: add chain");
  return c;
}

// fill_sub_gadget (ed25519_field_air.rs:584-668): c = a - b + net[9] p, net in {-1, 0, 1}
F fill_sub(Emit& e, const GSub& g, const uint32_t a[NL], const uint32_t b[NL]) {
  const F av = pack(a), bv = pack(b), c = sub(av, bv);
  uint32_t cl[NL];
  limbs_of(c, cl);
  e.elem(g.c, g.bits, cl);
  const int64_t top = bn::cmp((const uint32_t*)av.v, (const uint32_t*)bv.v, 8) < 0 ? 1 : 0;
  int64_t prev = 19 * top;
  for (int k = 0; k < NL; ++k) {
    const int64_t v = lval(a, k) - lval(b, k) - prev, d = (int64_t)cl[k] - v;
    const int64_t net = d >> LW[k];
    require(net * (1ll << LW[k]) == d && net >= -1 && net <= 1, "ed25519 witness: sub carry");
    const uint32_t w = e.word((uint64_t)net);
    e.set(g.pos + k, code(OP_POS, w));
    e.set(g.neg + k, code(OP_NEG, w));
    prev = net;
  }
  require(prev == top, "ed25519 witness: sub chain");
  return c;
}

// fill_mul_gadget (ed25519_field_air.rs:874-996): T[k] = sum of f a_i b_j over the
// pairs that fold onto limb k (f = 2 for two odd limbs, x 19 across 2^255),
// T[k] + carry_in[k] = c[k] + carry[k] 2^w_k with carry_in[0] = 19 carry[9], so
// sum T[k] 2^off_k - c = carry[9] p; the carries go out biased by 2^35.
F fill_mul(Emit& e, const GMul& g, const uint32_t a[NL], const uint32_t b[NL]) {
  const F c = mul(pack(a), pack(b));
  uint32_t cl[NL];
  limbs_of(c, cl);
  e.elem(g.c, g.bits, cl);
  // limbs below 2^27 (the unreduced 2d constant; the others below 2^26): a sum of ten
  // products times at most 38 stays below 10 * 38 * 2^54 < 2^63
  int64_t t64[NL] = {0};
  for (int i = 0; i < NL; ++i)
    for (int j = 0; j < NL; ++j) {
      int64_t f = ((i & 1) && (j & 1)) ? 2 : 1;
      int s = i + j;
      if (s >= NL) s -= NL, f *= 19;
      t64[s] += f * ((int64_t)a[i] * (int64_t)b[j]);
    }
  __int128 t[NL];
  for (int k = 0; k < NL; ++k) t[k] = t64[k];
  // S = sum (T[k] - c[k]) 2^off_k in a 320-bit two's-complement accumulator; S = x p
  uint64_t acc[5] = {0};
  for (int k = 0; k < NL; ++k) {
    const __int128 u = t[k] - cl[k];
    const unsigned sh = LOFF[k], w0 = sh / 64, bs = sh % 64;
    // u 2^bs spans up to three words (|u| < 2^63); sign-extended over the rest
    uint64_t part[5] = {0};
    const unsigned __int128 uu = (unsigned __int128)u;
    const uint64_t lo = (uint64_t)uu, hi = (uint64_t)(uu >> 64);
    const uint64_t ext = u < 0 ? ~0ull : 0;
    uint64_t words3[3] = {lo << bs, bs ? (hi << bs | lo >> (64 - bs)) : hi, bs ? (ext << bs | hi >> (64 - bs)) : ext};
    for (unsigned i = 0; i < 5; ++i) part[i] = i < w0 ? 0 : (i - w0 < 3 ? words3[i - w0] : ext);
    unsigned __int128 cc = 0;
    for (int i = 0; i < 5; ++i) {
      cc += (unsigned __int128)acc[i] + part[i];
      acc[i] = (uint64_t)cc;
      cc >>= 64;
    }
  }
  // x = floor(S / 2^255) + (S > 0): S = x 2^255 - 19 x with |19 x| < 2^255
  const int64_t fl = (int64_t)(acc[3] >> 63 | acc[4] << 1);
  const bool pos = !((int64_t)acc[4] < 0) && (acc[0] | acc[1] | acc[2] | acc[3] | acc[4]);
  const __int128 x = (__int128)fl + (pos ? 1 : 0);
  __int128 prev = 19 * x;
  const __int128 half = (__int128)1 << (MUL_CB - 1);
  for (int k = 0; k < NL; ++k) {
    const __int128 d = t[k] + prev - cl[k];
    const __int128 cy = d >> LW[k];
    require(cy * ((__int128)1 << LW[k]) == d && cy >= -half && cy < half, "ed25519 witness: mul carry");
    const uint32_t w = e.word((uint64_t)(cy + half));
    e.bits(g.carry + k * MUL_CB, w, MUL_CB);
    prev = cy;
  }
  require(prev == x, "ed25519 witness: mul chain");
  return c;
}

void fill_sel(Emit& e, const GSel& g, const uint32_t a[NL], const uint32_t b[NL], int bit) {
  e.value(g.bit, (uint64_t)bit);
  e.limbs(g.c, bit ? b : a);
}

struct PtL {  // canonical limbs of X, Y, Z, T
  uint32_t l[4][NL];
};
PtL limbs_pt(const Pt& p) {
  PtL r;
  limbs_of(p.X, r.l[0]);
  limbs_of(p.Y, r.l[1]);
  limbs_of(p.Z, r.l[2]);
  limbs_of(p.T, r.l[3]);
  return r;
}

// fill_point_add_gadget (ed25519_group_air.rs:251-321)
Pt fill_point_add(Emit& e, const PAdd& g, const Pt& p1, const Pt& p2, const uint32_t d2[NL]) {
  e.limbs(g.d2, d2);
  const PtL A1 = limbs_pt(p1), A2 = limbs_pt(p2);
  uint32_t t0[NL], t1[NL], t2[NL], t3[NL], t4[NL], t5[NL], t6[NL], t7[NL], t8[NL], t9[NL];
  limbs_of(fill_sub(e, g.sub_ym1, A1.l[1], A1.l[0]), t0);  // ym1
  limbs_of(fill_sub(e, g.sub_ym2, A2.l[1], A2.l[0]), t1);  // ym2
  limbs_of(fill_add(e, g.add_yp1, A1.l[1], A1.l[0]), t2);  // yp1
  limbs_of(fill_add(e, g.add_yp2, A2.l[1], A2.l[0]), t3);  // yp2
  limbs_of(fill_mul(e, g.mul_A, t0, t1), t4);              // A
  limbs_of(fill_mul(e, g.mul_B, t2, t3), t5);              // B
  limbs_of(fill_mul(e, g.mul_tt, A1.l[3], A2.l[3]), t6);   // tt
  limbs_of(fill_mul(e, g.mul_C, t6, d2), t7);              // C
  limbs_of(fill_mul(e, g.mul_zz, A1.l[2], A2.l[2]), t8);   // zz
  limbs_of(fill_add(e, g.add_D, t8, t8), t9);              // D
  uint32_t E[NL], Fl[NL], Gl[NL], H[NL];
  limbs_of(fill_sub(e, g.sub_E, t5, t4), E);
  limbs_of(fill_sub(e, g.sub_F, t9, t7), Fl);
  limbs_of(fill_add(e, g.add_G, t9, t7), Gl);
  limbs_of(fill_add(e, g.add_H, t5, t4), H);
  Pt r;
  r.X = fill_mul(e, g.mul_X3, E, Fl);
  r.Y = fill_mul(e, g.mul_Y3, Gl, H);
  r.T = fill_mul(e, g.mul_T3, E, H);
  r.Z = fill_mul(e, g.mul_Z3, Fl, Gl);
  return r;
}

// fill_point_double_gadget (ed25519_group_air.rs:507-546)
Pt fill_point_double(Emit& e, const PDbl& g, const Pt& p) {
  const PtL A1 = limbs_pt(p);
  uint32_t A[NL], B[NL], zz[NL], C[NL], H[NL], xy[NL], xy2[NL], E[NL], G[NL], Fl[NL];
  limbs_of(fill_mul(e, g.sq_A, A1.l[0], A1.l[0]), A);
  limbs_of(fill_mul(e, g.sq_B, A1.l[1], A1.l[1]), B);
  limbs_of(fill_mul(e, g.sq_zz, A1.l[2], A1.l[2]), zz);
  limbs_of(fill_add(e, g.add_C, zz, zz), C);
  limbs_of(fill_add(e, g.add_H, A, B), H);
  limbs_of(fill_add(e, g.add_xy, A1.l[0], A1.l[1]), xy);
  limbs_of(fill_mul(e, g.sq_xy, xy, xy), xy2);
  limbs_of(fill_sub(e, g.sub_E, H, xy2), E);
  limbs_of(fill_sub(e, g.sub_G, A, B), G);
  limbs_of(fill_add(e, g.add_F, C, G), Fl);
  Pt r;
  r.X = fill_mul(e, g.mul_X3, E, Fl);
  r.Y = fill_mul(e, g.mul_Y3, G, H);
  r.T = fill_mul(e, g.mul_T3, E, H);
  r.Z = fill_mul(e, g.mul_Z3, Fl, G);
  return r;
}

}  // namespace

namespace {
// The words of consecutive ladder rows and where each row's words start.
struct LadderChunk {
  std::vector<uint64_t> words;
  std::vector<uint32_t> start;
  std::exception_ptr err;
};
}  // namespace

void build_witness(const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg, uint64_t len, uint32_t k,
                   Witness* w) {
  require(pub && sig && (msg || len == 0), "ed25519: null argument");
  Pt R, A;
  F r_y, a_y;
  int r_sign = 0, a_sign = 0;
  require(decompress(sig, &R, &r_y, &r_sign), "ed25519: R does not decode");
  require(decompress(pub, &A, &a_y, &a_sign), "ed25519: A does not decode");
  // SHA-512(R || A || M), k = digest mod L (the hashed input of fill_verify_air_v0..v16)
  std::vector<uint8_t> sha_in(64 + len);
  memcpy(sha_in.data(), sig, 32);
  memcpy(sha_in.data() + 32, pub, 32);
  if (len) memcpy(sha_in.data() + 64, msg, len);
  Witness& W = *w;
  W.L = make_layout(sha_in.size(), k);
  const Layout& L = W.L;
  uint8_t digest[64];
  const uint64_t h_sha = sha512_witness(sha_in.data(), sha_in.size(), &W.sha, digest);
  require(h_sha == L.k_hash && W.sha.size() == L.n_blocks, "ed25519: SHA-512 trace shape");
  uint32_t dw[16], kr[8], q32[9];
  memcpy(dw, digest, 64);
  divmod_L(dw, 16, kr, q32, 9);
  uint8_t k_can[32];
  memcpy(k_can, kr, 32);
  std::vector<uint8_t> s_bits(k), k_bits(k);
  ladder_bits(sig + 32, k, s_bits.data());
  ladder_bits(k_can, k, k_bits.data());
  W.prog = make_program(L, s_bits.data(), k_bits.data(), r_y, r_sign, a_y, a_sign, A);

  // globals: the r thread (k bits) and the sB, kA and R threads (4 x 10 limbs each).
  // Their codes go into every phase's codes first (the ladder threads then record
  // their phases' other cells), their values once the ladders are done.
  const uint32_t n_lad = 2 * k;
  W.codes.assign((size_t)N_PHASES * L.width, 0);
  {
    std::vector<uint32_t> gcodes(L.width, 0);
    uint32_t gi = 0;
    for (uint32_t i = 0; i < k; ++i) gcodes[L.r_thread + i] = code(OP_GLOBAL, gi++);
    for (const uint32_t* thr : {L.thr_sB, L.thr_kA, L.thr_R})
      for (int q = 0; q < 4; ++q)
        for (int i = 0; i < NL; ++i) gcodes[thr[q] + i] = code(OP_GLOBAL, gi++);
    for (uint32_t ph = 0; ph < N_PHASES; ++ph) memcpy(&W.codes[(size_t)ph * L.width], gcodes.data(), 4 * L.width);
  }

  W.row_phase.assign(L.height, PH_IDLE);
  W.row_off.assign(L.height + 1, 0);
  W.words.clear();
  std::vector<bool> recorded(N_PHASES, false);
  uint32_t d[NL], d2[NL], one[NL], zero[NL] = {0};
  limbs_of(D(), d);
  for (int i = 0; i < NL; ++i) d2[i] = 2 * d[i];
  limbs_of(fe(1), one);
  // The 2k ladder rows (fill_scalar_mult_trace, ed25519_scalar_mult_air.rs:133-171,
  // and the v6 shift chain) in parallel chunks, each emitting its rows' words into
  // its own buffer. A row needs the accumulator entering it; this thread computes
  // them natively (padd and pdbl follow the gadgets' formulas, so the points are the
  // ones the rows compute) and publishes them step by step in acc_ready, so the
  // chunks start at once instead of after the whole pass (about 1 us a step against
  // some 20 us for a row's gadgets).
  require(L.kA_first == L.sB_first + k && L.kA_last == L.kA_first + k - 1, "ed25519: ladder rows");
  std::vector<Pt> acc_in(n_lad);
  std::atomic<uint32_t> acc_ready{0};  // steps j done: acc_in[j] and acc_in[k + j] are set
  // the host's threads shared among the witnesses being built at once (server workers
  // build theirs concurrently)
  static std::atomic<uint32_t> g_building{0};
  struct Building {
    uint32_t n;
    Building() : n(g_building.fetch_add(1) + 1) {}
    ~Building() { g_building.fetch_sub(1); }
  } building;
  const uint32_t hw = std::max(1u, std::thread::hardware_concurrency());
  const uint32_t n_thr = std::max(1u, std::min({16u, hw / building.n, n_lad / 16}));
  const uint32_t per_chunk = (n_lad + n_thr - 1) / n_thr;
  std::vector<LadderChunk> chunks((n_lad + per_chunk - 1) / per_chunk);
  auto run_chunk = [&](uint32_t ci) {
    LadderChunk& ch = chunks[ci];
    try {
      const uint32_t g0 = ci * per_chunk, g1 = std::min(n_lad, g0 + per_chunk);
      ch.words.reserve((size_t)(g1 - g0) * (k + 1024));
      for (uint32_t g = g0; g < g1; ++g) {
        const bool sb = g < k;
        const uint32_t j = sb ? g : g - k;
        while (acc_ready.load(std::memory_order_acquire) <= j) std::this_thread::yield();
        const uint32_t ph = sb ? PH_SB : PH_KA;
        ch.start.push_back((uint32_t)ch.words.size());
        Emit e{ch.words, j == 0 ? &W.codes[(size_t)ph * L.width] : nullptr};
        const Pt& base = sb ? basepoint() : A;
        const uint8_t* bits = sb ? s_bits.data() : k_bits.data();
        const Pt& acc = acc_in[g];
        const PtL bl = limbs_pt(base), al = limbs_pt(acc);
        for (int q = 0; q < 4; ++q) e.limbs(L.base[q], bl.l[q]);
        for (int q = 0; q < 4; ++q) e.limbs(L.acc[q], al.l[q]);
        const Pt dbl = fill_point_double(e, L.mdbl, acc);
        const Pt tmp = fill_point_add(e, L.cadd.add, dbl, base, d2);
        const PtL dl = limbs_pt(dbl), tl = limbs_pt(tmp);
        for (int q = 0; q < 4; ++q) fill_sel(e, L.cadd.sel[q], dl.l[q], tl.l[q], bits[j]);
        const uint32_t blk = sb ? L.sblock_sB : L.sblock_kA;
        for (uint32_t i = 0; i < k; ++i) e.value(blk + i, j + i < k ? bits[j + i] : 0);
      }
      ch.start.push_back((uint32_t)ch.words.size());
    } catch (...) {
      ch.err = std::current_exception();
    }
  };
  Pt sB = identity(), kA = identity();
  {
    std::vector<std::thread> th;
    try {
      for (uint32_t ci = 0; ci < chunks.size(); ++ci) th.emplace_back(run_chunk, ci);
      for (uint32_t j = 0; j < k; ++j) {
        acc_in[j] = sB;
        acc_in[k + j] = kA;
        acc_ready.store(j + 1, std::memory_order_release);
        sB = pdbl(sB);
        if (s_bits[j]) sB = padd(sB, basepoint());
        kA = pdbl(kA);
        if (k_bits[j]) kA = padd(kA, A);
      }
    } catch (...) {
      acc_ready.store(k, std::memory_order_release);  // no thread may wait for ever
      for (auto& t : th) t.join();
      throw;
    }
    for (auto& t : th) t.join();
    for (const LadderChunk& ch : chunks)
      if (ch.err) std::rethrow_exception(ch.err);
  }
  const Pt Rt{R.X, R.Y, fe(1), mul(R.X, R.Y)};
  const Pt res1 = padd(sB, pneg(Rt)), res2 = padd(res1, pneg(kA));
  W.globals.clear();
  for (uint32_t i = 0; i < k; ++i) W.globals.push_back(k_bits[i]);
  const Pt* const thread_pts[3] = {&sB, &kA, &Rt};
  for (const Pt* pt : thread_pts) {
    const PtL p = limbs_pt(*pt);
    for (int q = 0; q < 4; ++q)
      for (int i = 0; i < NL; ++i) W.globals.push_back(p.l[q][i]);
  }
  recorded[PH_SB] = recorded[PH_KA] = true;
  {
    size_t lad_words = 0;
    for (const LadderChunk& ch : chunks) lad_words += ch.words.size();
    W.words.reserve(lad_words + 65536);
  }
  for (uint32_t row = 0; row < L.height; ++row) {
    W.row_off[row] = (uint32_t)W.words.size();
    uint32_t ph = PH_IDLE;
    if (row + 1 < L.k_hash) ph = PH_SHA;
    else if (row + 1 == L.k_hash) ph = PH_DIGEST;
    else if (row == L.reduce_row) ph = PH_REDUCE;
    else if (row == L.decomp_R_row) ph = PH_DECOMP_R;
    else if (row == L.decomp_A_row) ph = PH_DECOMP_A;
    else if (row >= L.sB_first && row <= L.sB_last) ph = PH_SB;
    else if (row >= L.kA_first && row <= L.kA_last) ph = PH_KA;
    else if (row == L.residual_row) ph = PH_RESIDUAL;
    else if (row >= L.dbl_row[0] && row <= L.dbl_row[2]) ph = PH_DBL;
    else if (row == L.result_row) ph = PH_RESULT;
    W.row_phase[row] = (uint8_t)ph;
    Emit e{W.words, recorded[ph] ? nullptr : &W.codes[(size_t)ph * L.width]};
    recorded[ph] = true;
    switch (ph) {
      case PH_DIGEST:  // v1: the digest's bits, LSB first within each big-endian word
        for (int kk = 0; kk < 8; ++kk) {
          uint64_t hw = 0;
          for (int j = 0; j < 8; ++j) hw = hw << 8 | digest[8 * kk + j];
          const uint32_t wi = e.word(hw);
          for (uint32_t i = 0; i < 64; ++i) e.set(L.digest_bits + 64 * kk + i, code(OP_BIT, wi, i));
        }
        break;
      case PH_REDUCE: {  // v0 input limbs and fill_scalar_reduce_gadget (ed25519_scalar_air.rs:168-372)
        uint32_t in[RED_IN], q[RED_Q], r[RED_R], sl[RED_R], l16[RED_R];
        for (uint32_t i = 0; i < RED_IN; ++i) in[i] = digest[2 * i] | (uint32_t)digest[2 * i + 1] << 8;
        for (uint32_t i = 0; i < RED_Q; ++i) q[i] = (q32[i / 2] >> (16 * (i % 2))) & 0xFFFF;
        for (uint32_t i = 0; i < RED_R; ++i) r[i] = (kr[i / 2] >> (16 * (i % 2))) & 0xFFFF;
        for (uint32_t i = 0; i < RED_R; ++i) l16[i] = (L32[i / 2] >> (16 * (i % 2))) & 0xFFFF;
        {  // slack = L - 1 - r
          int32_t br = 0;
          for (uint32_t i = 0; i < RED_R; ++i) {
            int32_t v = (int32_t)l16[i] - (i == 0 ? 1 : 0) - (int32_t)r[i] - br;
            br = v < 0;
            sl[i] = (uint32_t)(v + (br ? 65536 : 0));
          }
          require(br == 0, "ed25519 witness: r >= L");
        }
        for (uint32_t i = 0; i < RED_IN; ++i) e.value(L.red.input + i, in[i]);
        auto bits16 = [&](uint32_t limbs, uint32_t bits, const uint32_t* v, uint32_t n) {
          for (uint32_t i = 0; i < n; ++i) {
            const uint32_t wi = e.word(v[i]);
            e.set(limbs + i, code(OP_WORD, wi));
            for (uint32_t b = 0; b < RED_LB; ++b) e.set(bits + i * RED_LB + b, code(OP_BIT, wi, b));
          }
        };
        bits16(L.red.q, L.red.q_bits, q, RED_Q);
        bits16(L.red.r, L.red.r_bits, r, RED_R);
        bits16(L.red.slack, L.red.slack_bits, sl, RED_R);
        int64_t prev = 0;
        for (uint32_t kk = 0; kk < RED_PROD; ++kk) {
          int64_t prod = 0;
          for (uint32_t i = 0; i < RED_Q; ++i)
            if (kk >= i && kk - i < RED_R) prod += (int64_t)q[i] * l16[kk - i];
          const int64_t resid = (kk < RED_IN ? (int64_t)in[kk] : 0) - prod - (kk < RED_R ? (int64_t)r[kk] : 0);
          const int64_t tot = resid + prev;
          require((tot & 0xFFFF) == 0, "ed25519 witness: reduction chain");
          const int64_t cy = tot >> RED_LB;
          const uint32_t wi = e.word((uint64_t)(cy + (1ll << (RED_CB - 1))));
          for (uint32_t b = 0; b < RED_CB; ++b) e.set(L.red.carry_bits + kk * RED_CB + b, code(OP_BIT, wi, b));
          prev = cy;
        }
        require(prev == 0, "ed25519 witness: reduction chain end");
        break;
      }
      case PH_DECOMP_R:
      case PH_DECOMP_A: {  // v2 and fill_point_decompress_gadget (ed25519_group_air.rs:957-1029)
        const Pt& pt = ph == PH_DECOMP_R ? R : A;
        const F& y = ph == PH_DECOMP_R ? r_y : a_y;
        const int sign = ph == PH_DECOMP_R ? r_sign : a_sign;
        const Decomp& g = L.decomp;
        uint32_t yl[NL], xl[NL];
        limbs_of(y, yl);
        limbs_of(pt.X, xl);
        e.limbs(g.y, yl);
        e.value(g.sign, (uint64_t)sign);
        e.limbs(g.d, d);
        e.limbs(g.one, one);
        e.elem(g.x, g.x_bits, xl);
        uint32_t x2[NL], y2[NL], dx2[NL], dxy[NL], y2m1[NL], lhs[NL];
        limbs_of(fill_mul(e, g.sq_x, xl, xl), x2);
        limbs_of(fill_mul(e, g.sq_y, yl, yl), y2);
        limbs_of(fill_mul(e, g.mul_dx2, d, x2), dx2);
        limbs_of(fill_mul(e, g.mul_dxy, dx2, y2), dxy);
        limbs_of(fill_sub(e, g.sub_y2m1, y2, one), y2m1);
        limbs_of(fill_sub(e, g.sub_lhs, y2m1, x2), lhs);
        fill_sub(e, g.sub_eq, lhs, dxy);
        if (ph == PH_DECOMP_R) {  // v13: the one constant and T = X Y
          e.limbs(L.one_R, one);
          uint32_t rx[NL], ry[NL];
          limbs_of(Rt.X, rx);
          limbs_of(Rt.Y, ry);
          fill_mul(e, L.mul_RT, rx, ry);
        }
        break;
      }
      case PH_SB:
      case PH_KA: {  // filled by the ladder chunks: copy this row's words
        const uint32_t g = row - L.sB_first;  // sB rows, then kA rows, contiguous
        const LadderChunk& ch = chunks[g / per_chunk];
        const uint32_t r = g % per_chunk;
        W.words.insert(W.words.end(), ch.words.begin() + ch.start[r], ch.words.begin() + ch.start[r + 1]);
        break;
      }
      case PH_RESIDUAL: {  // v14, v15
        const PtL rl = limbs_pt(Rt), kl = limbs_pt(kA);
        fill_sub(e, L.sub_negR_X, zero, rl.l[0]);
        fill_sub(e, L.sub_negR_T, zero, rl.l[3]);
        fill_point_add(e, L.pa_R1, sB, pneg(Rt), d2);
        fill_sub(e, L.sub_negkA_X, zero, kl.l[0]);
        fill_sub(e, L.sub_negkA_T, zero, kl.l[3]);
        fill_point_add(e, L.pa_R2, res1, pneg(kA), d2);
        break;
      }
      case PH_DBL: {  // the cofactor doublings of residual_2 (v9/v10 cells at the v14 rows)
        Pt p = res2;
        for (uint32_t i = L.dbl_row[0]; i < row; ++i) p = pdbl(p);
        const PtL pl = limbs_pt(p);
        for (int q = 0; q < 3; ++q) e.limbs(L.dbl_in[q], pl.l[q]);
        fill_point_double(e, L.dbl, p);
        break;
      }
      case PH_RESULT: {  // [8] residual_2 and the three SUB canonicalisations
        const Pt p8 = pdbl(pdbl(pdbl(res2)));
        const PtL pl = limbs_pt(p8);
        for (int q = 0; q < 4; ++q) e.limbs(L.result[q], pl.l[q]);
        fill_sub(e, L.sub_X, pl.l[0], zero);
        fill_sub(e, L.sub_T, pl.l[3], zero);
        fill_sub(e, L.sub_YZ, pl.l[1], pl.l[2]);
        break;
      }
      default:
        break;
    }
  }
  W.row_off[L.height] = (uint32_t)W.words.size();
  // every row of a phase reads its cells through the same codes: same word count
  std::vector<int64_t> per_phase(N_PHASES, -1);
  for (uint32_t row = 0; row < L.height; ++row) {
    const int64_t nw = (int64_t)W.row_off[row + 1] - W.row_off[row];
    int64_t& want = per_phase[W.row_phase[row]];
    if (want < 0) want = nw;
    require(nw == want && nw < (1 << 23), "ed25519 witness: rows of a phase differ in word count");
  }
}

void expand_host(const Witness& w, uint64_t* trace) {
  const Layout& L = w.L;
  const uint64_t H = L.height;
  auto cols = [&](uint32_t c0, uint32_t c1) {
    for (uint32_t c = c0; c < c1; ++c)
      for (uint64_t r = 0; r < H; ++r) {
        const uint32_t cd = w.codes[(size_t)w.row_phase[r] * L.width + c];
        trace[c * H + r] = cell_value(cd, w.words.data() + w.row_off[r], w.globals.data());
      }
  };
  const uint32_t nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<std::thread> th;
  const uint32_t chunk = (L.width + nt - 1) / nt;
  for (uint32_t t = 0; t < nt; ++t)
    th.emplace_back(cols, std::min(L.width, t * chunk), std::min(L.width, (t + 1) * chunk));
  for (auto& x : th) x.join();
  // the SHA-512 rows (columns below 1510, rows below k_hash) from the block witnesses
  std::vector<uint64_t> sha((size_t)SHA_W * L.k_hash);
  sha512_fill_host(w.sha.data(), L.n_blocks, L.k_hash, sha.data());
  for (uint32_t c = 0; c < SHA_W; ++c) memcpy(trace + c * H, sha.data() + (size_t)c * L.k_hash, 8 * L.k_hash);
}

namespace {

// The cells a block reads at this row (cur) and at the next row (nxt).
template <class Cur, class Nxt>
void block_cells(const Block& b, const Program& P, Cur cur, Nxt nxt) {
  auto span = [&](uint32_t base, uint32_t n) {
    for (uint32_t i = 0; i < n; ++i) cur(base + i);
  };
  const uint32_t* p = b.p;
  switch (b.kind) {
    case B_SHA512:
      for (uint32_t c = 0; c < SHA_W; ++c) cur(c), nxt(c);
      break;
    case B_REDUCE:
      span(p[0], RED_IN), span(p[1], RED_Q), span(p[2], RED_Q * RED_LB), span(p[3], RED_R);
      span(p[4], RED_R * RED_LB), span(p[5], RED_R), span(p[6], RED_R * RED_LB), span(p[7], RED_PROD * RED_CB);
      break;
    case B_FORMAT:
      span(p[0], 512), span(p[2], 16);
      for (uint32_t i = 0; i < RED_IN; ++i) nxt(p[1] + i);
      break;
    case B_MUL: span(p[0], NL), span(p[1], NL), span(p[2], NL), span(p[3], 255), span(p[4], MUL_CB * NL); break;
    case B_ADD: span(p[0], NL), span(p[1], NL), span(p[2], NL), span(p[3], 255), span(p[4], NL); break;
    case B_SUB: span(p[0], NL), span(p[1], NL), span(p[2], NL), span(p[3], 255), span(p[4], NL), span(p[5], NL); break;
    case B_SEL: span(p[0], NL), span(p[1], NL), cur(p[2]), span(p[3], NL); break;
    case B_RANGE: span(p[0], NL), span(p[1], 255); break;
    case B_SIGN: cur(p[0]), cur(p[1]); break;
    default:
      for (uint32_t i = 0; i < p[1]; ++i)
        for (int h = 0; h < 2; ++h) {
          const uint64_t r = P.pairs[2 * (p[0] + i) + h], src = r >> 62;
          if (src == SRC_CUR) cur((uint32_t)(r & 0xFFFFFFFFu));
          if (src == SRC_NXT) nxt((uint32_t)(r & 0xFFFFFFFFu));
        }
  }
}

}  // namespace

LdePlan make_lde_plan(const Witness& w) {
  const Layout& L = w.L;
  const uint32_t W = L.width, H = L.height, D = L.r_thread, K = LdePlan::kSparseRows;
  LdePlan plan;
  plan.dense = D;
  // row sets of the columns at and above D, capped: more than K rows marks a column wide
  std::vector<std::vector<uint32_t>> nz(W - D), rd(W - D);
  std::vector<char> nz_wide(W - D, 0), rd_wide(W - D, 0);
  auto add = [&](std::vector<uint32_t>& set, char& wide, uint32_t row) {
    if (wide) return;
    if (std::find(set.begin(), set.end(), row) != set.end()) return;
    if (set.size() == K) {
      wide = 1;
      return;
    }
    set.push_back(row);
  };
  std::vector<std::vector<uint32_t>> phase_rows(N_PHASES);
  for (uint32_t r = 0; r < H; ++r) phase_rows[w.row_phase[r]].push_back(r);
  // constant columns: the same global word in every phase that has rows
  std::vector<char> is_const(W - D, 1);
  for (uint32_t c = D; c < W; ++c) {
    uint32_t code0 = ~0u;
    for (uint32_t ph = 0; ph < N_PHASES; ++ph) {
      if (phase_rows[ph].empty()) continue;
      const uint32_t cd = w.codes[(size_t)ph * W + c];
      if (code0 == ~0u) code0 = cd;
      if (cd != code0 || (cd >> 29) != OP_GLOBAL) is_const[c - D] = 0;
      if (cd != 0)
        for (uint32_t r : phase_rows[ph]) add(nz[c - D], nz_wide[c - D], r);
    }
  }
  for (const Block& b : w.prog.blocks) {
    std::vector<uint32_t> rows;
    for (uint32_t r = 0; r < H; ++r)
      if (gate_open(b, r)) rows.push_back(r);
    if (rows.empty()) continue;
    block_cells(
        b, w.prog,
        [&](uint32_t c) {
          if (c >= D)
            for (uint32_t r : rows) add(rd[c - D], rd_wide[c - D], r);
        },
        [&](uint32_t c) {
          if (c >= D)
            for (uint32_t r : rows) add(rd[c - D], rd_wide[c - D], (r + 1) % H);
        });
  }
  std::map<std::pair<std::vector<uint32_t>, std::vector<uint32_t>>, size_t> gid;
  for (uint32_t c = D; c < W; ++c) {
    const uint32_t i = c - D;
    if (is_const[i]) {
      plan.const_cols.push_back(c);
      continue;
    }
    if (nz_wide[i] || rd_wide[i]) return LdePlan{};  // a column outside the plan: full LDE
    std::sort(nz[i].begin(), nz[i].end());
    std::sort(rd[i].begin(), rd[i].end());
    auto key = std::make_pair(nz[i], rd[i]);
    auto it = gid.find(key);
    if (it == gid.end()) {
      it = gid.emplace(key, plan.groups.size()).first;
      plan.groups.push_back(LdePlan::Group{nz[i], rd[i], {}});
    }
    plan.groups[it->second].cols.push_back(c);
  }
  plan.ok = true;
  return plan;
}

bool verify(const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg, uint64_t len) {
  Pt R, A;
  if (!decompress(sig, &R, nullptr, nullptr) || !decompress(pub, &A, nullptr, nullptr)) return false;
  if (!scalar_canonical(sig + 32)) return false;
  std::vector<uint8_t> in(64 + len);
  memcpy(in.data(), sig, 32);
  memcpy(in.data() + 32, pub, 32);
  if (len) memcpy(in.data() + 64, msg, len);
  std::vector<sha512::BlockWitness> wit;
  uint8_t digest[64];
  sha512_witness(in.data(), in.size(), &wit, digest);
  uint32_t dw[16], kr[8];
  memcpy(dw, digest, 64);
  divmod_L(dw, 16, kr, nullptr, 0);
  uint8_t sb[256], kb[256];
  ladder_bits(sig + 32, 256, sb);
  ladder_bits((const uint8_t*)kr, 256, kb);
  Pt res = padd(padd(ladder(basepoint(), sb, 256), pneg(R)), pneg(ladder(A, kb, 256)));
  res = pdbl(pdbl(pdbl(res)));
  return is_identity(res);
}

void pi_hash(const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg, uint64_t len,
             const uint8_t fs_binding[32], const uint8_t merkle_root[32], const uint8_t root_f0[32], uint8_t out[32]) {
  kc::Sha3 h;
  h.update("ZSK-KSK-PIHASH-V2-ST", 20);
  h.update(pub, 32);
  h.update(sig, 64);
  uint8_t ln[8];
  for (int i = 0; i < 8; ++i) ln[i] = (uint8_t)(len >> (8 * i));
  h.update(ln, 8);
  if (len) h.update(msg, len);
  h.update(fs_binding, 32);
  h.update(merkle_root, 32);
  h.update(root_f0, 32);
  h.finalize(out);
}

}  // namespace ed25519
}  // namespace sg

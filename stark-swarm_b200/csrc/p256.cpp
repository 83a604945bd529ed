// p256.cpp — host side of the P-256 ECDSA double-chain AIR: the row layout as a
// gadget program, the chains' witnesses from exact arithmetic modulo p, the
// u1/u2 scalars modulo n, and the pi_hash recipe.
//
// Every value the gadgets pass on is canonical (below p): a mul gadget outputs
// a b mod p, an add or sub gadget is always followed by a freeze. So the trace
// is a function of canonical integers; the gadgets' limb chains (carries,
// borrows, quotient) are replayed here exactly as the reference's fill
// functions compute them (p256_field_air.rs:344-398, 570-610, 953-1040,
// 1229-1241, 1374-1447).
#include "p256.hpp"

#include <cstring>
#include <exception>
#include <mutex>
#include <thread>

#include "bigint.hpp"
#include "context.hpp"
#include "keccak.cuh"
#include "p256_cells.cuh"

namespace sg {
namespace p256 {

const uint8_t GX[32] = {0x6b, 0x17, 0xd1, 0xf2, 0xe1, 0x2c, 0x42, 0x47, 0xf8, 0xbc, 0xe6, 0xe5, 0x63, 0xa4, 0x40, 0xf2,
                        0x77, 0x03, 0x7d, 0x81, 0x2d, 0xeb, 0x33, 0xa0, 0xf4, 0xa1, 0x39, 0x45, 0xd8, 0x98, 0xc2, 0x96};
const uint8_t GY[32] = {0x4f, 0xe3, 0x42, 0xe2, 0xfe, 0x1a, 0x7f, 0x9b, 0x8e, 0xe7, 0xeb, 0x4a, 0x7c, 0x0f, 0x9e, 0x16,
                        0x2b, 0xce, 0x33, 0x57, 0x6b, 0x31, 0x5e, 0xce, 0xcb, 0xb6, 0x40, 0x68, 0x37, 0xbf, 0x51, 0xf5};

namespace {

// 288-bit values (9 words): canonical elements use 8, sums below 2p need the 9th.
struct U {
  uint32_t w[9];
};
// p = 2^256 - 2^224 + 2^192 + 2^96 - 1, n = the group order, b = the curve's b
const U kP = {{0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0x00000000, 0x00000000, 0x00000000, 0x00000001, 0xFFFFFFFF, 0}};
const U kN = {{0xFC632551, 0xF3B9CAC2, 0xA7179E84, 0xBCE6FAAD, 0xFFFFFFFF, 0xFFFFFFFF, 0x00000000, 0xFFFFFFFF, 0}};
const U kB = {{0x27D2604B, 0x3BCE3C3E, 0xCC53B0F6, 0x651D06B0, 0x769886BC, 0xB3EBBD55, 0xAA3A93E7, 0x5AC635D8, 0}};

U from_be(const uint8_t b[32]) {
  U u{};
  for (int i = 0; i < 8; ++i) {
    const uint8_t* p = b + 32 - 4 * (i + 1);
    u.w[i] = (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3];
  }
  return u;
}
bool lt(const U& a, const U& b) { return bn::cmp(a.w, b.w, 9) < 0; }
U add9(const U& a, const U& b) {
  U r{};
  uint64_t c = 0;
  for (int i = 0; i < 9; ++i) {
    const uint64_t s = (uint64_t)a.w[i] + b.w[i] + c;
    r.w[i] = (uint32_t)s;
    c = s >> 32;
  }
  return r;
}
U sub9(const U& a, const U& b) {  // a >= b
  U r{};
  int64_t br = 0;
  for (int i = 0; i < 9; ++i) {
    const int64_t d = (int64_t)a.w[i] - b.w[i] + br;
    r.w[i] = (uint32_t)d;
    br = d >> 32;
  }
  return r;
}
// a * b = q m + r for a, b below 2^256 and the modulus m (8 significant words)
void muldiv(const U& a, const U& b, const U& m, U* q, U* r) {
  uint32_t prod[16], qw[16] = {0}, rw[8] = {0};
  bn::mul(a.w, 8, b.w, 8, prod);
  bn::divmod(prod, 16, m.w, 8, qw, rw);
  if (q) {
    *q = U{};
    memcpy(q->w, qw, 36);
  }
  *r = U{};
  memcpy(r->w, rw, 32);
}
U mulmod(const U& a, const U& b, const U& m) {
  U r;
  muldiv(a, b, m, nullptr, &r);
  return r;
}
void limbs(const U& u, uint32_t out[NL]) {  // 26-bit limbs of a value below 2^260
  for (uint32_t i = 0; i < NL; ++i) {
    const uint32_t bit = i * LB, wi = bit / 32, sh = bit % 32;
    uint64_t x = u.w[wi];
    if (wi + 1 < 9) x |= (uint64_t)u.w[wi + 1] << 32;
    out[i] = (uint32_t)(x >> sh) & ((1u << LB) - 1);
  }
}
U from_limbs(const uint32_t l[NL]) {
  U u{};
  for (uint32_t i = 0; i < NL; ++i) {
    const uint32_t bit = i * LB, wi = bit / 32, sh = bit % 32;
    const uint64_t x = (uint64_t)l[i] << sh;
    u.w[wi] |= (uint32_t)x;
    if (wi + 1 < 9) u.w[wi + 1] |= (uint32_t)(x >> 32);
  }
  return u;
}

// ---------------------------------------------------------------- layout as a program
struct Op {
  uint8_t type;  // 0 mul, 1 add + freeze, 2 sub + freeze
  uint32_t g, fz;
};
struct GroupBuild {
  uint32_t cursor, b_base;
  std::vector<Gadget> muls, adds, subs, fz_adds, fz_subs;
  std::vector<Op> prog;  // indices into the lists above until `place` rebases them
  uint32_t result[3];
  explicit GroupBuild(uint32_t c) : cursor(c), b_base(c) { cursor += ELEM; }
  uint32_t take(uint32_t n) {
    const uint32_t b = cursor;
    cursor += n;
    return b;
  }
  Gadget freeze(uint32_t a) {
    const uint32_t d = take(FREEZE_OWNED);
    return Gadget{G_FREEZE, {a, d, d + NL, d + ELEM, d + ELEM + NL, d + 2 * ELEM, d + 2 * ELEM + NL}};
  }
  uint32_t mul(uint32_t a, uint32_t b) {
    const uint32_t c = take(MUL_OWNED);
    muls.push_back(Gadget{G_MUL, {a, b, c, c + NL, c + ELEM, c + ELEM + NL, c + 2 * ELEM}});
    prog.push_back(Op{0, (uint32_t)muls.size() - 1, 0});
    return c;
  }
  uint32_t addf(uint32_t a, uint32_t b) {
    const uint32_t c = take(ADD_OWNED);
    adds.push_back(Gadget{G_ADD, {a, b, c, c + NL, c + ELEM, 0, 0}});
    fz_adds.push_back(freeze(c));
    prog.push_back(Op{1, (uint32_t)adds.size() - 1, (uint32_t)fz_adds.size() - 1});
    return fz_adds.back().p[3];
  }
  uint32_t subf(uint32_t a, uint32_t b) {
    const uint32_t c = take(SUB_OWNED);
    subs.push_back(Gadget{G_SUB, {a, b, c, c + NL, c + ELEM, c + ELEM + NL, 0}});
    fz_subs.push_back(freeze(c));
    prog.push_back(Op{2, (uint32_t)subs.size() - 1, (uint32_t)fz_subs.size() - 1});
    return fz_subs.back().p[3];
  }
  // append in emission order to the table and rebase the program's indices
  void place(std::vector<Gadget>* t, std::vector<Op>* out) {
    const uint32_t m0 = (uint32_t)t->size(), a0 = m0 + (uint32_t)muls.size(), s0 = a0 + (uint32_t)adds.size(),
                   fa0 = s0 + (uint32_t)subs.size(), fs0 = fa0 + (uint32_t)fz_adds.size();
    for (auto* v : {&muls, &adds, &subs, &fz_adds, &fz_subs}) t->insert(t->end(), v->begin(), v->end());
    for (Op o : prog) {
      if (o.type == 0) o.g += m0;
      if (o.type == 1) o.g += a0, o.fz += fa0;
      if (o.type == 2) o.g += s0, o.fz += fs0;
      out->push_back(o);
    }
  }
};

// p256_group_air.rs:302-447 build_group_double_layout
GroupBuild group_double(uint32_t cursor, uint32_t x, uint32_t y, uint32_t z) {
  GroupBuild g(cursor);
  const uint32_t b = g.b_base;
  uint32_t t0 = g.mul(x, x), t1 = g.mul(y, y), t2 = g.mul(z, z), t3 = g.mul(x, y);
  t3 = g.addf(t3, t3);
  uint32_t z3 = g.mul(x, z);
  z3 = g.addf(z3, z3);
  uint32_t y3 = g.mul(b, t2);
  y3 = g.subf(y3, z3);
  uint32_t x3 = g.addf(y3, y3);
  y3 = g.addf(x3, y3);
  x3 = g.subf(t1, y3);
  y3 = g.addf(t1, y3);
  y3 = g.mul(x3, y3);
  x3 = g.mul(x3, t3);
  t3 = g.addf(t2, t2);
  t2 = g.addf(t2, t3);
  z3 = g.mul(b, z3);
  z3 = g.subf(z3, t2);
  z3 = g.subf(z3, t0);
  t3 = g.addf(z3, z3);
  z3 = g.addf(z3, t3);
  t3 = g.addf(t0, t0);
  t0 = g.addf(t3, t0);
  t0 = g.subf(t0, t2);
  t0 = g.mul(t0, z3);
  g.result[1] = g.addf(y3, t0);
  t0 = g.mul(y, z);
  t0 = g.addf(t0, t0);
  z3 = g.mul(t0, z3);
  g.result[0] = g.subf(x3, z3);
  z3 = g.mul(t0, t1);
  z3 = g.addf(z3, z3);
  g.result[2] = g.addf(z3, z3);
  return g;
}

// p256_group_air.rs:705-869 build_group_add_layout
GroupBuild group_add(uint32_t cursor, uint32_t px, uint32_t py, uint32_t pz, uint32_t qx, uint32_t qy, uint32_t qz) {
  GroupBuild g(cursor);
  const uint32_t b = g.b_base;
  uint32_t t0 = g.mul(px, qx), t1 = g.mul(py, qy), t2 = g.mul(pz, qz);
  uint32_t t3 = g.addf(px, py), t4 = g.addf(qx, qy);
  t3 = g.mul(t3, t4);
  t4 = g.addf(t0, t1);
  t3 = g.subf(t3, t4);
  t4 = g.addf(py, pz);
  uint32_t x3 = g.addf(qy, qz);
  t4 = g.mul(t4, x3);
  x3 = g.addf(t1, t2);
  t4 = g.subf(t4, x3);
  x3 = g.addf(px, pz);
  uint32_t y3 = g.addf(qx, qz);
  x3 = g.mul(x3, y3);
  y3 = g.addf(t0, t2);
  y3 = g.subf(x3, y3);
  uint32_t z3 = g.mul(b, t2);
  x3 = g.subf(y3, z3);
  z3 = g.addf(x3, x3);
  x3 = g.addf(x3, z3);
  z3 = g.subf(t1, x3);
  x3 = g.addf(t1, x3);
  y3 = g.mul(b, y3);
  t1 = g.addf(t2, t2);
  t2 = g.addf(t1, t2);
  y3 = g.subf(y3, t2);
  y3 = g.subf(y3, t0);
  t1 = g.addf(y3, y3);
  y3 = g.addf(t1, y3);
  t1 = g.addf(t0, t0);
  t0 = g.addf(t1, t0);
  t0 = g.subf(t0, t2);
  t1 = g.mul(t4, y3);
  t2 = g.mul(t0, y3);
  y3 = g.mul(x3, z3);
  g.result[1] = g.addf(y3, t2);
  x3 = g.mul(t3, x3);
  g.result[0] = g.subf(x3, t1);
  z3 = g.mul(t4, z3);
  t1 = g.mul(t3, t0);
  g.result[2] = g.addf(z3, t1);
  return g;
}

struct Chain {
  uint32_t acc[3], base[3], bit, b_double, b_add, sel_g[3], out[3];
  std::vector<Op> prog_double, prog_add;
};
struct Built {
  Layout L;
  Chain ch[2];
};

Built build() {
  Built B;
  Layout& L = B.L;
  uint32_t cur = 0;
  for (int c = 0; c < 2; ++c) {
    Chain& C = B.ch[c];
    for (int k = 0; k < 3; ++k) {
      C.acc[k] = cur + NL * k;
      C.base[k] = cur + NL * (3 + k);
    }
    C.bit = cur + 6 * NL;
    cur = C.bit + 1;
    // p256_scalar_mul_air.rs:74-160: double, add of the base, three selects
    GroupBuild d = group_double(cur, C.acc[0], C.acc[1], C.acc[2]);
    GroupBuild a = group_add(d.cursor, d.result[0], d.result[1], d.result[2], C.base[0], C.base[1], C.base[2]);
    C.b_double = d.b_base;
    C.b_add = a.b_base;
    d.place(&L.table, &C.prog_double);
    a.place(&L.table, &C.prog_add);
    cur = a.cursor;
    for (int k = 0; k < 3; ++k) {
      C.sel_g[k] = (uint32_t)L.table.size();
      L.table.push_back(Gadget{G_SELECT, {a.result[k], d.result[k], cur, cur + NL, C.bit, 0, 0}});
      C.out[k] = cur;
      cur += ELEM;
    }
  }
  for (int k = 0; k < 6; ++k) L.tail[12 + k] = cur + NL * k;
  L.width = cur + 6 * NL;
  for (int c = 0; c < 2; ++c)
    for (int k = 0; k < 3; ++k) {
      L.tail[6 * c + k] = B.ch[c].acc[k];
      L.tail[6 * c + 3 + k] = B.ch[c].out[k];
    }
  uint32_t k = 0;
  for (const Gadget& g : L.table) {
    L.lam_base.push_back(k);
    k += gadget_constraints(g.kind);
  }
  L.n_constraints = k + TAIL_CONSTRAINTS;
  // every cell's owner
  L.cell_code.assign(L.width, 0xFFFFFFFFu);
  for (uint32_t gi = 0; gi < L.table.size(); ++gi) {
    const Gadget& g = L.table[gi];
    const uint32_t s = owned_start(g), n = owned_len(g.kind);
    for (uint32_t o = 0; o < n; ++o) L.cell_code[s + o] = gi << 11 | o;
  }
  for (int c = 0; c < 2; ++c) {
    const Chain& C = B.ch[c];
    for (int x = 0; x < 3; ++x)
      for (uint32_t i = 0; i < NL; ++i) {
        L.cell_code[C.acc[x] + i] = C_ACC << 28 | (uint32_t)(3 * c + x) << 4 | i;
        L.cell_code[C.base[x] + i] = C_BASE << 28 | (uint32_t)(3 * c + x) << 4 | i;
      }
    L.cell_code[C.bit] = C_BIT << 28 | (uint32_t)c;
    for (uint32_t o = 0; o < ELEM; ++o) L.cell_code[C.b_double + o] = L.cell_code[C.b_add + o] = C_B << 28 | o;
  }
  for (uint32_t r = 0; r < 6; ++r)
    for (uint32_t i = 0; i < NL; ++i) L.cell_code[L.tail[12 + r] + i] = C_RPROJ << 28 | r << 4 | i;
  for (uint32_t c : L.cell_code)
    if (c == 0xFFFFFFFFu) throw SgError{SG_EINVAL, "p256: layout leaves a cell without owner"};
  limbs(kB, L.b_limbs);
  return B;
}

const Built& built() {
  static Built b = build();
  return b;
}

// ---------------------------------------------------------------- gadget fills
U fill_mul(const U& a, const U& b, GadgetW* w) {
  U q, c;
  muldiv(a, b, kP, &q, &c);
  uint32_t al[NL], bl[NL];
  limbs(a, al);
  limbs(b, bl);
  limbs(c, w->l0);
  limbs(q, w->l1);
  int64_t prev = 0;
  for (uint32_t k = 0; k < MUL_SP; ++k) {
    int64_t pab = 0, pqp = 0;
    const uint32_t lo = k >= NL - 1 ? k - (NL - 1) : 0, hi = k < NL - 1 ? k : NL - 1;
    for (uint32_t i = lo; i <= hi; ++i) {
      pab += (int64_t)al[i] * bl[k - i];
      pqp += (int64_t)w->l1[i] * (int64_t)P_TIGHT[k - i];
    }
    const int64_t lhs = pab - pqp - (k < NL ? (int64_t)w->l0[k] : 0) + prev;
    if (k + 1 < MUL_SP) {
      if (lhs % (1ll << LB) != 0) throw SgError{SG_EINVAL, "p256: mul carry chain residual"};
      prev = lhs >> LB;
      if (prev <= -(1ll << (MUL_CB - 1)) || prev >= (1ll << (MUL_CB - 1)))
        throw SgError{SG_EINVAL, "p256: mul carry out of the biased range"};
      w->cy[k] = prev;
    } else if (lhs != 0) {
      throw SgError{SG_EINVAL, "p256: mul carry chain does not close"};
    }
  }
  return c;
}
U fill_add(const U& a, const U& b, GadgetW* w) {
  uint32_t al[NL], bl[NL];
  limbs(a, al);
  limbs(b, bl);
  int64_t prev = 0;
  for (uint32_t k = 0; k < NL; ++k) {
    const int64_t s = (int64_t)al[k] + bl[k] + prev;
    w->l0[k] = (uint32_t)(s & ((1 << LB) - 1));
    prev = s >> LB;
    w->cy[k] = prev;
  }
  return add9(a, b);
}
void signed_chain(const uint32_t* al, const uint32_t* bl, int64_t sign, uint32_t* out, int64_t* cy) {
  int64_t prev = 0;
  for (uint32_t k = 0; k < NL; ++k) {
    const int64_t lhs = (int64_t)al[k] + sign * (int64_t)P_TIGHT[k] - (bl ? (int64_t)bl[k] : 0) + prev;
    const int64_t m = lhs & ((1ll << LB) - 1);  // rem_euclid for a power of two
    out[k] = (uint32_t)m;
    prev = (lhs - m) >> LB;  // div_euclid
    cy[k] = prev;
  }
}
U fill_sub(const U& a, const U& b, GadgetW* w) {
  uint32_t al[NL], bl[NL];
  limbs(a, al);
  limbs(b, bl);
  signed_chain(al, bl, 1, w->l0, w->cy);
  return sub9(add9(a, kP), b);
}
U fill_freeze(const U& raw, GadgetW* w) {
  uint32_t al[NL];
  limbs(raw, al);
  signed_chain(al, nullptr, -1, w->l0, w->cy);
  if (w->cy[NL - 1] == -1)
    memcpy(w->l1, al, sizeof al);
  else
    memcpy(w->l1, w->l0, sizeof al);
  return from_limbs(w->l1);
}

void run_group(const std::vector<Op>& prog, const std::vector<Gadget>& T, std::vector<U>& val, GadgetW* gw) {
  for (const Op& o : prog) {
    const Gadget& g = T[o.g];
    if (o.type == 0) {
      val[g.p[2]] = fill_mul(val[g.p[0]], val[g.p[1]], &gw[o.g]);
    } else {
      const U raw = o.type == 1 ? fill_add(val[g.p[0]], val[g.p[1]], &gw[o.g])
                                : fill_sub(val[g.p[0]], val[g.p[1]], &gw[o.g]);
      val[T[o.fz].p[3]] = fill_freeze(raw, &gw[o.fz]);
    }
  }
}

void check_point(const U& x, const U& y) {
  require(lt(x, kP) && lt(y, kP), "p256: coordinate not below p");
  // y^2 = x^3 - 3x + b
  const U x3 = mulmod(mulmod(x, x, kP), x, kP);
  U rhs = add9(x3, kB);
  for (int i = 0; i < 3; ++i) {
    rhs = add9(rhs, sub9(kP, x));  // + (p - x)
  }
  uint32_t w18[18] = {0}, q[18], r[8];
  memcpy(w18, rhs.w, 36);
  bn::divmod(w18, 9, kP.w, 8, q, r);
  U rr{};
  memcpy(rr.w, r, 32);
  const U y2 = mulmod(y, y, kP);
  require(bn::cmp(rr.w, y2.w, 9) == 0, "p256: point not on the curve");
}

}  // namespace

const Layout& layout() { return built().L; }

void chain_witness(const uint8_t ax[32], const uint8_t ay[32], const uint8_t* a_bits, const uint8_t bx[32],
                   const uint8_t by[32], const uint8_t* b_bits, uint64_t k, RowW* rows, GadgetW* gw,
                   uint32_t r_proj[6][NL]) {
  const Built& B = built();
  const Layout& L = B.L;
  const uint32_t NG = (uint32_t)L.table.size();
  U base[2][3] = {{from_be(ax), from_be(ay), U{{1}}}, {from_be(bx), from_be(by), U{{1}}}};
  check_point(base[0][0], base[0][1]);
  check_point(base[1][0], base[1][1]);
  memset(rows, 0, k * sizeof(RowW));
  memset(gw, 0, k * NG * sizeof(GadgetW));
  U acc[2][3];
  memcpy(acc, base, sizeof acc);
  // The two chains share no cells or gadgets, so chain A runs on a second host
  // thread while this one builds chain B (each fills its own fields of the rows).
  auto run_chain = [&](int c) {
    const Chain& C = B.ch[c];
    std::vector<U> val(L.width);
    for (uint64_t r = 0; r < k; ++r) {
      RowW& rw = rows[r];
      GadgetW* g = gw + r * NG;
      const uint8_t bit = (c == 0 ? a_bits : b_bits)[r] ? 1 : 0;
      rw.bit[c] = bit;
      for (int x = 0; x < 3; ++x) {
        limbs(acc[c][x], rw.acc[c][x]);
        limbs(base[c][x], rw.base[c][x]);
        val[C.acc[x]] = acc[c][x];
        val[C.base[x]] = base[c][x];
      }
      val[C.b_double] = kB;
      val[C.b_add] = kB;
      run_group(C.prog_double, L.table, val, g);
      run_group(C.prog_add, L.table, val, g);
      for (int x = 0; x < 3; ++x) {
        const Gadget& s = L.table[C.sel_g[x]];
        const U chosen = bit ? val[s.p[0]] : val[s.p[1]];
        limbs(chosen, g[C.sel_g[x]].l0);
        acc[c][x] = chosen;
      }
    }
  };
  std::exception_ptr err_a;
  std::thread ta([&] {
    try {
      run_chain(0);
    } catch (...) {
      err_a = std::current_exception();
    }
  });
  std::exception_ptr err_b;
  try {
    run_chain(1);
  } catch (...) {
    err_b = std::current_exception();
  }
  ta.join();
  if (err_a) std::rethrow_exception(err_a);
  if (err_b) std::rethrow_exception(err_b);
  for (int c = 0; c < 2; ++c)
    for (int x = 0; x < 3; ++x) limbs(acc[c][x], r_proj[3 * c + x]);
}

void expand_host(const RowW* rows, const GadgetW* gw, const uint32_t r_proj[6][NL], uint64_t k, uint64_t* trace) {
  const Layout& L = layout();
  const uint32_t NG = (uint32_t)L.table.size();
  for (uint32_t col = 0; col < L.width; ++col)
    for (uint64_t r = 0; r < k; ++r)
      trace[col * k + r] =
          cell_value(L.cell_code[col], L.table.data(), rows[r], gw + r * NG, &r_proj[0][0], L.b_limbs);
}

void u_bits(const uint8_t digest[32], const uint8_t r_be[32], const uint8_t s_be[32], uint8_t u1[256],
            uint8_t u2[256]) {
  const U r = from_be(r_be), s = from_be(s_be);
  const U zero{};
  require(lt(r, kN) && lt(s, kN) && bn::cmp(r.w, zero.w, 9) != 0 && bn::cmp(s.w, zero.w, 9) != 0,
          "p256: r and s must lie in [1, n-1]");
  U e = from_be(digest);
  if (!lt(e, kN)) e = sub9(e, kN);  // a 256-bit digest is below 2n
  // w = s^(n-2) mod n
  U w{{1}};
  U nm2 = sub9(kN, U{{2}});
  for (int i = 255; i >= 0; --i) {
    w = mulmod(w, w, kN);
    if ((nm2.w[i / 32] >> (i % 32)) & 1) w = mulmod(w, s, kN);
  }
  const U a = mulmod(e, w, kN), b = mulmod(r, w, kN);
  for (int i = 0; i < 256; ++i) {
    u1[i] = (a.w[(255 - i) / 32] >> ((255 - i) % 32)) & 1;
    u2[i] = (b.w[(255 - i) / 32] >> ((255 - i) % 32)) & 1;
  }
}

void pi_hash(const uint8_t qx[32], const uint8_t qy[32], const uint8_t r[32], const uint8_t s[32],
             const uint8_t digest[32], uint8_t out[32]) {
  kc::Sha3 h;
  h.update("ECDSA-V1-PI-PRE", 15);
  h.update(qx, 32);
  h.update(qy, 32);
  h.update(r, 32);
  h.update(s, 32);
  h.update(digest, 32);
  h.finalize(out);
}

}  // namespace p256
}  // namespace sg

// oracle/gl.hpp — CPU restatement of the Goldilocks field and its sextic tower.
//
// TEST INFRASTRUCTURE ONLY. This file belongs to the oracle: the CPU model the
// GPU path is checked against. Nothing in the shipped library includes it.
//
// Follows (stark-stir-swarm paths):
//   crates/ark-goldilocks/build.rs:8-24       p = 2^64 - 2^32 + 1, generator 7,
//                                              two-adicity 32, root = 7^((p-1)/2^32)
//   crates/ark-goldilocks/src/lib.rs:28-43    Fp<MontBackend<_,2>,2>; values are
//                                              exchanged as canonical u64 (into_bigint().0[0])
//   crates/deep_ali/src/cubic_ext.rs:63-76    Fp3 = Fp[a]/(a^3 - 7), schoolbook mul (:166-175)
//   crates/deep_ali/src/cubic_ext.rs:205-226  Fp3 norm inverse
//   crates/deep_ali/src/sextic_ext.rs:72-100  Fp6 = Fp3[u]/(u^2 - a), mul_by_nonresidue
//   crates/deep_ali/src/sextic_ext.rs:200-287 Karatsuba mul, norm inverse, components
//                                              [c0.c0,c0.c1,c0.c2,c1.c0,c1.c1,c1.c2]
// Every value here is an exact field element, so any correct formula yields
// the same bits as the reference.
#pragma once
#include <cstdint>
#include <cstddef>

namespace orc {

static constexpr uint64_t P = 0xFFFFFFFF00000001ull;
static constexpr uint64_t EPS = 0xFFFFFFFFull;  // 2^64 mod p

struct Fp {
  uint64_t v;  // canonical, < P
  Fp() : v(0) {}
  explicit Fp(uint64_t x) : v(x >= P ? x - P : x) {}
  static Fp raw(uint64_t x) { Fp r; r.v = x; return r; }
  bool operator==(const Fp& o) const { return v == o.v; }
  bool operator!=(const Fp& o) const { return v != o.v; }
  bool is_zero() const { return v == 0; }
};

inline Fp add(Fp a, Fp b) {
  uint64_t s = a.v + b.v;
  bool carry = s < a.v;
  if (carry || s >= P) s -= P;  // with carry, s + 2^64 - P = s + EPS wraps correctly
  return Fp::raw(s);
}
inline Fp sub(Fp a, Fp b) {
  uint64_t d = a.v - b.v;
  if (a.v < b.v) d += P;
  return Fp::raw(d);
}
inline Fp neg(Fp a) { return a.v == 0 ? a : Fp::raw(P - a.v); }

// 128-bit reduction using 2^64 = 2^32 - 1 and 2^96 = -1 (mod p).
inline Fp reduce128(unsigned __int128 x) {
  uint64_t lo = (uint64_t)x, hi = (uint64_t)(x >> 64);
  uint64_t hh = hi >> 32, hl = hi & EPS;
  uint64_t t0 = lo - hh;
  if (lo < hh) t0 -= EPS;  // borrow: add p == subtract EPS mod 2^64
  uint64_t t1 = hl * EPS;
  uint64_t r = t0 + t1;
  if (r < t0) r += EPS;    // carry
  if (r >= P) r -= P;
  return Fp::raw(r);
}
inline Fp mul(Fp a, Fp b) { return reduce128((unsigned __int128)a.v * b.v); }
inline Fp sqr(Fp a) { return mul(a, a); }
inline Fp pow(Fp a, uint64_t e) {
  Fp r = Fp::raw(1);
  while (e) {
    if (e & 1) r = mul(r, a);
    a = mul(a, a);
    e >>= 1;
  }
  return r;
}
inline Fp inv(Fp a) { return pow(a, P - 2); }  // a != 0 assumed by callers

inline Fp operator+(Fp a, Fp b) { return add(a, b); }
inline Fp operator-(Fp a, Fp b) { return sub(a, b); }
inline Fp operator*(Fp a, Fp b) { return mul(a, b); }
inline Fp operator-(Fp a) { return neg(a); }

// Primitive 2^k-th root: square 7^((p-1)/2^32) (32-k) times
// (ark-ff get_root_of_unity, as used by ark-poly Radix2EvaluationDomain::new).
inline Fp root_of_unity(unsigned log_n) {
  Fp r = pow(Fp::raw(7), (P - 1) >> 32);
  for (unsigned i = log_n; i < 32; ++i) r = sqr(r);
  return r;
}

// ---------------------------------------------------------------- Fp3
struct Fp3 {
  Fp c[3];
};
inline Fp mul7(Fp x) { return mul(x, Fp::raw(7)); }
inline Fp3 f3_add(const Fp3& a, const Fp3& b) { return {{a.c[0] + b.c[0], a.c[1] + b.c[1], a.c[2] + b.c[2]}}; }
inline Fp3 f3_sub(const Fp3& a, const Fp3& b) { return {{a.c[0] - b.c[0], a.c[1] - b.c[1], a.c[2] - b.c[2]}}; }
inline Fp3 f3_mul(const Fp3& a, const Fp3& b) {
  Fp c0 = a.c[0] * b.c[0] + mul7(a.c[1] * b.c[2] + a.c[2] * b.c[1]);
  Fp c1 = a.c[0] * b.c[1] + a.c[1] * b.c[0] + mul7(a.c[2] * b.c[2]);
  Fp c2 = a.c[0] * b.c[2] + a.c[1] * b.c[1] + a.c[2] * b.c[0];
  return {{c0, c1, c2}};
}
inline Fp3 f3_scale(const Fp3& a, Fp s) { return {{a.c[0] * s, a.c[1] * s, a.c[2] * s}}; }
// multiply by the Fp6 non-residue (the cube root a): (x0,x1,x2) -> (7 x2, x0, x1)
inline Fp3 f3_mul_nr(const Fp3& x) { return {{mul7(x.c[2]), x.c[0], x.c[1]}}; }
inline Fp f3_norm(const Fp3& a) {
  Fp a0 = a.c[0], a1 = a.c[1], a2 = a.c[2];
  Fp w = Fp::raw(7), w2 = Fp::raw(49), three_w = Fp::raw(21);
  return a0 * a0 * a0 + w * (a1 * a1 * a1) + w2 * (a2 * a2 * a2) - three_w * a0 * a1 * a2;
}
inline bool f3_inv(const Fp3& a, Fp3* out) {
  Fp n = f3_norm(a);
  if (n.is_zero()) return false;
  Fp ni = inv(n);
  Fp a0 = a.c[0], a1 = a.c[1], a2 = a.c[2];
  out->c[0] = (a0 * a0 - mul7(a1 * a2)) * ni;
  out->c[1] = (mul7(a2 * a2) - a0 * a1) * ni;
  out->c[2] = (a1 * a1 - a0 * a2) * ni;
  return true;
}

// ---------------------------------------------------------------- Fp6
struct Fp6 {
  Fp3 a, b;  // a + b u, u^2 = (0,1,0)
  bool operator==(const Fp6& o) const {
    for (int i = 0; i < 3; ++i)
      if (a.c[i] != o.a.c[i] || b.c[i] != o.b.c[i]) return false;
    return true;
  }
  bool operator!=(const Fp6& o) const { return !(*this == o); }
  bool is_zero() const {
    for (int i = 0; i < 3; ++i)
      if (!a.c[i].is_zero() || !b.c[i].is_zero()) return false;
    return true;
  }
  Fp comp(int i) const { return i < 3 ? a.c[i] : b.c[i - 3]; }
  void set_comp(int i, Fp x) {
    if (i < 3) a.c[i] = x; else b.c[i - 3] = x;
  }
};
inline Fp6 e_zero() { return Fp6{}; }
inline Fp6 e_one() { Fp6 r{}; r.a.c[0] = Fp::raw(1); return r; }
inline Fp6 e_from(Fp x) { Fp6 r{}; r.a.c[0] = x; return r; }
inline Fp6 e_add(const Fp6& x, const Fp6& y) { return {f3_add(x.a, y.a), f3_add(x.b, y.b)}; }
inline Fp6 e_sub(const Fp6& x, const Fp6& y) { return {f3_sub(x.a, y.a), f3_sub(x.b, y.b)}; }
inline Fp6 e_mul(const Fp6& x, const Fp6& y) {
  Fp3 v0 = f3_mul(x.a, y.a), v1 = f3_mul(x.b, y.b);
  Fp3 c0 = f3_add(v0, f3_mul_nr(v1));
  Fp3 c1 = f3_sub(f3_sub(f3_mul(f3_add(x.a, x.b), f3_add(y.a, y.b)), v0), v1);
  return {c0, c1};
}
inline Fp6 e_scale(const Fp6& x, Fp s) { return {f3_scale(x.a, s), f3_scale(x.b, s)}; }
inline bool e_inv(const Fp6& x, Fp6* out) {
  Fp3 n = f3_sub(f3_mul(x.a, x.a), f3_mul_nr(f3_mul(x.b, x.b)));
  Fp3 ni;
  if (!f3_inv(n, &ni)) return false;
  out->a = f3_mul(x.a, ni);
  Fp3 t = f3_mul(x.b, ni);
  out->b = {{-t.c[0], -t.c[1], -t.c[2]}};
  return true;
}
// square-and-multiply (fri.rs:146-159 ext_pow)
inline Fp6 e_pow(Fp6 base, uint64_t e) {
  Fp6 r = e_one();
  while (e) {
    if (e & 1) r = e_mul(r, base);
    base = e_mul(base, base);
    e >>= 1;
  }
  return r;
}

}  // namespace orc

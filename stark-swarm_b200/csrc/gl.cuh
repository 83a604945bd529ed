// gl.cuh — Goldilocks field p = 2^64 - 2^32 + 1 and its sextic tower, for
// host and device. Elements are canonical uint64 (< p) everywhere in this
// library: trace, LDE, quotient and STIR layers are stored canonical, which is
// also the byte form the reference hashes (le64 of into_bigint().0[0],
// merkle/src/lib.rs:56-62) and serializes.
//
// Tower (deep_ali/src/cubic_ext.rs:63-76, sextic_ext.rs:72-100):
//   Fp3 = Fp[a]/(a^3 - 7),  Fp6 = Fp3[u]/(u^2 - a),
//   components ordered [c0.c0, c0.c1, c0.c2, c1.c0, c1.c1, c1.c2].
// On the device the 64x64-bit products compile to 32-bit IMAD chains
// (mul.lo.u64 / mul.hi.u64); reduction uses 2^64 = 2^32 - 1 and 2^96 = -1.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define GL_HD __host__ __device__ __forceinline__
#else
#define GL_HD inline
#endif

namespace gl {

static constexpr uint64_t P = 0xFFFFFFFF00000001ull;
static constexpr uint64_t EPS = 0xFFFFFFFFull;

#if defined(__CUDA_ARCH__)
// Device versions: 32-bit carry chains in hand-written PTX. A 64-bit add or
// compare costs the compiler several ALU instructions each; with explicit
// carries the canonical add is 9, sub 5 and the 128-bit reduction 20 ALU
// instructions, and the 64x64 product is 9 IMADs on the (otherwise idle) FMA pipe.
// a + b = a - (p - b). For b = 0 the subtrahend is p itself and a - p borrows
// back to a, so no special case is needed: 2 + 5 instructions.
__device__ __forceinline__ uint64_t add(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("{\n\t.reg .u32 a0, a1, b0, b1, n0, n1, d0, d1, bw;\n\t"
      "mov.b64 {a0, a1}, %1;\n\tmov.b64 {b0, b1}, %2;\n\t"
      "sub.cc.u32 n0, 1, b0;\n\tsubc.u32 n1, 0xFFFFFFFF, b1;\n\t"
      "sub.cc.u32 d0, a0, n0;\n\tsubc.cc.u32 d1, a1, n1;\n\tsubc.u32 bw, 0, 0;\n\t"
      "sub.cc.u32 d0, d0, bw;\n\tsubc.u32 d1, d1, 0;\n\t"
      "mov.b64 %0, {d0, d1};\n\t}"
      : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ uint64_t sub(uint64_t a, uint64_t b) {
  uint64_t r;
  asm("{\n\t.reg .u32 a0, a1, b0, b1, d0, d1, bw;\n\t"
      "mov.b64 {a0, a1}, %1;\n\tmov.b64 {b0, b1}, %2;\n\t"
      "sub.cc.u32 d0, a0, b0;\n\tsubc.cc.u32 d1, a1, b1;\n\tsubc.u32 bw, 0, 0;\n\t"
      "sub.cc.u32 d0, d0, bw;\n\tsubc.u32 d1, d1, 0;\n\t"
      "mov.b64 %0, {d0, d1};\n\t}"
      : "=l"(r) : "l"(a), "l"(b));
  return r;
}
// x = x0 + x1 2^32 + x2 2^64 + x3 2^96 = (lo) + x2 (2^32 - 1) - x3  (mod p), canonical result
__device__ __forceinline__ uint64_t reduce128(uint64_t hi, uint64_t lo) {
  uint64_t r;
  asm("{\n\t.reg .u32 x0, x1, x2, x3, t0, t1, u0, u1, c, m;\n\t.reg .pred p;\n\t"
      "mov.b64 {x0, x1}, %1;\n\tmov.b64 {x2, x3}, %2;\n\t"
      "sub.cc.u32 t0, x0, x3;\n\tsubc.cc.u32 t1, x1, 0;\n\tsubc.u32 c, 0, 0;\n\t"
      "sub.cc.u32 t0, t0, c;\n\tsubc.u32 t1, t1, 0;\n\t"
      "sub.cc.u32 u0, 0, x2;\n\tsubc.u32 u1, x2, 0;\n\t"
      "add.cc.u32 t0, t0, u0;\n\taddc.cc.u32 t1, t1, u1;\n\taddc.u32 c, 0, 0;\n\t"
      "sub.u32 m, 0, c;\n\tadd.cc.u32 t0, t0, m;\n\taddc.u32 t1, t1, 0;\n\t"
      "add.cc.u32 u0, t0, 0xFFFFFFFF;\n\taddc.cc.u32 u1, t1, 0;\n\taddc.u32 c, 0, 0;\n\t"
      "setp.ne.u32 p, c, 0;\n\tselp.b32 t0, u0, t0, p;\n\tselp.b32 t1, u1, t1, p;\n\t"
      "mov.b64 %0, {t0, t1};\n\t}"
      : "=l"(r) : "l"(lo), "l"(hi));
  return r;
}
__device__ __forceinline__ uint64_t mul(uint64_t a, uint64_t b) {
  uint64_t lo, hi;
  asm("{\n\t.reg .u32 a0, a1, b0, b1, x0, x1, x2, x3;\n\t"
      "mov.b64 {a0, a1}, %2;\n\tmov.b64 {b0, b1}, %3;\n\t"
      "mul.lo.u32 x0, a0, b0;\n\tmul.hi.u32 x1, a0, b0;\n\t"
      "mad.lo.cc.u32 x1, a0, b1, x1;\n\tmadc.hi.u32 x2, a0, b1, 0;\n\t"
      "mad.lo.cc.u32 x1, a1, b0, x1;\n\tmadc.hi.cc.u32 x2, a1, b0, x2;\n\taddc.u32 x3, 0, 0;\n\t"
      "mad.lo.cc.u32 x2, a1, b1, x2;\n\tmadc.hi.u32 x3, a1, b1, x3;\n\t"
      "mov.b64 %0, {x0, x1};\n\tmov.b64 %1, {x2, x3};\n\t}"
      : "=l"(lo), "=l"(hi) : "l"(a), "l"(b));
  return reduce128(hi, lo);
}
#else
inline uint64_t add(uint64_t a, uint64_t b) {
  uint64_t s = a + b;
  bool c = s < a;
  return (c || s >= P) ? s - P : s;
}
inline uint64_t sub(uint64_t a, uint64_t b) {
  uint64_t d = a - b;
  return a < b ? d + P : d;
}
inline uint64_t reduce128(uint64_t hi, uint64_t lo) {
  uint64_t hh = hi >> 32, hl = hi & EPS;
  uint64_t t0 = lo - hh;
  if (lo < hh) t0 -= EPS;
  uint64_t t1 = hl * EPS;
  uint64_t r = t0 + t1;
  if (r < t0) r += EPS;
  return r >= P ? r - P : r;
}
inline uint64_t mul(uint64_t a, uint64_t b) {
  unsigned __int128 x = (unsigned __int128)a * b;
  return reduce128((uint64_t)(x >> 64), (uint64_t)x);
}
#endif
#if defined(__CUDACC__)
// x * 2^e for canonical x and 0 <= e < 96, canonical result. With
// x * 2^f = y2 2^64 + y1 2^32 + y0 (f < 32), 2^64 = 2^32 - 1 and 2^96 = -1:
//   e = f:       (y1:y0) + y2 (2^32 - 1)
//   e = 32 + f:  (s + c) 2^32 - (c + y1 + y2),  s + c 2^32 = y0 + y1
//   e = 64 + f:  y0 2^32 - (y2 2^32 + y0 + y1)
// The shifts stay in C++ so a constant e folds into them; only the carry chains
// are PTX (16, 15 and 10 instructions, against 24 to 50 through reduce128).
__device__ __forceinline__ void shl96(uint64_t x, unsigned f, uint32_t& y0, uint32_t& y1, uint32_t& y2) {
  const uint32_t x0 = (uint32_t)x, x1 = (uint32_t)(x >> 32);
  if (f == 0) {
    y0 = x0;
    y1 = x1;
    y2 = 0;
  } else {
    y0 = x0 << f;
    y1 = __funnelshift_l(x0, x1, f);
    y2 = x1 >> (32 - f);
  }
}
__device__ __forceinline__ uint64_t mul2e_lo(uint32_t y0, uint32_t y1, uint32_t y2) {
  uint64_t r;
  asm("{\n\t.reg .u32 t0, t1, s0, s1, u0, u1, c, m;\n\t.reg .pred p;\n\t"
      "sub.cc.u32 t0, 0, %3;\n\tsubc.u32 t1, %3, 0;\n\t"
      "add.cc.u32 s0, %1, t0;\n\taddc.cc.u32 s1, %2, t1;\n\taddc.u32 c, 0, 0;\n\t"
      "sub.u32 m, 0, c;\n\tadd.cc.u32 s0, s0, m;\n\taddc.u32 s1, s1, 0;\n\t"
      "add.cc.u32 u0, s0, 0xFFFFFFFF;\n\taddc.cc.u32 u1, s1, 0;\n\taddc.u32 c, 0, 0;\n\t"
      "setp.ne.u32 p, c, 0;\n\tselp.b32 s0, u0, s0, p;\n\tselp.b32 s1, u1, s1, p;\n\t"
      "mov.b64 %0, {s0, s1};\n\t}"
      : "=l"(r) : "r"(y0), "r"(y1), "r"(y2));
  return r;
}
__device__ __forceinline__ uint64_t mul2e_mid(uint32_t y0, uint32_t y1, uint32_t y2) {
  uint64_t r;
  asm("{\n\t.reg .u32 s, c, d0, d1, r0, r1, bw;\n\t"
      "add.cc.u32 s, %1, %2;\n\taddc.u32 c, 0, 0;\n\tadd.u32 s, s, c;\n\t"
      "add.cc.u32 d0, %2, %3;\n\taddc.u32 d1, 0, 0;\n\tadd.cc.u32 d0, d0, c;\n\taddc.u32 d1, d1, 0;\n\t"
      "sub.cc.u32 r0, 0, d0;\n\tsubc.cc.u32 r1, s, d1;\n\tsubc.u32 bw, 0, 0;\n\t"
      "sub.cc.u32 r0, r0, bw;\n\tsubc.u32 r1, r1, 0;\n\t"
      "mov.b64 %0, {r0, r1};\n\t}"
      : "=l"(r) : "r"(y0), "r"(y1), "r"(y2));
  return r;
}
__device__ __forceinline__ uint64_t mul2e_hi(uint32_t y0, uint32_t y1, uint32_t y2) {
  uint64_t r;
  asm("{\n\t.reg .u32 b0, b1, r0, r1, bw;\n\t"
      "add.cc.u32 b0, %1, %2;\n\taddc.u32 b1, %3, 0;\n\t"
      "sub.cc.u32 r0, 0, b0;\n\tsubc.cc.u32 r1, %1, b1;\n\tsubc.u32 bw, 0, 0;\n\t"
      "sub.cc.u32 r0, r0, bw;\n\tsubc.u32 r1, r1, 0;\n\t"
      "mov.b64 %0, {r0, r1};\n\t}"
      : "=l"(r) : "r"(y0), "r"(y1), "r"(y2));
  return r;
}
__device__ __forceinline__ uint64_t mul2e(uint64_t x, unsigned e) {
  uint32_t y0, y1, y2;
  if (e == 0) return x;
  if (e < 32) {
    shl96(x, e, y0, y1, y2);
    return mul2e_lo(y0, y1, y2);
  }
  if (e < 64) {
    shl96(x, e - 32, y0, y1, y2);
    return mul2e_mid(y0, y1, y2);
  }
  shl96(x, e - 64, y0, y1, y2);
  return mul2e_hi(y0, y1, y2);
}
// Sum of x_b 2^b terms (b < 32) in a 128-bit accumulator with one reduction at the
// end: 7 instructions a term instead of a reduction and a field add.
struct Acc128 {
  uint32_t a0 = 0, a1 = 0, a2 = 0, a3 = 0;
  __device__ __forceinline__ void add_shl(uint64_t x, unsigned f) {
    uint32_t y0, y1, y2;
    shl96(x, f, y0, y1, y2);
    asm("add.cc.u32 %0, %0, %4;\n\taddc.cc.u32 %1, %1, %5;\n\taddc.cc.u32 %2, %2, %6;\n\taddc.u32 %3, %3, 0;"
        : "+r"(a0), "+r"(a1), "+r"(a2), "+r"(a3) : "r"(y0), "r"(y1), "r"(y2));
  }
  // x 2^(32 + f), f < 32: the same three words one limb up (the sum must stay below 2^128)
  __device__ __forceinline__ void add_shl32(uint64_t x, unsigned f) {
    uint32_t y0, y1, y2;
    shl96(x, f, y0, y1, y2);
    asm("add.cc.u32 %0, %0, %3;\n\taddc.cc.u32 %1, %1, %4;\n\taddc.u32 %2, %2, %5;"
        : "+r"(a1), "+r"(a2), "+r"(a3) : "r"(y0), "r"(y1), "r"(y2));
  }
  // lam * x for lam < 2^32: 4 IMADs and 3 adds
  __device__ __forceinline__ void add_mul32(uint32_t lam, uint64_t x) {
    const uint32_t x0 = (uint32_t)x, x1 = (uint32_t)(x >> 32);
    asm("mad.lo.cc.u32 %0, %4, %6, %0;\n\tmadc.hi.cc.u32 %1, %4, %6, %1;\n\t"
        "addc.cc.u32 %2, %2, 0;\n\taddc.u32 %3, %3, 0;\n\t"
        "mad.lo.cc.u32 %1, %5, %6, %1;\n\tmadc.hi.cc.u32 %2, %5, %6, %2;\n\taddc.u32 %3, %3, 0;"
        : "+r"(a0), "+r"(a1), "+r"(a2), "+r"(a3) : "r"(x0), "r"(x1), "r"(lam));
  }
  __device__ __forceinline__ uint64_t reduce() const {
    return reduce128((uint64_t)a3 << 32 | a2, (uint64_t)a1 << 32 | a0);
  }
};
#endif
GL_HD uint64_t neg(uint64_t a) { return a ? P - a : 0; }
GL_HD uint64_t sqr(uint64_t a) { return mul(a, a); }

GL_HD uint64_t pow(uint64_t a, uint64_t e) {
  uint64_t r = 1;
  while (e) {
    if (e & 1) r = mul(r, a);
    a = mul(a, a);
    e >>= 1;
  }
  return r;
}
GL_HD uint64_t inv(uint64_t a) { return pow(a, P - 2); }

// x * 2^e for 0 <= e < 64 (shifts and one reduction, no multiply)
GL_HD uint64_t mul_pow2_lt64(uint64_t x, unsigned e) {
#if defined(__CUDA_ARCH__)
  return mul2e(x, e);
#else
  if (e == 0) return x;
  return reduce128(x >> (64 - e), x << e);
#endif
}
// x * 2^e for any 0 <= e < 192 (2 has order 192 in this field; 2^96 = -1)
GL_HD uint64_t mul_pow2(uint64_t x, unsigned e) {
  bool negate = false;
  if (e >= 96) {
    e -= 96;
    negate = true;
  }
#if defined(__CUDA_ARCH__)
  const uint64_t r = mul2e(x, e);
#else
  const uint64_t r = e < 64 ? mul_pow2_lt64(x, e) : mul_pow2_lt64(mul_pow2_lt64(x, e - 32), 32);
#endif
  return negate ? neg(r) : r;
}

// Primitive 2^k-th root of unity of ark-poly's Radix2EvaluationDomain:
// 7^((p-1)/2^32) squared (32-k) times (ark-goldilocks/build.rs:20-24).
GL_HD uint64_t root_of_unity(unsigned log_n) {
  uint64_t r = pow(7, (P - 1) >> 32);
  for (unsigned i = log_n; i < 32; ++i) r = sqr(r);
  return r;
}

// ------------------------------------------------------------------ Fp6
struct Fp6 {
  uint64_t c[6];
};

GL_HD Fp6 e_zero() { return Fp6{{0, 0, 0, 0, 0, 0}}; }
GL_HD Fp6 e_one() { return Fp6{{1, 0, 0, 0, 0, 0}}; }
GL_HD Fp6 e_from(uint64_t x) { return Fp6{{x, 0, 0, 0, 0, 0}}; }
GL_HD bool e_eq(const Fp6& a, const Fp6& b) {
  bool r = true;
  for (int i = 0; i < 6; ++i) r = r && a.c[i] == b.c[i];
  return r;
}
GL_HD Fp6 e_add(const Fp6& a, const Fp6& b) {
  Fp6 r;
  for (int i = 0; i < 6; ++i) r.c[i] = add(a.c[i], b.c[i]);
  return r;
}
GL_HD Fp6 e_sub(const Fp6& a, const Fp6& b) {
  Fp6 r;
  for (int i = 0; i < 6; ++i) r.c[i] = sub(a.c[i], b.c[i]);
  return r;
}
GL_HD Fp6 e_scale(const Fp6& a, uint64_t s) {
  Fp6 r;
  for (int i = 0; i < 6; ++i) r.c[i] = mul(a.c[i], s);
  return r;
}
GL_HD uint64_t mul7(uint64_t x) {
  // 7x = 8x - x with one reduction
  return sub(mul_pow2_lt64(x, 3), x);
}
// Fp3 product, schoolbook with a^3 = 7 (cubic_ext.rs:166-175)
GL_HD void f3_mul(const uint64_t* a, const uint64_t* b, uint64_t* r) {
  uint64_t c0 = add(mul(a[0], b[0]), mul7(add(mul(a[1], b[2]), mul(a[2], b[1]))));
  uint64_t c1 = add(add(mul(a[0], b[1]), mul(a[1], b[0])), mul7(mul(a[2], b[2])));
  uint64_t c2 = add(add(mul(a[0], b[2]), mul(a[1], b[1])), mul(a[2], b[0]));
  r[0] = c0;
  r[1] = c1;
  r[2] = c2;
}
// Fp6 product, Karatsuba over Fp3 with u^2 = a (sextic_ext.rs:200-206)
GL_HD Fp6 e_mul(const Fp6& x, const Fp6& y) {
  uint64_t v0[3], v1[3], sa[3], sb[3], m[3];
  f3_mul(x.c, y.c, v0);
  f3_mul(x.c + 3, y.c + 3, v1);
  for (int i = 0; i < 3; ++i) {
    sa[i] = add(x.c[i], x.c[3 + i]);
    sb[i] = add(y.c[i], y.c[3 + i]);
  }
  f3_mul(sa, sb, m);
  Fp6 r;
  // c0 = v0 + a*v1 ; a*(t0,t1,t2) = (7 t2, t0, t1)
  r.c[0] = add(v0[0], mul7(v1[2]));
  r.c[1] = add(v0[1], v1[0]);
  r.c[2] = add(v0[2], v1[1]);
  for (int i = 0; i < 3; ++i) r.c[3 + i] = sub(sub(m[i], v0[i]), v1[i]);
  return r;
}
#if defined(__CUDACC__)
// e_mul as a real call: one copy of its code per kernel. For kernels that run a
// few CTAs once through (the small STIR layers), fully inlined Fp6 products make
// the warps wait on instruction fetch; a call keeps the code small and cached.
static __device__ __noinline__ Fp6 e_mul_call(const Fp6 x, const Fp6 y) { return e_mul(x, y); }
static __device__ __forceinline__ Fp6 e_pow_call(Fp6 b, uint64_t e) {
  Fp6 r = e_one();
#pragma unroll 1
  while (e) {
    if (e & 1) r = e_mul_call(r, b);
    b = e_mul_call(b, b);
    e >>= 1;
  }
  return r;
}
#endif
GL_HD Fp6 e_pow(Fp6 b, uint64_t e) {
  Fp6 r = e_one();
  while (e) {
    if (e & 1) r = e_mul(r, b);
    b = e_mul(b, b);
    e >>= 1;
  }
  return r;
}
// Inverse through the Fp3 and Fp norms (cubic_ext.rs:205-226, sextic_ext.rs:240-256).
// Returns false for zero.
GL_HD bool e_inv(const Fp6& x, Fp6* out) {
  uint64_t aa[3], bb[3], n3[3];
  f3_mul(x.c, x.c, aa);
  f3_mul(x.c + 3, x.c + 3, bb);
  n3[0] = sub(aa[0], mul7(bb[2]));
  n3[1] = sub(aa[1], bb[0]);
  n3[2] = sub(aa[2], bb[1]);
  // Fp3 inverse of n3
  uint64_t a0 = n3[0], a1 = n3[1], a2 = n3[2];
  uint64_t t = mul(mul(a0, a0), a0);
  t = add(t, mul(7, mul(mul(a1, a1), a1)));
  t = add(t, mul(49, mul(mul(a2, a2), a2)));
  t = sub(t, mul(21, mul(mul(a0, a1), a2)));
  if (t == 0) return false;
  uint64_t ti = inv(t);
  uint64_t i3[3];
  i3[0] = mul(sub(mul(a0, a0), mul7(mul(a1, a2))), ti);
  i3[1] = mul(sub(mul7(mul(a2, a2)), mul(a0, a1)), ti);
  i3[2] = mul(sub(mul(a1, a1), mul(a0, a2)), ti);
  uint64_t r0[3], r1[3];
  f3_mul(x.c, i3, r0);
  f3_mul(x.c + 3, i3, r1);
  for (int i = 0; i < 3; ++i) {
    out->c[i] = r0[i];
    out->c[3 + i] = neg(r1[i]);
  }
  return true;
}

}  // namespace gl

// oracle/rsa2048_air.hpp — CPU restatement of the RSA-2048 exponentiation AIR.
//
// TEST INFRASTRUCTURE ONLY (part of the oracle; never linked into the product).
//
// Follows (stark-stir-swarm paths):
//   crates/deep_ali/src/rsa2048_field_air.rs:56-104   80 limbs of 26 bits, 159 cross slots,
//                                                     40 carry bits biased by 2^39
//   crates/deep_ali/src/rsa2048_field_air.rs:131-170  mul-gadget cell order: c, q, q_bits, c_bits, carry bits
//   crates/deep_ali/src/rsa2048_field_air.rs:339-412  eval_rsa_mul_gadget constraint order
//   crates/deep_ali/src/rsa2048_exp_air.rs:97-124     record cell order: acc, s, n, phase, op2, em, gadget
//   crates/deep_ali/src/rsa2048_exp_air.rs:219-286    eval_rsa_exp_multirow_per_row (boundary row 16,
//                                                     transitions gated by row + 1 < n_trace)
//   crates/deep_ali/src/rsa2048_stacked_air.rs:22-70  records side by side, constraints concatenated
// The trace itself is built in Python (tests/oracle_lib.py) with Python
// integers, so the oracle's big-integer arithmetic is independent of the
// library's.
#pragma once
#include <cstddef>
#include <cstdint>

#include "gl.hpp"

namespace orc {
namespace rsa {

static constexpr size_t LIMBS = 80, LIMB_BITS = 26, SLOTS = 2 * LIMBS - 1, CARRY_BITS = 40,
                        CARRY_POS = SLOTS - 1;
static constexpr uint64_t CARRY_OFFSET = 1ull << (CARRY_BITS - 1);
// record layout
static constexpr size_t ACC = 0, S = 80, N = 160, PHASE = 240, OP2 = 241, EM = 321, C = 401, Q = 481,
                        Q_BITS = 561, C_BITS = Q_BITS + LIMBS * LIMB_BITS, CARRY = C_BITS + LIMBS * LIMB_BITS,
                        WIDTH = CARRY + CARRY_BITS * CARRY_POS;
static constexpr size_t GADGET_CONSTRAINTS = 2 * LIMBS * (1 + LIMB_BITS) + SLOTS + CARRY_POS * CARRY_BITS;
static constexpr size_t CONSTRAINTS = 1 + LIMBS + GADGET_CONSTRAINTS + LIMBS + 4 * LIMBS;
static constexpr size_t OUTPUT_ROW = 16;
static_assert(WIDTH == 11041, "record width");
static_assert(GADGET_CONSTRAINTS == 10799, "gadget constraint count (rsa2048_field_air.rs:88-92)");
static_assert(CONSTRAINTS == 11280, "per-row constraint count");

// One record's 11,280 constraint values at one row; cur/nxt point at the record's first cell.
inline void eval_record(const Fp* cur, const Fp* nxt, size_t row, size_t n_trace, Fp* out) {
  size_t o = 0;
  const Fp one = Fp::raw(1);
  const Fp phase = cur[PHASE];
  out[o++] = phase * (one - phase);
  for (size_t i = 0; i < LIMBS; ++i) out[o++] = cur[OP2 + i] - (phase * (cur[S + i] - cur[ACC + i]) + cur[ACC + i]);
  auto range = [&](size_t limbs, size_t bits) {
    for (size_t i = 0; i < LIMBS * LIMB_BITS; ++i) out[o++] = cur[bits + i] * (one - cur[bits + i]);
    for (size_t i = 0; i < LIMBS; ++i) {
      Fp s;
      for (size_t b = 0; b < LIMB_BITS; ++b) s = s + Fp(1ull << b) * cur[bits + i * LIMB_BITS + b];
      out[o++] = cur[limbs + i] - s;
    }
  };
  range(C, C_BITS);
  range(Q, Q_BITS);
  auto carry = [&](size_t k) {
    if (k >= CARRY_POS) return Fp();
    Fp s;
    for (size_t b = 0; b < CARRY_BITS; ++b) s = s + Fp(1ull << b) * cur[CARRY + k * CARRY_BITS + b];
    return s - Fp(CARRY_OFFSET);
  };
  const Fp radix = Fp(1ull << LIMB_BITS);
  for (size_t k = 0; k < SLOTS; ++k) {
    Fp ab, qn;
    const size_t lo = k >= LIMBS - 1 ? k - (LIMBS - 1) : 0, hi = k < LIMBS - 1 ? k : LIMBS - 1;
    for (size_t i = lo; i <= hi; ++i) {
      ab = ab + cur[ACC + i] * cur[OP2 + k - i];
      qn = qn + cur[Q + i] * cur[N + k - i];
    }
    const Fp ck = k < LIMBS ? cur[C + k] : Fp();
    const Fp cin = k == 0 ? Fp() : carry(k - 1);
    out[o++] = ab - qn - ck + cin - radix * carry(k);
  }
  for (size_t i = 0; i < CARRY_POS * CARRY_BITS; ++i) out[o++] = cur[CARRY + i] * (one - cur[CARRY + i]);
  for (size_t i = 0; i < LIMBS; ++i) out[o++] = row == OUTPUT_ROW ? cur[C + i] - cur[EM + i] : Fp();
  const bool tr = row + 1 < n_trace;
  for (size_t i = 0; i < LIMBS; ++i) out[o++] = tr ? nxt[ACC + i] - cur[C + i] : Fp();
  for (size_t i = 0; i < LIMBS; ++i) out[o++] = tr ? nxt[S + i] - cur[S + i] : Fp();
  for (size_t i = 0; i < LIMBS; ++i) out[o++] = tr ? nxt[N + i] - cur[N + i] : Fp();
  for (size_t i = 0; i < LIMBS; ++i) out[o++] = tr ? nxt[EM + i] - cur[EM + i] : Fp();
}

}  // namespace rsa
}  // namespace orc

// oracle/p256_air.hpp — CPU restatement of the P-256 ECDSA double-chain AIR's constraints.
//
// TEST INFRASTRUCTURE ONLY (part of the oracle; never linked into the product).
//
// The row layout is a table of gadget instances in constraint-emission order,
// built by tests/oracle_p256.py from the reference's layout builders; this file
// evaluates each gadget exactly as the reference does:
//   crates/deep_ali/src/p256_field_air.rs:404-434   eval_add_gadget      (290 constraints)
//   crates/deep_ali/src/p256_field_air.rs:636-690   eval_sub_gadget      (311)
//   crates/deep_ali/src/p256_field_air.rs:1044-1140 eval_mul_gadget      (1207)
//   crates/deep_ali/src/p256_field_air.rs:1243-1268 eval_select_gadget   (281)
//   crates/deep_ali/src/p256_field_air.rs:1449-1535 eval_freeze_gadget   (591)
//   crates/deep_ali/src/p256_group_air.rs:645-680,1048-1071  group double / add: muls, adds,
//       subs, freezes after adds, freezes after subs
//   crates/deep_ali/src/p256_scalar_mul_air.rs:224-240  step: double, add, select x/y/z
//   crates/deep_ali/src/p256_ecdsa_double_multirow_air.rs:236-308  two steps, 60 boundary
//       slots (last row), 120 transition slots (rows + 1 < n_trace)
#pragma once
#include <cstddef>
#include <cstdint>

#include "gl.hpp"

namespace orc {
namespace p256 {

static constexpr size_t NL = 10, LB = 26, MUL_CB = 36, MUL_CP = 18, MUL_SP = 19;
static const uint64_t P_TIGHT[NL] = {0x3FFFFFF, 0x3FFFFFF, 0x3FFFFFF, 0x003FFFF, 0, 0, 0, 0x0000400, 0x3FF0000,
                                     0x03FFFFF};
enum : uint64_t { G_MUL = 1, G_ADD = 2, G_SUB = 3, G_FREEZE = 4, G_SELECT = 5 };
// gadget record: kind, then up to 7 cell bases
//   MUL    a b c c_bits q q_bits carry_bits
//   ADD    a b c c_bits carries
//   SUB    a b c c_bits c_pos c_neg
//   FREEZE a diff diff_bits c c_bits c_pos c_neg
//   SELECT a b c c_bits sel
static constexpr size_t REC = 8;

inline size_t gadget_constraints(uint64_t kind) {
  switch (kind) {
    case G_MUL: return 2 * (NL * LB + NL) + MUL_SP + MUL_CP * MUL_CB;
    case G_ADD: return NL * LB + NL + 2 * NL;
    case G_SUB: return NL * LB + NL + NL + 2 * NL + NL + 1;
    case G_FREEZE: return 2 * (NL * LB + NL) + NL + 2 * NL + NL + 1 + NL;
    case G_SELECT: return NL * LB + NL + NL + 1;
    default: return 0;
  }
}

inline void range(const Fp* cur, uint64_t limbs, uint64_t bits, Fp*& out) {
  const Fp one = Fp::raw(1);
  for (size_t i = 0; i < NL * LB; ++i) *out++ = cur[bits + i] * (one - cur[bits + i]);
  for (size_t i = 0; i < NL; ++i) {
    Fp s;
    for (size_t b = 0; b < LB; ++b) s = s + Fp(1ull << b) * cur[bits + i * LB + b];
    *out++ = cur[limbs + i] - s;
  }
}

inline void eval_gadget(const Fp* cur, const uint64_t* g, Fp*& out) {
  const Fp one = Fp::raw(1), radix = Fp(1ull << LB);
  switch (g[0]) {
    case G_MUL: {
      const uint64_t a = g[1], b = g[2], c = g[3], cb = g[4], q = g[5], qb = g[6], cy = g[7];
      range(cur, c, cb, out);
      range(cur, q, qb, out);
      auto carry = [&](size_t k) {
        if (k >= MUL_CP) return Fp();
        Fp s;
        for (size_t bb = 0; bb < MUL_CB; ++bb) s = s + Fp(1ull << bb) * cur[cy + k * MUL_CB + bb];
        return s - Fp(1ull << (MUL_CB - 1));
      };
      for (size_t k = 0; k < MUL_SP; ++k) {
        Fp ab, qp;
        const size_t lo = k >= NL - 1 ? k - (NL - 1) : 0, hi = k < NL - 1 ? k : NL - 1;
        for (size_t i = lo; i <= hi; ++i) {
          ab = ab + cur[a + i] * cur[b + k - i];
          qp = qp + cur[q + i] * Fp(P_TIGHT[k - i]);
        }
        const Fp ck = k < NL ? cur[c + k] : Fp();
        const Fp cin = k == 0 ? Fp() : carry(k - 1);
        *out++ = ab - qp - ck + cin - radix * carry(k);
      }
      for (size_t i = 0; i < MUL_CP * MUL_CB; ++i) *out++ = cur[cy + i] * (one - cur[cy + i]);
      break;
    }
    case G_ADD: {
      const uint64_t a = g[1], b = g[2], c = g[3], cb = g[4], cr = g[5];
      range(cur, c, cb, out);
      for (size_t k = 0; k < NL; ++k) {
        const Fp cin = k == 0 ? Fp() : cur[cr + k - 1];
        *out++ = cur[a + k] + cur[b + k] + cin - cur[c + k] - radix * cur[cr + k];
      }
      for (size_t k = 0; k + 1 < NL; ++k) *out++ = cur[cr + k] * (one - cur[cr + k]);
      *out++ = cur[cr + NL - 1];
      break;
    }
    case G_SUB: {
      const uint64_t a = g[1], b = g[2], c = g[3], cb = g[4], pos = g[5], neg = g[6];
      range(cur, c, cb, out);
      auto net = [&](size_t k) { return cur[pos + k] - cur[neg + k]; };
      for (size_t k = 0; k < NL; ++k) {
        const Fp cin = k == 0 ? Fp() : net(k - 1);
        *out++ = cur[a + k] + Fp(P_TIGHT[k]) - cur[b + k] + cin - cur[c + k] - radix * net(k);
      }
      for (size_t k = 0; k < NL; ++k) *out++ = cur[pos + k] * (one - cur[pos + k]);
      for (size_t k = 0; k < NL; ++k) *out++ = cur[neg + k] * (one - cur[neg + k]);
      for (size_t k = 0; k < NL; ++k) *out++ = cur[pos + k] * cur[neg + k];
      *out++ = cur[pos + NL - 1] + cur[neg + NL - 1];
      break;
    }
    case G_FREEZE: {
      const uint64_t a = g[1], d = g[2], db = g[3], c = g[4], cb = g[5], pos = g[6], neg = g[7];
      range(cur, d, db, out);
      range(cur, c, cb, out);
      auto net = [&](size_t k) { return cur[pos + k] - cur[neg + k]; };
      for (size_t k = 0; k < NL; ++k) {
        const Fp cin = k == 0 ? Fp() : net(k - 1);
        *out++ = cur[a + k] - Fp(P_TIGHT[k]) - cur[d + k] + cin - radix * net(k);
      }
      for (size_t k = 0; k < NL; ++k) *out++ = cur[pos + k] * (one - cur[pos + k]);
      for (size_t k = 0; k < NL; ++k) *out++ = cur[neg + k] * (one - cur[neg + k]);
      for (size_t k = 0; k < NL; ++k) *out++ = cur[pos + k] * cur[neg + k];
      *out++ = cur[pos + NL - 1];
      const Fp n9 = cur[neg + NL - 1];
      for (size_t k = 0; k < NL; ++k) *out++ = cur[c + k] - cur[d + k] - n9 * (cur[a + k] - cur[d + k]);
      break;
    }
    case G_SELECT: {
      const uint64_t a = g[1], b = g[2], c = g[3], cb = g[4], sel = g[5];
      range(cur, c, cb, out);
      const Fp s = cur[sel];
      for (size_t k = 0; k < NL; ++k) *out++ = cur[c + k] - cur[b + k] - s * (cur[a + k] - cur[b + k]);
      *out++ = s * (one - s);
      break;
    }
    default: break;
  }
}

// tail[0..11]: chain A acc x,y,z; chain A select outputs x,y,z; chain B acc x,y,z;
// chain B select outputs x,y,z; tail[12..17]: r_proj a x,y,z, b x,y,z.
inline void eval_tail(const Fp* cur, const Fp* nxt, const uint64_t* tail, size_t row, size_t n_trace, Fp*& out) {
  const bool last = row + 1 == n_trace;
  for (int ch = 0; ch < 2; ++ch)
    for (int x = 0; x < 3; ++x) {
      const uint64_t c = tail[6 * ch + 3 + x], r = tail[12 + 3 * ch + x];
      for (size_t i = 0; i < NL; ++i) *out++ = last ? cur[c + i] - cur[r + i] : Fp();
    }
  const bool tr = row + 1 < n_trace;
  for (int ch = 0; ch < 2; ++ch)
    for (int x = 0; x < 3; ++x) {
      const uint64_t acc = tail[6 * ch + x], c = tail[6 * ch + 3 + x];
      for (size_t i = 0; i < NL; ++i) *out++ = tr ? nxt[acc + i] - cur[c + i] : Fp();
    }
  for (int k = 0; k < 6; ++k) {
    const uint64_t r = tail[12 + k];
    for (size_t i = 0; i < NL; ++i) *out++ = tr ? nxt[r + i] - cur[r + i] : Fp();
  }
}

}  // namespace p256
}  // namespace orc

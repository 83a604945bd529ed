// oracle/ed25519_air.hpp — CPU restatement of the Ed25519 verify AIR's (v16) constraints.
//
// TEST INFRASTRUCTURE ONLY (part of the oracle; never linked into the product).
//
// The row's constraint vector is a program of blocks in emission order, each with
// a row gate (built by tests/oracle_ed25519.py from the v0..v16 compositions of
// ed25519_verify_air.rs); a block whose gate is closed emits its count of zeros,
// as the reference's evaluators do. Each block is evaluated as the reference does
// (crates/deep_ali/src/ paths):
//   sha512_air.rs:909-1270            eval_sha512_constraints (sha512_air.hpp)
//   ed25519_scalar_air.rs:412-583     eval_scalar_reduce_gadget (1674; its 16 r + slack slots are 0)
//   ed25519_verify_air.rs:487-538     v1 format conversion: digest-bit booleanity, H-state
//                                     packs, byte-swapped input limbs (560)
//   ed25519_field_air.rs:431-486      eval_add_gadget    (285)
//   ed25519_field_air.rs:672-730      eval_sub_gadget    (305)
//   ed25519_field_air.rs:1000-1076    eval_mul_gadget    (635)
//   ed25519_field_air.rs:1457-1475    eval_select_gadget (11)
//   ed25519_group_air.rs:1050-1068    decompressed-x range check (265)
//   ed25519_group_air.rs:1080-1086    sign-bit booleanity and match (2)
//   ed25519_verify_air.rs (v4..v16)   pins, copies and transitions: A - B pairs
#pragma once
#include <cstddef>
#include <cstdint>

#include "gl.hpp"
#include "sha512_air.hpp"

namespace orc {
namespace ed25519 {

static constexpr size_t NL = 10, MUL_CB = 36, REC = 16;
static constexpr unsigned LW[NL] = {26, 25, 26, 25, 26, 25, 26, 25, 26, 25};
static constexpr unsigned RED_IN = 32, RED_R = 16, RED_Q = 17, RED_LB = 16, RED_CB = 24, RED_PROD = 33;
enum : uint64_t { GATE_ALWAYS = 0, GATE_EQ = 1, GATE_RANGE = 2, GATE_SET = 3 };
enum : uint64_t { B_SHA512 = 1, B_REDUCE, B_FORMAT, B_MUL, B_ADD, B_SUB, B_SEL, B_RANGE, B_SIGN, B_PAIRS };
static constexpr uint64_t SRC_MASK = (1ull << 62) - 1;

// L = 2^252 + 27742317777372353535851937790883648493 in 16-bit limbs (ed25519_scalar.rs:33-39)
static constexpr uint64_t L16[RED_R] = {0xd3ed, 0x5cf5, 0x631a, 0x5812, 0x9cd6, 0xa2f7, 0xf9de, 0x14de,
                                        0,      0,      0,      0,      0,      0,      0,      0x1000};

inline size_t block_count(const uint64_t* r, const uint64_t* /*pairs*/) {
  switch (r[4]) {
    case B_SHA512: return sha512::NUM_CONSTRAINTS;
    case B_REDUCE: return RED_Q * RED_LB + RED_Q + 2 * (RED_R * RED_LB + RED_R) + RED_R + RED_PROD + RED_PROD * RED_CB;
    case B_FORMAT: return 512 + 16 + 32;
    case B_MUL: return 265 + NL + MUL_CB * NL;
    case B_ADD: return 265 + 2 * NL;
    case B_SUB: return 265 + 4 * NL;
    case B_SEL: return 1 + NL;
    case B_RANGE: return 265;
    case B_SIGN: return 2;
    default: return r[6];  // B_PAIRS: offset, count
  }
}

inline bool gate_open(const uint64_t* r, size_t row) {
  switch (r[0]) {
    case GATE_ALWAYS: return true;
    case GATE_EQ: return row == r[1];
    case GATE_RANGE: return row >= r[1] && row < r[2];
    default: return row == r[1] || row == r[2] || row == r[3];
  }
}

// 255 booleanity constraints of the bits, then the 10 limb packs
inline void range(const Fp* cur, uint64_t limbs, uint64_t bits, Fp*& out) {
  const Fp one = Fp::raw(1);
  for (size_t b = 0; b < 255; ++b) *out++ = cur[bits + b] * (one - cur[bits + b]);
  size_t off = 0;
  for (size_t i = 0; i < NL; ++i) {
    Fp s;
    for (unsigned b = 0; b < LW[i]; ++b) s = s + Fp(1ull << b) * cur[bits + off + b];
    *out++ = cur[limbs + i] - s;
    off += LW[i];
  }
}

inline Fp ref(const Fp* cur, const Fp* nxt, uint64_t r) {
  const uint64_t src = r >> 62, v = r & SRC_MASK;
  return src == 0 ? cur[v] : src == 1 ? nxt[v] : Fp(v);
}

inline void eval_block(const Fp* cur, const Fp* nxt, size_t row, const uint64_t* r, const uint64_t* pairs, Fp*& out) {
  const Fp one = Fp::raw(1);
  const uint64_t* p = r + 5;
  switch (r[4]) {
    case B_SHA512:
      sha512::eval(cur, nxt, row, p[0], out);
      out += sha512::NUM_CONSTRAINTS;
      return;
    case B_REDUCE: {
      const uint64_t in = p[0], q = p[1], qb = p[2], rl = p[3], rb = p[4], sl = p[5], sb = p[6], cb = p[7];
      auto rc = [&](uint64_t limbs, uint64_t bits, size_t n) {
        for (size_t i = 0; i < n * RED_LB; ++i) *out++ = cur[bits + i] * (one - cur[bits + i]);
        for (size_t i = 0; i < n; ++i) {
          Fp s;
          for (unsigned b = 0; b < RED_LB; ++b) s = s + Fp(1ull << b) * cur[bits + i * RED_LB + b];
          *out++ = cur[limbs + i] - s;
        }
      };
      rc(q, qb, RED_Q);
      rc(rl, rb, RED_R);
      rc(sl, sb, RED_R);
      for (size_t i = 0; i < RED_R; ++i) *out++ = Fp();  // the unenforced r + slack = L - 1 slots
      auto carry = [&](size_t k) {
        Fp s;
        for (unsigned b = 0; b < RED_CB; ++b) s = s + Fp(1ull << b) * cur[cb + k * RED_CB + b];
        return s - Fp(1ull << (RED_CB - 1));
      };
      for (size_t k = 0; k < RED_PROD; ++k) {
        const Fp in_k = k < RED_IN ? cur[in + k] : Fp();
        Fp ql;
        for (size_t i = 0; i < RED_Q; ++i)
          if (k >= i && k - i < RED_R) ql = ql + cur[q + i] * Fp(L16[k - i]);
        const Fp r_k = k < RED_R ? cur[rl + k] : Fp();
        const Fp cin = k == 0 ? Fp() : carry(k - 1);
        *out++ = in_k - ql - r_k + cin - Fp(1ull << RED_LB) * carry(k);
      }
      for (size_t i = 0; i < RED_PROD * RED_CB; ++i) *out++ = cur[cb + i] * (one - cur[cb + i]);
      return;
    }
    case B_FORMAT: {
      const uint64_t db = p[0], in = p[1], h0 = p[2];
      for (size_t i = 0; i < 512; ++i) *out++ = cur[db + i] * (one - cur[db + i]);
      for (size_t k = 0; k < 8; ++k) {
        Fp lo, hi;
        for (unsigned i = 0; i < 32; ++i) {
          lo = lo + Fp(1ull << i) * cur[db + 64 * k + i];
          hi = hi + Fp(1ull << i) * cur[db + 64 * k + 32 + i];
        }
        *out++ = cur[h0 + 2 * k] - lo;
        *out++ = cur[h0 + 2 * k + 1] - hi;
      }
      for (size_t k = 0; k < 8; ++k)
        for (size_t m = 0; m < 4; ++m) {
          const size_t lb = 56 - 16 * m, hb = lb - 8;
          Fp s;
          for (unsigned j = 0; j < 8; ++j) s = s + Fp(1ull << j) * cur[db + 64 * k + lb + j];
          for (unsigned j = 0; j < 8; ++j) s = s + Fp(1ull << (8 + j)) * cur[db + 64 * k + hb + j];
          *out++ = nxt[in + 4 * k + m] - s;
        }
      return;
    }
    case B_MUL: {
      const uint64_t a = p[0], b = p[1], c = p[2], cbits = p[3], cy = p[4];
      range(cur, c, cbits, out);
      auto carry = [&](size_t k) {
        Fp s;
        for (size_t bb = 0; bb < MUL_CB; ++bb) s = s + Fp(1ull << bb) * cur[cy + k * MUL_CB + bb];
        return s - Fp(1ull << (MUL_CB - 1));
      };
      for (size_t k = 0; k < NL; ++k) {
        Fp t;
        for (size_t i = 0; i < NL; ++i)
          for (size_t j = 0; j < NL; ++j) {
            const bool odd = (i & 1) && (j & 1);
            if (i + j == k)
              t = t + Fp(odd ? 2 : 1) * cur[a + i] * cur[b + j];
            else if (i + j == k + NL)
              t = t + Fp(odd ? 38 : 19) * cur[a + i] * cur[b + j];
          }
        const Fp cin = k == 0 ? Fp(19) * carry(NL - 1) : carry(k - 1);
        *out++ = t + cin - cur[c + k] - Fp(1ull << LW[k]) * carry(k);
      }
      for (size_t i = 0; i < MUL_CB * NL; ++i) *out++ = cur[cy + i] * (one - cur[cy + i]);
      return;
    }
    case B_ADD: {
      const uint64_t a = p[0], b = p[1], c = p[2], cbits = p[3], cr = p[4];
      range(cur, c, cbits, out);
      for (size_t k = 0; k < NL; ++k) {
        const Fp cin = k == 0 ? Fp(19) * cur[cr + NL - 1] : cur[cr + k - 1];
        *out++ = cur[a + k] + cur[b + k] + cin - cur[c + k] - Fp(1ull << LW[k]) * cur[cr + k];
      }
      for (size_t k = 0; k < NL; ++k) *out++ = cur[cr + k] * (one - cur[cr + k]);
      return;
    }
    case B_SUB: {
      const uint64_t a = p[0], b = p[1], c = p[2], cbits = p[3], pos = p[4], neg = p[5];
      range(cur, c, cbits, out);
      auto net = [&](size_t k) { return cur[pos + k] - cur[neg + k]; };
      for (size_t k = 0; k < NL; ++k) {
        const Fp nin = k == 0 ? Fp(19) * net(NL - 1) : net(k - 1);
        *out++ = cur[a + k] - cur[b + k] - nin - cur[c + k] + Fp(1ull << LW[k]) * net(k);
      }
      for (size_t k = 0; k < NL; ++k) *out++ = cur[pos + k] * (one - cur[pos + k]);
      for (size_t k = 0; k < NL; ++k) *out++ = cur[neg + k] * (one - cur[neg + k]);
      for (size_t k = 0; k < NL; ++k) *out++ = cur[pos + k] * cur[neg + k];
      return;
    }
    case B_SEL: {
      const uint64_t a = p[0], b = p[1], bit = p[2], c = p[3];
      const Fp s = cur[bit];
      *out++ = s * (one - s);
      for (size_t k = 0; k < NL; ++k) *out++ = cur[c + k] - cur[a + k] - s * (cur[b + k] - cur[a + k]);
      return;
    }
    case B_RANGE:
      range(cur, p[0], p[1], out);
      return;
    case B_SIGN: {
      const Fp sb = cur[p[0]];
      *out++ = sb * (one - sb);
      *out++ = cur[p[1]] - sb;
      return;
    }
    default:
      for (size_t i = 0; i < p[1]; ++i) {
        const uint64_t* pr = pairs + 2 * (p[0] + i);
        *out++ = ref(cur, nxt, pr[0]) - ref(cur, nxt, pr[1]);
      }
      return;
  }
}

// The row's constraint vector; returns the number of values written.
inline size_t eval_row(const Fp* cur, const Fp* nxt, size_t row, const uint64_t* recs, size_t n_recs,
                       const uint64_t* pairs, Fp* out) {
  Fp* o = out;
  for (size_t i = 0; i < n_recs; ++i) {
    const uint64_t* r = recs + i * REC;
    if (gate_open(r, row)) {
      eval_block(cur, nxt, row, r, pairs, o);
    } else {
      const size_t n = block_count(r, pairs);
      for (size_t j = 0; j < n; ++j) *o++ = Fp();
    }
  }
  return (size_t)(o - out);
}

}  // namespace ed25519
}  // namespace orc

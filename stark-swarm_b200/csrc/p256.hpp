// p256.hpp — P-256 ECDSA signature check as an AIR: the double-chain scalar
// multiplication of deep_ali/src/p256_ecdsa_double_multirow_air.rs.
//
// Each trace row holds two scalar-multiplication steps (chain A for u1·G, chain
// B for u2·Q). A step doubles the accumulator, adds the chain's base point and
// selects the sum or the double by the row's bit (p256_scalar_mul_air.rs). Double
// and add are straight-line programs of field gadgets (p256_group_air.rs): mul
// (c = a b mod p with witness quotient q and 18 carries biased by 2^35), add
// (limb carries 0/1), sub (a + p - b, carries -1/0/1), freeze (canonical form of
// a value below 2p) and select (p256_field_air.rs). Field elements are 10 limbs
// of 26 bits.
//
// The row is described by a table of gadget instances in constraint-emission
// order (per group gadget: muls, adds, subs, freezes after adds, freezes after
// subs; per step: double, add, selects x/y/z; then chain B) plus 180 tail
// constraints: 60 boundary slots binding the chains' outputs to the r_proj
// columns on the last row, and 120 transition slots (next accumulator = this
// row's selected point, r_proj constant). Row width 151,334 cells; 155,774
// constraints per row.
#pragma once
#include <cstdint>
#include <vector>

namespace sg {
namespace p256 {

enum : uint32_t {
  NL = 10, LB = 26, ELEM = NL + NL * LB, MUL_CB = 36, MUL_CP = 18, MUL_SP = 19,
  MUL_OWNED = 2 * ELEM + MUL_CP * MUL_CB, ADD_OWNED = ELEM + NL, SUB_OWNED = ELEM + 2 * NL,
  FREEZE_OWNED = 2 * ELEM + 2 * NL,
  G_MUL = 1, G_ADD = 2, G_SUB = 3, G_FREEZE = 4, G_SELECT = 5,
  TAIL_CONSTRAINTS = 180, BLOWUP = 32, K_ECDSA = 256
};
static constexpr uint64_t P_TIGHT[NL] = {0x3FFFFFF, 0x3FFFFFF, 0x3FFFFFF, 0x003FFFF, 0, 0, 0,
                                         0x0000400, 0x3FF0000, 0x03FFFFF};

// A gadget instance: kind and its cell bases (see oracle layout comment):
//   MUL    a b c c_bits q q_bits carry_bits
//   ADD    a b c c_bits carries
//   SUB    a b c c_bits c_pos c_neg
//   FREEZE a diff diff_bits c c_bits c_pos c_neg
//   SELECT a b c c_bits sel
struct Gadget {
  uint32_t kind, p[7];
};
#if defined(__CUDACC__)
__host__ __device__
#endif
inline uint32_t gadget_constraints(uint32_t kind) {
  switch (kind) {
    case G_MUL: return 2 * ELEM + MUL_SP + MUL_CP * MUL_CB;
    case G_ADD: return ELEM + 2 * NL;
    case G_SUB: return ELEM + NL + 2 * NL + NL + 1;
    case G_FREEZE: return 2 * ELEM + NL + 2 * NL + NL + 1 + NL;
    case G_SELECT: return ELEM + NL + 1;
    default: return 0;
  }
}
// first cell of a gadget's own region, and its length
inline uint32_t owned_start(const Gadget& g) { return g.kind == G_FREEZE ? g.p[1] : g.p[2]; }
inline uint32_t owned_len(uint32_t kind) {
  return kind == G_MUL ? MUL_OWNED : kind == G_ADD ? ADD_OWNED : kind == G_SUB ? SUB_OWNED
                                                    : kind == G_FREEZE ? FREEZE_OWNED : ELEM;
}

// Per-row witness of one gadget instance (everything its own cells are read from):
//   MUL    l0 = c limbs, l1 = q limbs, cy = the 18 signed carries
//   ADD    l0 = c limbs, cy[0..9] = carries (0/1)
//   SUB    l0 = c limbs, cy[0..9] = carries (-1/0/1)
//   FREEZE l0 = diff limbs, l1 = c limbs, cy[0..9] = carries (-1/0/1)
//   SELECT l0 = c limbs
struct GadgetW {
  uint32_t l0[NL], l1[NL];
  int64_t cy[MUL_CP];
};
// Per-row cells outside every gadget: the chains' accumulators, bases and bits.
struct RowW {
  uint32_t acc[2][3][NL], base[2][3][NL], bit[2], pad[2];
};

// Cells not owned by a gadget are classified by a per-cell code
// (category << 28 | payload); gadget-owned cells carry gadget index << 11 | offset.
enum : uint32_t { C_GADGET = 0, C_ACC = 1, C_BASE = 2, C_BIT = 3, C_B = 4, C_RPROJ = 5 };

struct Layout {
  uint32_t width = 0, n_constraints = 0;
  std::vector<Gadget> table;        // constraint order
  std::vector<uint32_t> lam_base;   // first constraint index of each gadget
  uint32_t tail[18];                // acc A xyz, out A xyz, acc B xyz, out B xyz, r_proj A xyz, B xyz
  std::vector<uint32_t> cell_code;  // width entries
  uint32_t b_limbs[NL];             // the curve's b, canonical limbs
};
const Layout& layout();

// The per-row witnesses of the two chains: each starts at (x, y, 1) of its affine
// point (32-byte big-endian coordinates) and takes one bit per row (k rows).
// Fills rows (k entries), gadget witnesses (k * 260, row-major) and the chains'
// final projective outputs (r_proj: A x,y,z then B x,y,z as limbs); the caller
// provides the buffers (pinned host memory on the proving path). Throws SgError
// (SG_EINVAL) for a coordinate >= p or a point not on the curve.
void chain_witness(const uint8_t ax[32], const uint8_t ay[32], const uint8_t* a_bits, const uint8_t bx[32],
                   const uint8_t by[32], const uint8_t* b_bits, uint64_t k, RowW* rows, GadgetW* gw,
                   uint32_t r_proj[6][NL]);
// The column-major width x k trace on the host.
void expand_host(const RowW* rows, const GadgetW* gw, const uint32_t r_proj[6][NL], uint64_t k, uint64_t* trace);
// u1 = e s^-1, u2 = r s^-1 mod n as MSB-first bits (e = digest mod n); throws
// SgError (SG_EINVAL) unless 1 <= r, s < n.
void u_bits(const uint8_t digest[32], const uint8_t r[32], const uint8_t s[32], uint8_t u1[256], uint8_t u2[256]);
// pi_hash of prove_ecdsa_record_v1.rs:213-222.
void pi_hash(const uint8_t qx[32], const uint8_t qy[32], const uint8_t r[32], const uint8_t s[32],
             const uint8_t digest[32], uint8_t out[32]);
// The generator G (FIPS 186-4 D.1.2.3), 32-byte big-endian coordinates.
extern const uint8_t GX[32], GY[32];

}  // namespace p256
}  // namespace sg

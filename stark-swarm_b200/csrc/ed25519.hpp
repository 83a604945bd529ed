// ed25519.hpp — Ed25519 signature verification as an AIR: the v16 composition of
// deep_ali/src/ed25519_verify_air.rs, which proves the RFC 8032 §5.1.7 cofactored
// predicate [8]([s]B - R - [k]A) = O with k = SHA-512(R || A || M) mod L.
//
// Trace rows (ed25519_verify_air.rs:64-80): the SHA-512 compression rows of
// R || A || M (k_hash rows, the last one also carrying the digest's 512 bits),
// the scalar reduction mod L, the decompressions of R and of A, the [s]B ladder
// (k rows), the [k]A ladder (k rows), the residual row (two subtractions as
// point additions of negated points), three doublings and the verdict row;
// height next_pow2(k_hash + 3 + 2k + 5). Field elements of 2^255 - 19 are 10
// limbs of 26/25 bits; every gadget (add, sub, mul, select) owns its output
// limbs, their 255 range bits and its carries (ed25519_field_air.rs).
//
// The constraint vector (70,606 values for k = 256) is a program of blocks in
// the reference's emission order, each gated by the row; the trace is held as
// per-row words (limb values, carries, bits) and per-phase cell codes from which
// every cell is read (ed25519_cells), so only the words cross to the device.
#pragma once
#include <cstdint>
#include <vector>

#include "sha512_air.cuh"

#if defined(__CUDACC__)
#define ED_HD __host__ __device__ __forceinline__
#else
#define ED_HD inline
#endif

namespace sg {
namespace ed25519 {

enum : uint32_t {
  NL = 10, ELEM = 265, MUL_CB = 36, SHA_W = 1510, SHA_K = 1526, SHA_H0_LO = 1066, BLOWUP = 32, K_FULL = 256,
  RED_IN = 32, RED_R = 16, RED_Q = 17, RED_LB = 16, RED_CB = 24, RED_PROD = 33,
  MUL_K = ELEM + NL + MUL_CB * NL, ADD_K = ELEM + 2 * NL, SUB_K = ELEM + 4 * NL, SEL_K = 1 + NL,
  REDUCE_K = RED_Q * RED_LB + RED_Q + 2 * (RED_R * RED_LB + RED_R) + RED_R + RED_PROD + RED_PROD * RED_CB,
  FORMAT_K = 512 + 16 + 32
};
static constexpr uint32_t LW[NL] = {26, 25, 26, 25, 26, 25, 26, 25, 26, 25};
static constexpr uint32_t LOFF[NL] = {0, 26, 51, 77, 102, 128, 153, 179, 204, 230};

// ---------------------------------------------------------------- layout
struct GMul { uint32_t a, b, c, bits, carry; };
struct GAdd { uint32_t a, b, c, bits, carries; };
struct GSub { uint32_t a, b, c, bits, pos, neg; };
struct GSel { uint32_t a, b, bit, c; };
// point_add_layout_at (ed25519_group_air.rs:202-249): out = X3, Y3, Z3, T3
struct PAdd {
  uint32_t p1[4], p2[4], d2;
  GSub sub_ym1, sub_ym2;
  GAdd add_yp1, add_yp2;
  GMul mul_A, mul_B, mul_tt, mul_C, mul_zz;
  GAdd add_D;
  GSub sub_E, sub_F;
  GAdd add_G, add_H;
  GMul mul_X3, mul_Y3, mul_T3, mul_Z3;
  uint32_t out[4], end;
};
// point_double_layout_at (ed25519_group_air.rs:476-505)
struct PDbl {
  uint32_t p1[3];
  GMul sq_A, sq_B, sq_zz;
  GAdd add_C, add_H, add_xy;
  GMul sq_xy;
  GSub sub_E, sub_G;
  GAdd add_F;
  GMul mul_X3, mul_Y3, mul_T3, mul_Z3;
  uint32_t out[4], end;
};
// cond_add_layout_at (ed25519_group_air.rs:662-719)
struct CAdd {
  uint32_t bit, out[4];
  PAdd add;
  GSel sel[4];
  uint32_t end;
};
// point_decompress_layout_at (ed25519_group_air.rs:887-955)
struct Decomp {
  uint32_t y, sign, d, x, x_bits;
  GMul sq_x, sq_y, mul_dx2, mul_dxy;
  uint32_t one;
  GSub sub_y2m1, sub_lhs, sub_eq;
  uint32_t sign_match, end;
};
struct Reduce { uint32_t input, q, q_bits, r, r_bits, slack, slack_bits, carry_bits; };

// VerifyAirLayoutV16 (ed25519_verify_air.rs:4670-4814)
struct Layout {
  uint32_t k = 0, n_blocks = 0, k_hash = 0, width = 0, height = 0, n_constraints = 0;
  uint32_t reduce_row, decomp_R_row, decomp_A_row, sB_first, sB_last, kA_first, kA_last, residual_row, dbl_row[3],
      result_row;
  Reduce red;
  uint32_t digest_bits;
  Decomp decomp;
  uint32_t base[4], acc[4];
  PDbl mdbl;
  CAdd cadd;
  uint32_t sblock_sB, sblock_kA, r_thread;
  uint32_t result[4], zero_const;
  GSub sub_X, sub_T, sub_YZ;
  uint32_t dbl_in[3];
  PDbl dbl;
  uint32_t thr_sB[4], thr_kA[4], thr_R[4], one_R;
  GMul mul_RT;
  uint32_t zero_R1;
  GSub sub_negR_X, sub_negR_T;
  PAdd pa_R1;
  GSub sub_negkA_X, sub_negkA_T;
  PAdd pa_R2;
};
// sha_len = 64 + message bytes (the SHA-512 input R || A || M); 2 <= k <= 256.
Layout make_layout(uint64_t sha_len, uint32_t k);
// verify_v16_per_row_constraints
uint32_t n_constraints(uint32_t k);

// ---------------------------------------------------------------- constraint program
enum : uint32_t { GATE_ALWAYS = 0, GATE_EQ = 1, GATE_RANGE = 2, GATE_SET = 3 };
enum : uint32_t { B_SHA512 = 1, B_REDUCE, B_FORMAT, B_MUL, B_ADD, B_SUB, B_SEL, B_RANGE, B_SIGN, B_PAIRS };
// A block of the constraint vector: row gate (EQ r; RANGE lo <= row < hi; SET of
// up to three rows, unused = ~0), kind, cell bases (PAIRS: first pair, count), the
// index of its first constraint, and its length. A pair is two references
// src << 62 | cell (src 0 = this row, 1 = next row) or 2 << 62 | constant; its
// constraint is A - B.
struct Block {
  uint32_t gate, g[3], kind, p[8], lam, count;
};
enum : uint64_t { SRC_CUR = 0, SRC_NXT = 1, SRC_CONST = 2 };
struct Program {
  std::vector<Block> blocks;
  std::vector<uint64_t> pairs;  // 2 per pair
  uint32_t n_constraints = 0;
};
ED_HD bool gate_open(const Block& b, uint32_t row) {
  switch (b.gate) {
    case GATE_ALWAYS: return true;
    case GATE_EQ: return row == b.g[0];
    case GATE_RANGE: return row >= b.g[0] && row < b.g[1];
    default: return row == b.g[0] || row == b.g[1] || row == b.g[2];
  }
}

// ---------------------------------------------------------------- trace cells
// A cell code: op (3 bits) << 29 | bit (6 bits) << 23 | index (23 bits) into the
// row's words (or the proof's global words for threads shared by every row).
enum : uint32_t { OP_ZERO = 0, OP_WORD = 1, OP_BIT = 2, OP_POS = 3, OP_NEG = 4, OP_GLOBAL = 5 };
// row kinds of the trace: which cells a row fills
enum : uint32_t {
  PH_IDLE, PH_SHA, PH_DIGEST, PH_REDUCE, PH_DECOMP_R, PH_DECOMP_A, PH_SB, PH_KA, PH_RESIDUAL, PH_DBL, PH_RESULT,
  N_PHASES
};
ED_HD uint32_t code(uint32_t op, uint32_t idx, uint32_t bit = 0) { return op << 29 | bit << 23 | idx; }
ED_HD uint64_t cell_value(uint32_t c, const uint64_t* words, const uint64_t* globals) {
  const uint32_t op = c >> 29, bit = (c >> 23) & 63, idx = c & 0x7FFFFF;
  switch (op) {
    case OP_WORD: return words[idx];
    case OP_BIT: return (words[idx] >> bit) & 1;
    case OP_POS: return words[idx] == 1;
    case OP_NEG: return words[idx] == ~0ull;
    case OP_GLOBAL: return globals[idx];
    default: return 0;
  }
}

// Everything the trace is read from: the SHA-512 block witnesses (rows < k_hash,
// columns < 1510), per-phase codes (N_PHASES x width), each row's phase and words.
struct Witness {
  Layout L;
  Program prog;
  std::vector<sha512::BlockWitness> sha;
  std::vector<uint32_t> codes;
  std::vector<uint8_t> row_phase;
  std::vector<uint32_t> row_off;  // height + 1
  std::vector<uint64_t> words, globals;
};

// fill_verify_air_v16 (ed25519_verify_air.rs:4820-4868) for prove_zsk_ksk_binding_v2's
// inputs (swarm-dns/src/prover.rs:856-903): the public key, the 64-byte signature
// R || S and the signed data; k ladder rows (256 for Ed25519). Throws SgError
// (SG_EINVAL) when R or A does not decode (y >= p, not on the curve, or x = 0
// with the sign bit set) or k is out of range.
void build_witness(const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg, uint64_t len, uint32_t k,
                   Witness* w);
// The column-major width x height trace on the host.
void expand_host(const Witness& w, uint64_t* trace);

// Which LDE values the merge reads. The trace LDE feeds only the merge (the proof
// commits to c_eval alone, swarm-dns/src/prover.rs:904-916), and a point reads a
// cell only when a block open on its row (or, through a next-row reference, on the
// row before) names it. Columns below `dense` are read on most rows and get the
// full LDE; a constant column's LDE is its value; a sparse column is non-zero on at
// most kSparseRows trace rows and read on at most kSparseRows rows, so its LDE at
// the points of a read row a (point a blowup + j) is sum over its non-zero rows r
// of v_r L_r(w_N^(a blowup + j)), with L_r the Lagrange basis of the trace domain.
struct LdePlan {
  static constexpr uint32_t kSparseRows = 8;
  uint32_t dense = 0;           // columns [0, dense) take the NTT LDE
  bool ok = false;              // false: every column takes the NTT LDE
  std::vector<uint32_t> const_cols;
  // sparse columns in groups with the same non-zero and read rows
  struct Group {
    std::vector<uint32_t> nz, read, cols;
  };
  std::vector<Group> groups;
};
LdePlan make_lde_plan(const Witness& w);
// RFC 8032 §5.1.7 cofactored verification (ed25519_verify.rs:54-117).
bool verify(const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg, uint64_t len);
// zsk_ksk_pi_hash_v2_stark (swarm-dns/src/prover.rs:763-780).
void pi_hash(const uint8_t pub[32], const uint8_t sig[64], const uint8_t* msg, uint64_t len,
             const uint8_t fs_binding[32], const uint8_t merkle_root[32], const uint8_t root_f0[32], uint8_t out[32]);

}  // namespace ed25519
}  // namespace sg

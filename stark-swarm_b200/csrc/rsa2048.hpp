// rsa2048.hpp — RSA-2048 PKCS#1 v1.5 (SHA-256) signature check as an AIR:
// the e = 65537 exponentiation chain of deep_ali/src/rsa2048_exp_air.rs with one
// witness-quotient multiply gadget per row (rsa2048_field_air.rs), n_records
// records side by side (rsa2048_stacked_air.rs).
//
// Record layout (11,041 cells; rsa2048_exp_air.rs:97-124, rsa2048_field_air.rs:131-170):
//   acc[80] s[80] n[80] phase op2[80] em[80] | c[80] q[80] q_bits[80*26] c_bits[80*26] carry_bits[158*40]
// 2048-bit integers are 80 little-endian limbs of 26 bits. Row r computes
// c = acc * op2 mod n with a * b = q * n + c checked slot by slot through a carry
// chain whose 158 carries are stored biased by 2^39 in 40 bits each. op2 = s on
// row 16 (phase 1) and acc elsewhere: 16 squarings, then the multiply by s.
//
// Constraint order per record (11,280; rsa2048_exp_air.rs:219-286,
// rsa2048_field_air.rs:339-412):
//   0            phase (1 - phase)
//   1..80        op2_i - (phase (s_i - acc_i) + acc_i)
//   81..2160     c bits b (1 - b);  2161..2240  c_i - sum_b 2^b c_bit
//   2241..4320   q bits;            4321..4400  q_i - sum_b 2^b q_bit
//   4401..4559   slot k: sum a_i b_{k-i} - sum q_i n_{k-i} - c_k + carry_{k-1} - 2^26 carry_k
//   4560..10879  carry bits b (1 - b)
//   10880..10959 row 16 only: c_i - em_i
//   10960..11279 rows with row + 1 < n_trace: nxt acc - c, nxt s - s, nxt n - n, nxt em - em
#pragma once
#include <cstdint>
#include <vector>

namespace sg {
namespace rsa {

enum : uint32_t {
  LIMBS = 80, LIMB_BITS = 26, SLOTS = 159, CARRY_BITS = 40, CARRY_POS = 158,
  ACC = 0, S = 80, N = 160, PHASE = 240, OP2 = 241, EM = 321, C = 401, Q = 481,
  Q_BITS = 561, C_BITS = Q_BITS + LIMBS * LIMB_BITS, CARRY = C_BITS + LIMBS * LIMB_BITS,
  WIDTH = CARRY + CARRY_BITS * CARRY_POS,
  // constraint index bases
  K_PHASE = 0, K_SELECT = 1, K_CBOOL = 81, K_CPACK = 2161, K_QBOOL = 2241, K_QPACK = 4321, K_SLOT = 4401,
  K_CARRY = 4560, K_EM = 10880, K_TRANS = 10960, CONSTRAINTS = 11280,
  N_TRACE = 32, BLOWUP = 32, OUTPUT_ROW = 16
};
static_assert(WIDTH == 11041, "record width");
static_assert(K_CARRY + CARRY_BITS * CARRY_POS == K_EM, "constraint bases");
static constexpr uint64_t CARRY_OFFSET = 1ull << (CARRY_BITS - 1);

// Per-record constants and per-row witness: everything the 11,041 cells of a row
// are expanded from (bits are read out of the limbs and biased carries).
struct RecordW {
  uint32_t s[LIMBS], n[LIMBS], em[LIMBS];
};
struct RowW {
  uint32_t acc[LIMBS], op2[LIMBS], c[LIMBS], q[LIMBS];
  uint64_t carry[CARRY_POS];  // carry + 2^39
  uint32_t phase, pad;
};

// Cell `col` (< WIDTH) of one record row.
#if defined(__CUDACC__)
__host__ __device__
#endif
inline uint64_t cell(const RecordW& rc, const RowW& rw, uint32_t col) {
  if (col < S) return rw.acc[col];
  if (col < N) return rc.s[col - S];
  if (col < PHASE) return rc.n[col - N];
  if (col == PHASE) return rw.phase;
  if (col < EM) return rw.op2[col - OP2];
  if (col < C) return rc.em[col - EM];
  if (col < Q) return rw.c[col - C];
  if (col < Q_BITS) return rw.q[col - Q];
  if (col < C_BITS) return (rw.q[(col - Q_BITS) / LIMB_BITS] >> ((col - Q_BITS) % LIMB_BITS)) & 1u;
  if (col < CARRY) return (rw.c[(col - C_BITS) / LIMB_BITS] >> ((col - C_BITS) % LIMB_BITS)) & 1u;
  return (rw.carry[(col - CARRY) / CARRY_BITS] >> ((col - CARRY) % CARRY_BITS)) & 1u;
}

// EMSA-PKCS1-v1_5 encoding of SHA-256(msg) into k = 256 bytes (rsa2048.rs:71-90).
void em_encode(const uint8_t* msg, uint64_t len, uint8_t em[256]);
// s^65537 mod n == em (all 256-byte big-endian): the native check (rsa2048.rs:92-127).
bool verify_native(const uint8_t n_be[256], const uint8_t s_be[256], const uint8_t em_be[256]);
// fill_rsa_exp_multirow (rsa2048_exp_air.rs:126-204) as witnesses: throws SgError
// (SG_EINVAL) unless 1 < n, 0 <= s < n and em < 2^2048 (256 bytes each).
void witness(const uint8_t n_be[256], const uint8_t s_be[256], const uint8_t em_be[256], RecordW* rec,
             RowW rows[N_TRACE]);
// The column-major (n_records * WIDTH) x N_TRACE trace on the host.
void expand_host(const RecordW* recs, const RowW* rows, uint64_t n_records, uint64_t* trace);
// pi_hash recipes: prove_rsa2048_record_v1.rs:178-187 and stacked_rsa_zone_prover.rs:158-165.
void pi_record(const uint8_t n_be[256], const uint8_t s_be[256], const uint8_t* msg, uint64_t len,
               const uint8_t em[256], uint8_t out[32]);
void pi_stacked(const uint8_t n_be[256], uint64_t n_records, const uint8_t* ems, uint8_t out[32]);

}  // namespace rsa
}  // namespace sg

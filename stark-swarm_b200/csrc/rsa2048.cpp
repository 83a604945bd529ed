// rsa2048.cpp — host side of the RSA-2048 AIR: big-integer witness, EM encoding,
// pi_hash recipes, host trace expansion. Big integers are little-endian arrays of
// 32-bit words (bigint.hpp: schoolbook product, Knuth division).
#include "rsa2048.hpp"

#include <cstring>

#include "bigint.hpp"
#include "context.hpp"
#include "keccak.cuh"
#include "sha256_air.cuh"

namespace sg {
namespace rsa {
namespace {

constexpr int W = 64;  // 32-bit words of a 2048-bit value

void from_be(const uint8_t* b, uint32_t* w) {  // 256 bytes -> 64 words
  for (int i = 0; i < W; ++i) {
    const uint8_t* p = b + 256 - 4 * (i + 1);
    w[i] = (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3];
  }
}

// biguint_to_limbs80 (rsa2048_field_air.rs:190-210): 26-bit limbs, least significant first.
void limbs26(const uint32_t* w, int nw, uint32_t out[LIMBS]) {
  for (uint32_t i = 0; i < LIMBS; ++i) {
    const uint32_t bit = i * LIMB_BITS, wi = bit / 32, sh = bit % 32;
    uint64_t x = wi < (uint32_t)nw ? w[wi] : 0;
    if (wi + 1 < (uint32_t)nw) x |= (uint64_t)w[wi + 1] << 32;
    out[i] = (uint32_t)(x >> sh) & ((1u << LIMB_BITS) - 1);
  }
}

// c = a * b mod n, q = a * b / n as 26-bit limbs, with the biased carries of the
// slot identities (fill_rsa_mul_gadget, rsa2048_field_air.rs:241-326).
void mul_gadget(const uint32_t* a, const uint32_t* b, const uint32_t* n, int nn, RowW* row, uint32_t* c_words) {
  uint32_t prod[2 * W], qw[2 * W] = {0}, rw[W] = {0};
  bn::mul(a, W, b, W, prod);
  const int m = bn::top_word(prod, 2 * W) + 1;
  if (m < nn) {  // product below n: q = 0, c = product
    memcpy(rw, prod, 4 * (m > 0 ? m : 0));
  } else {
    bn::divmod(prod, m, n, nn, qw, rw);
  }
  memcpy(c_words, rw, 4 * W);
  uint32_t al[LIMBS], bl[LIMBS], nl[LIMBS];
  limbs26(a, W, al);
  limbs26(b, W, bl);
  limbs26(n, W, nl);
  limbs26(rw, W, row->c);
  limbs26(qw, 2 * W, row->q);
  memcpy(row->acc, al, sizeof al);
  memcpy(row->op2, bl, sizeof bl);
  // |slot sums| <= 80 * 2^52 each: i64 is exact (rsa2048_field_air.rs:266-276)
  int64_t carry = 0;
  for (uint32_t k = 0; k < SLOTS; ++k) {
    int64_t pab = 0, pqn = 0;
    const uint32_t lo = k >= LIMBS - 1 ? k - (LIMBS - 1) : 0, hi = k < LIMBS - 1 ? k : LIMBS - 1;
    for (uint32_t i = lo; i <= hi; ++i) {
      pab += (int64_t)al[i] * bl[k - i];
      pqn += (int64_t)row->q[i] * nl[k - i];
    }
    const int64_t lhs = pab - pqn - (k < LIMBS ? (int64_t)row->c[k] : 0) + carry;
    if (k + 1 < SLOTS) {
      if (lhs % (1ll << LIMB_BITS) != 0) throw SgError{SG_EINVAL, "rsa: carry chain residual"};
      carry = lhs >> LIMB_BITS;  // exact division (residual zero), floor for negatives
      if (carry <= -(int64_t)CARRY_OFFSET || carry >= (int64_t)CARRY_OFFSET)
        throw SgError{SG_EINVAL, "rsa: carry out of the biased range"};
      row->carry[k] = (uint64_t)(carry + (int64_t)CARRY_OFFSET);
    } else if (lhs != 0) {
      throw SgError{SG_EINVAL, "rsa: carry chain does not close"};
    }
  }
}

}  // namespace

void em_encode(const uint8_t* msg, uint64_t len, uint8_t em[256]) {
  static const uint8_t kDigestInfo[19] = {0x30, 0x31, 0x30, 0x0D, 0x06, 0x09, 0x60, 0x86, 0x48, 0x01,
                                          0x65, 0x03, 0x04, 0x02, 0x01, 0x05, 0x00, 0x04, 0x20};
  uint8_t dg[32];
  std::vector<sha::BlockWitness> w;
  sha256_witness(msg, len, &w, dg);
  const int t_len = 19 + 32, ps = 256 - t_len - 3;
  em[0] = 0x00;
  em[1] = 0x01;
  memset(em + 2, 0xFF, ps);
  em[2 + ps] = 0x00;
  memcpy(em + 3 + ps, kDigestInfo, 19);
  memcpy(em + 256 - 32, dg, 32);
}

void witness(const uint8_t n_be[256], const uint8_t s_be[256], const uint8_t em_be[256], RecordW* rec,
             RowW rows[N_TRACE]) {
  uint32_t n[W], s[W], em[W];
  from_be(n_be, n);
  from_be(s_be, s);
  from_be(em_be, em);
  const int nn = bn::top_word(n, W) + 1;
  require(nn >= 1 && !(nn == 1 && n[0] < 2), "rsa: modulus must be > 1");
  require(bn::cmp(s, n, W) < 0, "rsa: signature value must be below the modulus");
  limbs26(s, W, rec->s);
  limbs26(n, W, rec->n);
  limbs26(em, W, rec->em);
  uint32_t acc[W], c[W];
  memcpy(acc, s, sizeof acc);
  for (uint32_t r = 0; r < N_TRACE; ++r) {
    RowW& row = rows[r];
    memset(&row, 0, sizeof row);
    row.phase = r == OUTPUT_ROW;  // phase_for_row_e65537 (rsa2048_exp_air.rs:131-133)
    mul_gadget(acc, row.phase ? s : acc, n, nn, &row, c);
    memcpy(acc, c, sizeof acc);
  }
}

bool verify_native(const uint8_t n_be[256], const uint8_t s_be[256], const uint8_t em_be[256]) {
  uint32_t n[W], s[W], em[W];
  from_be(n_be, n);
  from_be(s_be, s);
  from_be(em_be, em);
  const int nn = bn::top_word(n, W) + 1;
  if (nn < 1 || (nn == 1 && n[0] < 2) || bn::cmp(s, n, W) >= 0) return false;
  if (bn::top_word(s, W) < 0) return false;  // rsa2048.rs:100-103 rejects s = 0
  RecordW rec;
  std::vector<RowW> rows(N_TRACE);
  witness(n_be, s_be, em_be, &rec, rows.data());
  // row 16's product is s^65537 mod n; compare its limbs with em's
  return memcmp(rows[OUTPUT_ROW].c, rec.em, sizeof rec.em) == 0;
}

void expand_host(const RecordW* recs, const RowW* rows, uint64_t n_records, uint64_t* trace) {
  for (uint64_t r = 0; r < n_records; ++r)
    for (uint32_t col = 0; col < WIDTH; ++col)
      for (uint32_t row = 0; row < N_TRACE; ++row)
        trace[(r * WIDTH + col) * N_TRACE + row] = cell(recs[r], rows[r * N_TRACE + row], col);
}

void pi_record(const uint8_t n_be[256], const uint8_t s_be[256], const uint8_t* msg, uint64_t len,
               const uint8_t em[256], uint8_t out[32]) {
  kc::Sha3 h;
  h.update("RSA2048-V2-PI-PRE", 17);
  h.update(n_be, 256);
  h.update(s_be, 256);
  h.update(msg, len);
  h.update(em, 256);
  h.finalize(out);
}

void pi_stacked(const uint8_t n_be[256], uint64_t n_records, const uint8_t* ems, uint8_t out[32]) {
  kc::Sha3 h;
  uint8_t le[8];
  for (int i = 0; i < 8; ++i) le[i] = (uint8_t)(n_records >> (8 * i));
  h.update("RSA2048-STACKED-ZONE", 20);
  h.update(n_be, 256);
  h.update(le, 8);
  h.update(ems, 256 * n_records);
  h.finalize(out);
}

}  // namespace rsa
}  // namespace sg

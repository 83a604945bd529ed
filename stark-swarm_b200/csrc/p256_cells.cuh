// p256_cells.cuh — value of one trace cell of the P-256 double-chain AIR from the
// row's witnesses (host trace expansion and the device kernel share it).
#pragma once
#include <cstdint>

#include "p256.hpp"

#if defined(__CUDACC__)
#define P256_HD __host__ __device__ __forceinline__
#else
#define P256_HD inline
#endif

namespace sg {
namespace p256 {

P256_HD uint64_t limb_bit(const uint32_t* l, uint32_t t) { return (l[t / LB] >> (t % LB)) & 1u; }

// code: gadget index << 11 | offset for gadget-owned cells, else category << 28 | payload
// (see Layout::cell_code); rproj: 6 x 10 limbs; b: the curve's b limbs.
P256_HD uint64_t cell_value(uint32_t code, const Gadget* table, const RowW& row, const GadgetW* gw,
                            const uint32_t* rproj, const uint32_t* b) {
  const uint32_t cat = code >> 28;
  if (cat == C_ACC) return row.acc[((code >> 4) & 0xFF) / 3][((code >> 4) & 0xFF) % 3][code & 15];
  if (cat == C_BASE) return row.base[((code >> 4) & 0xFF) / 3][((code >> 4) & 0xFF) % 3][code & 15];
  if (cat == C_BIT) return row.bit[code & 1];
  if (cat == C_RPROJ) return rproj[((code >> 4) & 0xFF) * NL + (code & 15)];
  if (cat == C_B) {
    const uint32_t o = code & 0xFFFF;
    return o < NL ? b[o] : limb_bit(b, o - NL);
  }
  const uint32_t gi = code >> 11, o = code & 2047;
  const GadgetW& w = gw[gi];
  switch (table[gi].kind) {
    case G_MUL:
      if (o < NL) return w.l0[o];
      if (o < ELEM) return limb_bit(w.l0, o - NL);
      if (o < ELEM + NL) return w.l1[o - ELEM];
      if (o < 2 * ELEM) return limb_bit(w.l1, o - ELEM - NL);
      {
        const uint32_t t = o - 2 * ELEM;
        const uint64_t biased = (uint64_t)(w.cy[t / MUL_CB] + (1ll << (MUL_CB - 1)));
        return (biased >> (t % MUL_CB)) & 1u;
      }
    case G_ADD:
      if (o < NL) return w.l0[o];
      if (o < ELEM) return limb_bit(w.l0, o - NL);
      return (uint64_t)w.cy[o - ELEM];
    case G_SUB:
      if (o < NL) return w.l0[o];
      if (o < ELEM) return limb_bit(w.l0, o - NL);
      if (o < ELEM + NL) return w.cy[o - ELEM] == 1;
      return w.cy[o - ELEM - NL] == -1;
    case G_FREEZE:
      if (o < NL) return w.l0[o];
      if (o < ELEM) return limb_bit(w.l0, o - NL);
      if (o < ELEM + NL) return w.l1[o - ELEM];
      if (o < 2 * ELEM) return limb_bit(w.l1, o - ELEM - NL);
      if (o < 2 * ELEM + NL) return w.cy[o - 2 * ELEM] == 1;
      return w.cy[o - 2 * ELEM - NL] == -1;
    default:  // G_SELECT
      return o < NL ? w.l0[o] : limb_bit(w.l0, o - NL);
  }
}

}  // namespace p256
}  // namespace sg

// p256_air.cuh — device side of the P-256 double-chain AIR (layout and constraint
// order in p256.hpp).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "p256.hpp"

namespace sg {

// Device copies of what the trace expansion reads.
struct P256Dev {
  const p256::Gadget* table;
  const uint32_t* cell_code;  // width entries
  const p256::RowW* rows;     // k rows
  const p256::GadgetW* gw;    // k * n_gadgets, row-major
  const uint32_t* rproj;      // 6 x 10 limbs
  const uint32_t* b;          // 10 limbs
  uint32_t width, n_gadgets;
};
// (width x k) column-major trace from the witnesses.
cudaError_t p256_expand(const P256Dev& d, uint64_t k, uint64_t* d_trace, cudaStream_t s);

struct P256Phi {
  const uint64_t* lde;  // width columns of n points
  uint64_t n, blowup, n_trace;
  // coset_len = 0: `lde` is the materialised LDE; point i is trace row i / blowup,
  // its next row is point (i + blowup) mod n, and Phi goes to d_phi[i].
  // coset_len = L > 0: `lde` holds n / L whole cosets of the LDE one after
  // another (coset out_off + c at c L .. c L + L - 1, point a = LDE point
  // out_off + c + out_stride a): point i = c L + a is trace row a, its next row is
  // point c L + (a + 1) mod L, and Phi goes to d_phi[out_off + c + out_stride a].
  uint64_t coset_len, out_stride, out_off;
  const p256::Gadget* table;
  const uint32_t* lam_base;  // first constraint index of each gadget
  const uint32_t* chunk;     // n_chunks + 1 gadget boundaries
  const uint32_t* tail;      // 18 bases
  uint32_t n_gadgets, lam_tail;
};
// Gadget boundaries splitting the row into chunks of about `target` constraints.
std::vector<uint32_t> p256_chunks(uint32_t target);
// Phi at the n LDE points; d_part holds n_chunks * n values.
cudaError_t p256_phi(const P256Phi& a, uint32_t n_chunks, uint64_t* d_part, uint64_t* d_phi, cudaStream_t s);

}  // namespace sg

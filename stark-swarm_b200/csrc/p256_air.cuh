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
  // Point i of the buffer is trace row i / row_div; the next row's point is
  // (i + step) mod n. A materialised LDE has row_div = step = blowup; one coset
  // of it (point a = LDE point r + blowup a) has row_div = step = 1.
  uint64_t row_div, step;
  // Phi of point i goes to d_phi[i * out_stride + out_off] (1, 0 for an LDE; blowup, r for coset r)
  uint64_t out_stride, out_off;
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

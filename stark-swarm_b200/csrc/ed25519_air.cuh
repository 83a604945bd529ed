// ed25519_air.cuh — device side of the Ed25519 verify AIR (layout, program and
// witness in ed25519.hpp).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "ed25519.hpp"

namespace sg {

// What the trace expansion reads (device pointers).
struct EdExpand {
  const uint32_t* codes;      // N_PHASES x width
  const uint8_t* row_phase;   // height
  const uint32_t* row_off;    // height + 1
  const uint64_t* words;
  const uint64_t* globals;
  uint32_t width, height;
};
// Every cell not on a SHA-512 row (rows < k_hash, columns < 1510 are left to
// sha512_expand_strided) of the width x height column-major trace.
cudaError_t ed25519_expand(const EdExpand& d, uint64_t* d_trace, cudaStream_t s);

// The LDE values the merge reads in the columns an LdePlan does not transform
// (device pointers): Lagrange basis values L_r at the points of read rows
// (ar: read row a and non-zero row r per pair), sparse tasks (5 u32 each: column,
// read row, first pair, offset into nz_rows, number of non-zero rows) and the
// constant columns. The trace is width x height column-major, the LDE width x n0.
struct EdLdeFill {
  const uint32_t* ar;
  uint32_t n_pairs;
  const uint32_t* tasks;
  uint32_t n_tasks;
  const uint32_t* nz_rows;
  const uint32_t* const_cols;
  uint32_t n_const;
};
cudaError_t ed25519_lde_fill(const EdLdeFill& f, const uint64_t* d_trace, uint64_t height, uint64_t blowup,
                             uint64_t* d_lval, uint64_t* d_lde, cudaStream_t s);

// A block of the constraint program on the device: kind, index of its first
// constraint, cell bases (B_PAIRS: first pair, count).
struct EdBlock {
  uint32_t kind, lam, p[8];
};
// The program split for the Phi kernel: rows with the same open blocks form a
// class; a class's open blocks (SHA-512 excluded) are cut into chunks of about
// equal constraint count, one chunk per grid.y slice.
struct EdPhiPlan {
  std::vector<EdBlock> blocks;
  std::vector<uint32_t> cls_list;   // block indices, class by class
  std::vector<uint32_t> chunk_rng;  // per chunk: [first, last) into cls_list
  std::vector<uint32_t> cls_chunk;  // per class: first chunk; n_classes + 1 entries
  std::vector<uint8_t> row_class;   // n_trace
  uint32_t max_chunks = 0;
};
EdPhiPlan ed25519_phi_plan(const ed25519::Program& prog, uint32_t n_trace, uint32_t chunk_constraints);

struct EdPhi {
  const uint64_t* lde;  // width columns of n points (column stride n)
  uint64_t n, blowup, n_trace;
  // coset_len = 0: point i is trace row i / blowup, next row (i + blowup) mod n, Phi to
  // d_phi[i]; coset_len = L: `lde` holds n / L cosets one after another, point c L + a
  // is row a of coset out_off + c, next row c L + (a + 1) mod L, Phi to d_phi[out_off + c + out_stride a].
  uint64_t coset_len, out_stride, out_off;
  const EdBlock* blocks;
  const uint64_t* pairs;
  const uint32_t* cls_list;
  const uint32_t* chunk_rng;
  const uint32_t* cls_chunk;
  const uint8_t* row_class;
  const uint64_t* phi_sha;  // the SHA-512 block's Phi at points whose row is below sha_rows
  uint64_t sha_rows;
  uint32_t max_chunks;
};
// Phi = sum_j (j + 1) C_j at the n points; d_part holds max_chunks * n values.
cudaError_t ed25519_phi(const EdPhi& a, uint64_t* d_part, uint64_t* d_phi, cudaStream_t s);
// The same in its two launches: the block kernel's per-chunk partial sums into
// d_part, then their sum (with the SHA-512 part, a.phi_sha, for the hash rows).
cudaError_t ed25519_phi_blocks(const EdPhi& a, uint64_t* d_part, cudaStream_t s);
cudaError_t ed25519_phi_add(const EdPhi& a, const uint64_t* d_part, uint64_t* d_phi, cudaStream_t s);

}  // namespace sg

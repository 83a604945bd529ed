// sha256_air.cuh — SHA-256 AIR layout (deep_ali/src/sha256_air.rs:140-248, 756 columns).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace sg {
namespace sha {

enum : uint32_t {
  A_a = 0, A_b, A_c, A_d, A_e, A_f, A_g, A_h,
  BIT_A = 8, BIT_B = 40, BIT_C = 72, BIT_E = 104, BIT_F = 136, BIT_G = 168,
  S0_T = 200, S0_BIT = 232, S0_W = 264,
  S1_T = 265, S1_BIT = 297, S1_W = 329,
  CH_BIT = 330, CH_W = 362,
  MAJ_AB = 363, MAJ_AC = 395, MAJ_BC = 427, MAJ_U = 459, MAJ_BIT = 491, MAJ_W = 523,
  W_ = 524,
  T1_LO = 525, T1_C0 = 526, T1_C1 = 527, T1_C2 = 528, T1_CW = 529,
  T2_LO = 530, T2_C0 = 531, T2_C1 = 532, T2_CW = 533,
  H0 = 534,
  WW0 = 542,
  BIT_WW14 = 557, BIT_WW1 = 589,
  SS0_T = 621, SS0_BIT = 653, SS0_W = 685,
  SS1_T = 686, SS1_BIT = 718, SS1_W = 750,
  WS_C0 = 751, WS_C1 = 752, WS_CW = 753,
  NA_C = 754, NE_C = 755,
  WIDTH = 756, NUM_CONSTRAINTS = 766, ROWS_PER_BLOCK = 128
};

// One compression of the trace: message schedule, the working state before each
// of the 64 rounds plus the post-compression state, and the chaining value in.
struct BlockWitness {
  uint32_t w[64];
  uint32_t st[65][8];
  uint32_t iv[8];
};

}  // namespace sha

// FIPS 180-4 padding and the compressions of msg: one witness per block, the
// digest, and the trace height (128 rows per block, next power of two).
uint64_t sha256_witness(const uint8_t* msg, uint64_t len, std::vector<sha::BlockWitness>* wit, uint8_t digest[32]);
uint64_t sha256_height(uint64_t n_blocks);
// Expands block witnesses into the 756 x h column-major trace on the host (threads).
void sha256_fill_host(const sha::BlockWitness* wit, uint64_t n_blocks, uint64_t h, uint64_t* out);
// The same expansion on the device: d_wit (n_blocks witnesses) -> d_trace (756 x h).
cudaError_t sha256_expand(const sha::BlockWitness* d_wit, uint64_t n_blocks, uint64_t h, uint64_t* d_trace,
                          cudaStream_t s);

// Host: build_sha256_trace_multi (sha256_air.rs:429-472) into a column-major
// WIDTH x height buffer (resized); returns height and sets n_blocks. The
// asserted digest is read from the H-state at row 128 (n_blocks - 1) + 65.
uint64_t sha256_build_trace(const uint8_t* msg, uint64_t len, std::vector<uint64_t>* trace, uint64_t* n_blocks,
                            uint8_t digest[32]);

// Phi = sum_j lambda_j C_j for the SHA-256 AIR (eval_sha256_constraints,
// sha256_air.rs:956-1294) at the points of an evaluation buffer: evals holds
// WIDTH columns of n points; point i pairs with point (i + step) mod n, has trace
// row i / row_div, and its value goes to phi[out_off + i * out_stride]. The whole
// LDE is (step, row_div, out_stride, out_off) = (blowup, blowup, 1, 0); one coset
// r of it (points r + blowup a) is (1, 1, blowup, r). lambdas are on the device.
cudaError_t sha256_phi_points(const uint64_t* evals, uint64_t n, uint64_t step, uint64_t row_div, uint64_t n_blocks,
                              const uint64_t* lambdas, uint64_t* phi, uint64_t out_stride, uint64_t out_off,
                              cudaStream_t s);

}  // namespace sg

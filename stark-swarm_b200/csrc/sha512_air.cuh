// sha512_air.cuh — SHA-512 AIR (deep_ali/src/sha512_air.rs): 1510 columns, 1526
// constraints; every 64-bit word is held as two 32-bit limbs.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace sg {
namespace sha512 {

// Column layout (sha512_air.rs:313-471). Word k of {a..h} is at A_LO + 2k (lo)
// and A_LO + 2k + 1 (hi); H_k at H0_LO + 2k, W_win[k] at WW0_LO + 2k.
enum : uint32_t {
  A_LO = 0,
  BIT_A = 16, BIT_B = 80, BIT_C = 144, BIT_E = 208, BIT_F = 272, BIT_G = 336,
  S0_T = 400, S0_BIT = 464, S0_LO = 528, S0_HI = 529,
  S1_T = 530, S1_BIT = 594, S1_LO = 658, S1_HI = 659,
  CH_BIT = 660, CH_LO = 724, CH_HI = 725,
  MAJ_AB = 726, MAJ_AC = 790, MAJ_BC = 854, MAJ_U = 918, MAJ_BIT = 982, MAJ_LO = 1046, MAJ_HI = 1047,
  W_LO = 1048, W_HI = 1049,
  T1_LO_LO = 1050, T1_LO_C0 = 1051, T1_LO_C1 = 1052, T1_LO_C2 = 1053, T1_LO_CW = 1054,
  T1_HI_LO = 1055, T1_HI_C0 = 1056, T1_HI_C1 = 1057, T1_HI_C2 = 1058, T1_HI_CW = 1059,
  T2_LO_LO = 1060, T2_LO_C0 = 1061, T2_LO_CW = 1062, T2_HI_LO = 1063, T2_HI_C0 = 1064, T2_HI_CW = 1065,
  H0_LO = 1066,
  WW0_LO = 1082,
  BIT_WW14 = 1112, BIT_WW1 = 1176,
  SS0_T = 1240, SS0_BIT = 1304, SS0_LO = 1368, SS0_HI = 1369,
  SS1_T = 1370, SS1_BIT = 1434, SS1_LO = 1498, SS1_HI = 1499,
  WS_LO_C0 = 1500, WS_LO_C1 = 1501, WS_LO_CW = 1502, WS_HI_C0 = 1503, WS_HI_C1 = 1504, WS_HI_CW = 1505,
  NA_LO_C = 1506, NA_HI_C = 1507, NE_LO_C = 1508, NE_HI_C = 1509,
  WIDTH = 1510, NUM_CONSTRAINTS = 1526, ROWS_PER_BLOCK = 128, ROUNDS = 80
};

// One compression: message schedule, the working state before each of the 80
// rounds plus the post-compression state, and the chaining value in.
struct BlockWitness {
  uint64_t w[80];
  uint64_t st[81][8];
  uint64_t iv[8];
};

}  // namespace sha512

// FIPS 180-4 §5.1.2 padding and the compressions: one witness per block, the
// 64-byte digest, and the trace height (128 rows per block, next power of two).
uint64_t sha512_witness(const uint8_t* msg, uint64_t len, std::vector<sha512::BlockWitness>* wit,
                        uint8_t digest[64]);
// Expands block witnesses into the 1510 x h column-major trace on the host (threads).
void sha512_fill_host(const sha512::BlockWitness* wit, uint64_t n_blocks, uint64_t h, uint64_t* out);
// The same expansion on the device.
cudaError_t sha512_expand(const sha512::BlockWitness* d_wit, uint64_t n_blocks, uint64_t h, uint64_t* d_trace,
                          cudaStream_t s);
// The h rows into a wider trace whose columns are `stride` rows apart.
cudaError_t sha512_expand_strided(const sha512::BlockWitness* d_wit, uint64_t n_blocks, uint64_t h, uint64_t stride,
                                  uint64_t* d_trace, cudaStream_t s);
// Phi at the points of a column-major evaluation buffer (n points per column):
// cur = point i, nxt = point (i + step) mod n, trace row i / row_div; result to
// phi[out_off + i * out_stride] (eval_sha512_constraints, sha512_air.rs:909-1270).
cudaError_t sha512_phi_points(const uint64_t* evals, uint64_t n, uint64_t step, uint64_t row_div, uint64_t n_blocks,
                              const uint64_t* lambdas, uint64_t* phi, uint64_t out_stride, uint64_t out_off,
                              cudaStream_t s);
// The same for points 0 .. count-1 only, with cell col of point i at evals[col * stride + i]
// (the next row is still point (i + step) mod n): the SHA-512 rows at the top of a wider AIR.
cudaError_t sha512_phi_points_ex(const uint64_t* evals, uint64_t n, uint64_t stride, uint64_t count, uint64_t step,
                                 uint64_t row_div, uint64_t n_blocks, const uint64_t* lambdas, uint64_t* phi,
                                 uint64_t out_stride, uint64_t out_off, cudaStream_t s);
// The first `rows` rows of each of n_cosets cosets held one after another (coset c's
// point a at evals[col * n_cosets * coset_len + c * coset_len + a], its next row
// point (a + 1) mod coset_len), in one launch; Phi of that point to phi[c coset_len + a].
cudaError_t sha512_phi_cosets(const uint64_t* evals, uint64_t n_cosets, uint64_t coset_len, uint64_t rows,
                              uint64_t n_blocks, const uint64_t* lambdas, uint64_t* phi, cudaStream_t s);

}  // namespace sg

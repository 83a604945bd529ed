// hash_air.hpp — the two hash AIRs (SHA-256: deep_ali/src/sha256_air.rs, SHA-512:
// deep_ali/src/sha512_air.rs) as one descriptor, so the merge (materialised LDE or
// coset-sliced) and the proof pipeline are written once.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace sg {

struct HashAir {
  const char* name;
  uint32_t width, num_constraints, digest_bytes;
  // host: padding + compressions -> per-block witnesses (opaque bytes), trace height
  uint64_t (*witness)(const uint8_t* msg, uint64_t len, std::vector<uint8_t>* blob, uint64_t* n_blocks,
                      uint8_t* digest);
  // device: witnesses -> width x h column-major trace
  cudaError_t (*expand)(const void* d_wit, uint64_t n_blocks, uint64_t h, uint64_t* d_trace, cudaStream_t s);
  // device: Phi at the points of an evaluation buffer (see sha256_phi_points)
  cudaError_t (*phi_points)(const uint64_t* evals, uint64_t n, uint64_t step, uint64_t row_div, uint64_t n_blocks,
                            const uint64_t* lambdas, uint64_t* phi, uint64_t out_stride, uint64_t out_off,
                            cudaStream_t s);
};

const HashAir& sha256_hash_air();
const HashAir& sha512_hash_air();

}  // namespace sg

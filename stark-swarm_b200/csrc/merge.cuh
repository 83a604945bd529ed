// merge.cuh — DEEP-ALI composition (deep_ali/src/lib.rs:190-545).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace sg {

enum AirId : int { kAirHashRollup = 4, kAirSha256 = 6 };

// Phi(w^i) = sum_j lambda_j C_j(cur = row i, nxt = row (i + blowup) mod n) for the
// HashRollup AIR (air_workloads.rs:591-599) over a column-major 4 x n LDE.
cudaError_t hash_rollup_phi(const uint64_t* lde, uint64_t n, uint64_t blowup, const uint64_t* lambdas,
                            uint64_t* phi, cudaStream_t s);

// poly_div_zh (lib.rs:190-228) on coefficients d[0..n): q[k] = sum_{t>=1} d[k + t m]
// for k < n - m, zero for k >= n - m (the remainder below m is dropped).
cudaError_t quotient_zh(const uint64_t* d, uint64_t n, uint64_t m, uint64_t* q, cudaStream_t s);

}  // namespace sg

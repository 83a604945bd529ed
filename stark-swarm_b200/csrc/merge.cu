// merge.cu — constraint evaluation, lambda-combination and division by X^m - 1.
#include "gl.cuh"
#include "merge.cuh"
#include "counters.hpp"

namespace sg {
namespace {

__global__ void hash_rollup_phi_kernel(const uint64_t* __restrict__ lde, uint64_t n, uint64_t blowup,
                                       uint64_t l0, uint64_t l1, uint64_t l2, uint64_t* __restrict__ phi) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t j = (i + blowup) & (n - 1);
  const uint64_t idx = lde[i], leaf = lde[n + i], st = lde[2 * n + i], sq = lde[3 * n + i];
  const uint64_t idx_n = lde[j], st_n = lde[2 * n + j];
  // C0 = idx' - idx - 1 ; C1 = sq - st^2 ; C2 = st' - sq - leaf
  const uint64_t c0 = gl::sub(gl::sub(idx_n, idx), 1);
  const uint64_t c1 = gl::sub(sq, gl::mul(st, st));
  const uint64_t c2 = gl::sub(gl::sub(st_n, sq), leaf);
  phi[i] = gl::add(gl::add(gl::mul(l0, c0), gl::mul(l1, c1)), gl::mul(l2, c2));
}

// One thread per residue r < m walks its class from the top: q[r + (t-1)m] =
// d[r + tm] + q[r + tm]; consecutive threads touch consecutive addresses.
__global__ void quotient_kernel(const uint64_t* __restrict__ d, uint64_t n, uint64_t m, uint64_t* __restrict__ q) {
  const uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (r >= m) return;
  const uint64_t B = n / m;
  uint64_t acc = 0;
  q[r + (B - 1) * m] = 0;
  for (uint64_t t = B - 1; t >= 1; --t) {
    acc = gl::add(acc, d[r + t * m]);
    q[r + (t - 1) * m] = acc;
  }
}

}  // namespace

cudaError_t hash_rollup_phi(const uint64_t* lde, uint64_t n, uint64_t blowup, const uint64_t* lambdas,
                            uint64_t* phi, cudaStream_t s) {
  const unsigned T = 256;
  SG_LAUNCH_SCOPE("merge_phi", s);
  hash_rollup_phi_kernel<<<(unsigned)((n + T - 1) / T), T, 0, s>>>(lde, n, blowup, lambdas[0] % gl::P,
                                                                    lambdas[1] % gl::P, lambdas[2] % gl::P, phi);
  return cudaGetLastError();
}

cudaError_t quotient_zh(const uint64_t* d, uint64_t n, uint64_t m, uint64_t* q, cudaStream_t s) {
  if (n <= m) return cudaMemsetAsync(q, 0, n * sizeof(uint64_t), s);
  if (n % m) return cudaErrorInvalidValue;
  const unsigned T = 256;
  SG_LAUNCH_SCOPE("merge_quotient", s);
  quotient_kernel<<<(unsigned)((m + T - 1) / T), T, 0, s>>>(d, n, m, q);
  return cudaGetLastError();
}

}  // namespace sg

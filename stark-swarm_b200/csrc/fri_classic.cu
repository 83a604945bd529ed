// fri_classic.cu — device kernels of the classic DEEP-FRI branch (stir = false,
// deep_ali/src/fri.rs:1398-1807): the DEEP quotient layer and the per-layer leaf
// matrix of (f, s, q).
#include "counters.hpp"
#include "fri_classic.cuh"
#include "ntt.cuh"

namespace sg {
namespace {

constexpr int kPointsPerThread = 4;

// compute_q_layer_ext_on_ext (fri.rs:255-336): q_i = (f_i - f(z)) / (w^i - z).
// Each thread takes 4 consecutive points and inverts the product of their
// denominators once (Montgomery's trick: prefix products, one inverse, then
// back-substitution).
__global__ void __launch_bounds__(128) deep_q_kernel(const uint64_t* __restrict__ f, bool base, uint64_t n,
                                                     int log_n, const uint64_t* __restrict__ tw_lo,
                                                     const uint64_t* __restrict__ tw_hi, gl::Fp6 z, gl::Fp6 fz,
                                                     uint64_t* __restrict__ q) {
  const uint64_t i0 = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) * kPointsPerThread;
  if (i0 >= n) return;
  const int cnt = (int)(n - i0 < kPointsPerThread ? n - i0 : kPointsPerThread);
  const uint64_t w = tw_pow(tw_lo, tw_hi, 1, log_n);
  uint64_t xs[kPointsPerThread];
  gl::Fp6 pre[kPointsPerThread];
  gl::Fp6 acc = gl::e_one();
  uint64_t x = tw_pow(tw_lo, tw_hi, i0, log_n);
  auto denom = [&](uint64_t xv) {  // w^i - z
    gl::Fp6 d;
    d.c[0] = gl::sub(xv, z.c[0]);
#pragma unroll
    for (int k = 1; k < 6; ++k) d.c[k] = gl::sub(0, z.c[k]);
    return d;
  };
#pragma unroll
  for (int j = 0; j < kPointsPerThread; ++j) {
    if (j < cnt) {
      xs[j] = x;
      pre[j] = acc;
      acc = gl::e_mul(acc, denom(x));
      x = gl::mul(x, w);
    }
  }
  gl::Fp6 inv;
  if (!gl::e_inv(acc, &inv)) inv = gl::e_zero();  // z on the domain: probability ~ n / p^6
#pragma unroll
  for (int j = kPointsPerThread - 1; j >= 0; --j) {
    if (j < cnt) {
      const uint64_t i = i0 + j;
      const gl::Fp6 dinv = gl::e_mul(inv, pre[j]);
      inv = gl::e_mul(inv, denom(xs[j]));
      gl::Fp6 fi;
      if (base) {
        fi = gl::e_from(f[i]);
      } else {
#pragma unroll
        for (int k = 0; k < 6; ++k) fi.c[k] = f[(uint64_t)k * n + i];
      }
      const gl::Fp6 qi = gl::e_mul(gl::e_sub(fi, fz), dinv);
#pragma unroll
      for (int k = 0; k < 6; ++k) q[(uint64_t)k * n + i] = qi.c[k];
    }
  }
}

// Rows 0..11 of the 18 x n leaf matrix (ext_leaf_fields, fri.rs:1356-1362): the
// six components of f and of s, where s_i = next[i mod n/m] (compute_s_layer_from_coeffs,
// fri.rs:773-789) or zero on the coefficient-committed last layer.
__global__ void fill_leaf_rows_kernel(const uint64_t* __restrict__ f, bool base, const uint64_t* __restrict__ next,
                                      uint64_t nn, uint64_t n, uint64_t* __restrict__ mat) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    mat[(uint64_t)k * n + i] = base ? (k == 0 ? f[i] : 0) : f[(uint64_t)k * n + i];
    mat[(uint64_t)(6 + k) * n + i] = next ? next[(uint64_t)k * nn + i % nn] : 0;
  }
}

}  // namespace

cudaError_t deep_quotient(const uint64_t* f, bool base, uint64_t n, int log_n, const uint64_t* tw_lo,
                          const uint64_t* tw_hi, const gl::Fp6& z, const gl::Fp6& fz, uint64_t* q, cudaStream_t s) {
  const uint64_t threads = (n + kPointsPerThread - 1) / kPointsPerThread;
  SG_LAUNCH_SCOPE("fri_deep_q", s);
  deep_q_kernel<<<(unsigned)((threads + 127) / 128), 128, 0, s>>>(f, base, n, log_n, tw_lo, tw_hi, z, fz, q);
  return cudaGetLastError();
}

cudaError_t fill_leaf_rows(const uint64_t* f, bool base, const uint64_t* next, uint64_t nn, uint64_t n,
                           uint64_t* mat, cudaStream_t s) {
  SG_LAUNCH_SCOPE("fri_leaf_rows", s);
  fill_leaf_rows_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(f, base, next, nn, n, mat);
  return cudaGetLastError();
}

}  // namespace sg

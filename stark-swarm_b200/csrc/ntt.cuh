// ntt.cuh — batched Goldilocks NTT/iNTT over column-major data.
//
// Semantics match ark-poly's Radix2EvaluationDomain (the reference calls it
// directly: trace_import.rs:272-280, lib.rs:400-410, fri.rs:273-282):
// forward = evaluations at w^0..w^{N-1} in natural order, inverse includes 1/N,
// w = root_of_unity(log2 N).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace sg {

struct NttTables {
  // w24 = primitive 2^24-th root; lo[i] = w24^i, hi[i] = w24^(4096 i), i < 4096,
  // and the same for w24^-1. Any w_N^e with N <= 2^24 is lo[E & 4095] * hi[E >> 12]
  // with E = e * 2^(24 - log N) mod 2^24.
  uint64_t* d_fwd_lo = nullptr;
  uint64_t* d_fwd_hi = nullptr;
  uint64_t* d_inv_lo = nullptr;
  uint64_t* d_inv_hi = nullptr;
};

static constexpr int kMaxLogN = 24;

cudaError_t ntt_tables_init(NttTables* t);
void ntt_tables_free(NttTables* t);

// Transform `n_cols` columns of length 2^log_n. Column c of the input starts at
// in + c*in_stride, of the output at out + c*out_stride. Input entries at index
// >= n_valid are treated as zero (zero-padded forward transform). `scratch`
// must hold n_cols * 2^log_n elements when log_n > 12 (two-pass transform);
// in == out is allowed. Returns cudaSuccess or the launch error.
cudaError_t ntt_batch(const NttTables& t, const uint64_t* in, uint64_t* out, uint32_t n_cols, uint64_t in_stride,
                      uint64_t out_stride, int log_n, bool inverse, uint64_t n_valid, uint64_t* scratch,
                      cudaStream_t s);

// out[c*stride + k] = in[c*stride + k] * g^k for k < n (coset scaling of coefficients).
cudaError_t scale_by_powers(const uint64_t* in, uint64_t* out, uint32_t n_cols, uint64_t stride, uint64_t n,
                            uint64_t g, cudaStream_t s);

}  // namespace sg

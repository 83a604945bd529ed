// fri_classic.cuh — device kernels of the classic DEEP-FRI branch (stir = false).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "gl.cuh"

namespace sg {

// q planes (6 x n) of compute_q_layer_ext_on_ext (fri.rs:255-336):
// q_i = (f_i - fz) / (w_n^i - z); f is one base column (base) or 6 planes.
// tw_lo / tw_hi: the forward two-level w28 tables.
cudaError_t deep_quotient(const uint64_t* f, bool base, uint64_t n, int log_n, const uint64_t* tw_lo,
                          const uint64_t* tw_hi, const gl::Fp6& z, const gl::Fp6& fz, uint64_t* q, cudaStream_t s);
// Rows 0..11 of a layer's 18 x n leaf matrix: f, then s_i = next[i mod nn]
// (next = NULL: s = 0).
cudaError_t fill_leaf_rows(const uint64_t* f, bool base, const uint64_t* next, uint64_t nn, uint64_t n,
                           uint64_t* mat, cudaStream_t s);

}  // namespace sg

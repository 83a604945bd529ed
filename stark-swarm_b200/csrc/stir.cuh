// stir.cuh — STIR layer kernels (deep_ali/src/fri.rs, STIR branch).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "gl.cuh"

namespace sg {

// Out-of-domain coset evaluation (fri.rs:338-391 evaluate_ood_coset):
// given the monomial coefficients c_k of f_l (1 plane when the layer is the
// base-field f0, else 6 component planes of length n), compute
//   evals[j] = f_l(zeta^j z), j < m,  zeta = w_n^{n/m} = w_m.
// Because zeta^m = 1: f(zeta^j z) = sum_r zeta^{jr} z^r T_r with
// T_r = sum_t c_{tm+r} (z^m)^t, so one pass over the coefficients suffices.
// `partials` needs ood_partials_len(n, m) u64; evals receives m*6 u64.
uint64_t ood_partials_len(uint64_t n, int m);
cudaError_t ood_evaluate(const uint64_t* coeffs, bool base, uint64_t n, int m, const gl::Fp6& z,
                         uint64_t* partials, uint64_t* evals, cudaStream_t s);

// Coset-interpolation fold (fri.rs:670-771): for every coset b < n/m with
// fibre f[b + j n/m], coefficients coeff_k = (1/m) DFT_{zeta^-1}(fibre)_k * w_n^{-bk}
// and next[b] = sum_k coeff_k alpha^k.
//   f: 1 plane (base) or 6 planes (stride n); next: 6 planes (stride n/m) or null;
//   tuples: if non-null, 6m planes (plane k*6+c, stride n/m) receive coeff_k;
//   leaves: if non-null, leaf digest of next[b] for a tree (label, arity0).
struct FoldArgs {
  const uint64_t* f;
  bool base;
  uint64_t n;
  int log_n;
  int m;
  gl::Fp6 alpha;
  uint64_t* next;
  uint64_t* tuples;
  uint64_t* leaves;
  uint64_t leaf_label;
  uint64_t leaf_arity0;
  const uint64_t* tw_inv_lo;
  const uint64_t* tw_inv_hi;
  // Several proofs of one shape in one launch (grid.y = proof g): each pointer
  // above advances by its g_* stride (u64 elements) per proof, and the fold
  // challenge is alphas[g] (device memory) when alphas is set. The defaults
  // describe one proof.
  uint32_t n_proofs = 1;
  uint64_t g_f = 0, g_next = 0, g_tuples = 0, g_leaves = 0;
  const gl::Fp6* alphas = nullptr;
};
cudaError_t stir_fold(const FoldArgs& a, cudaStream_t s);

// next[b] = sum_k tuple_k alpha^k over n_final tuples of m (planes as above).
cudaError_t fold_tuples(const uint64_t* tuples, uint64_t n_final, int m, const gl::Fp6& alpha, uint64_t* next,
                        cudaStream_t s);

// The same for n_proofs proofs of one shape (tuples and next advance by g_tup /
// g_next per proof; alpha of proof g = alphas[g], device memory).
cudaError_t fold_tuples_group(const uint64_t* tuples, uint64_t g_tup, uint64_t n_final, int m,
                              const gl::Fp6* alphas, uint64_t* next, uint64_t g_next, uint32_t n_proofs,
                              cudaStream_t s);

// Out-of-domain evaluation of n_proofs proofs of one shape in one launch set:
// proof g's coefficients at coeffs + g g_c, its evaluations at evals + g g_e,
// its point and the powers the kernels use in sc[g] (device memory, filled
// from ood_scalars). partials: n_proofs * ood_partials_len(n, m).
// Beside z and w = z^m, the powers the kernels read instead of forming them by
// chains of Fp6 products (a dependent Fp6 product costs microseconds on one
// thread): z^r (r < m); a thread's factor w^t (t < 256) = lo[t & 15] mid[t >> 4];
// a partial-pass block's factor w^(256 b) = blo[b & 15] bmid[(b >> 4) & 15]
// (b < 256), times w65536^(b >> 8) beyond.
struct OodScalars {
  gl::Fp6 z, w, w32, ws;  // z, w = z^m, w^32, w^(threads of the partial pass)
  gl::Fp6 w65536;
  gl::Fp6 zr[16], lo[16], mid[16], blo[16], bmid[16];
};
OodScalars ood_scalars(const gl::Fp6& z, uint64_t n, int m);
cudaError_t ood_evaluate_group(const uint64_t* coeffs, uint64_t g_c, bool base, uint64_t n, int m,
                               const OodScalars* sc, uint64_t* partials, uint64_t* evals, uint64_t g_e,
                               uint32_t n_proofs, cudaStream_t s);

}  // namespace sg

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

static constexpr int kMaxLogN = 28;     // largest transform (three passes above 2^24)
static constexpr int kTwBaseLog = 28;   // global twiddles are powers of w28 = w_{2^28}
static constexpr int kTwSplit = 14;     // w28^E = lo[E & (2^14-1)] * hi[E >> 14]
static constexpr int kTwEntries = 1 << kTwSplit;

struct NttTables {
  // Per direction (forward: w, inverse: w^-1):
  //   st[i] = w_4096^i (i < 4096)       — in-CTA Stockham stage twiddles
  //   lo[i] = w28^i, hi[i] = w28^(2^14 i) (i < 2^14) — any w_N^e, N <= 2^28
  uint64_t* d_fwd_st = nullptr;
  uint64_t* d_fwd_lo = nullptr;
  uint64_t* d_fwd_hi = nullptr;
  uint64_t* d_inv_st = nullptr;
  uint64_t* d_inv_lo = nullptr;
  uint64_t* d_inv_hi = nullptr;
  bool owned = false;
  // Two-pass transforms may read their pass twiddles w_N^{i k} from a per-size
  // table kept for the process (pass_twiddle_table); off for tables made by
  // ntt_tables_view (callers that must not allocate).
  bool pass_tables = false;
};

// Elements of one direction's block: st (4096) + lo + hi.
static constexpr uint64_t kTwDirElems = 4096 + 2 * kTwEntries;

// Host: fill `out` (2 * kTwDirElems u64: forward block, then inverse block).
void ntt_tables_host(uint64_t* out);
// Point a table struct at a device copy of ntt_tables_host's layout.
NttTables ntt_tables_view(uint64_t* dev);
cudaError_t ntt_tables_init(NttTables* t);
void ntt_tables_free(NttTables* t);

// Element-wise powers x[k] *= g^k (k = natural index inside the column), applied
// to the input by the transform itself as pass 1 loads it. g^k = lo[E & (2^14-1)] * hi[E >> 14] with
// E = ((k * mult) << shl) mod 2^28:
//   g = w_{2^L}^r, a root of unity: the w28 tables of NttTables, mult = r, shl = 28 - L;
//   any other g (the LDE shift): pow_tables_host(g), mult = 1, shl = 0, k < 2^28.
struct PowSpec {
  const uint64_t* lo = nullptr;
  const uint64_t* hi = nullptr;
  uint64_t mult = 1;
  int shl = 0;
  // instead of lo/hi: g^k read from a full table (k below its length)
  const uint64_t* tab = nullptr;
  __host__ __device__ bool active() const { return lo || tab; }
};
// Host: tab[k] = w_{2^log_n}^(mult k) for k < len on the device (the NttTables'
// forward direction), e.g. a coset twist applied by a transform's first pass.
cudaError_t pow_table_device(const NttTables& t, uint64_t mult, int log_n, uint64_t len, uint64_t* tab,
                             cudaStream_t s);
// Host: lo[i] = scale * g^i, hi[i] = g^(2^14 i) for i < 2^14 (out: 2 * 2^14 u64).
void pow_tables_host(uint64_t g, uint64_t scale, uint64_t* out);

// The four-step split ntt_batch uses for 2^13 .. 2^24 (log N1 of its second pass),
// per size and for zero-padded (forward LDE) input; ntt_set_split overrides the
// default log N / 2 (the measured choice of ntt_autotune), for every context.
// Every split gives the same output.
int ntt_split(int log_n, bool padded);
void ntt_set_split(int log_n, bool padded, int log_n1);

// Scratch (in elements) ntt_batch needs for n_cols columns of 2^log_n.
uint64_t ntt_scratch_elems(uint64_t n_cols, int log_n);

// Transform `n_cols` columns of length 2^log_n. Column c of the input starts at
// in + c*in_stride, of the output at out + c*out_stride. Input entries at index
// >= n_valid are treated as zero (zero-padded forward transform). `scratch`
// must hold ntt_scratch_elems(n_cols, log_n) elements; in == out is allowed.
// `pre` (optional) multiplies input element k by g^k first.
cudaError_t ntt_batch(const NttTables& t, const uint64_t* in, uint64_t* out, uint32_t n_cols, uint64_t in_stride,
                      uint64_t out_stride, int log_n, bool inverse, uint64_t n_valid, uint64_t* scratch,
                      cudaStream_t s, const PowSpec* pre = nullptr);

// Evaluate n_cols polynomials of degree < M = 2^log_m (coefficients contiguous,
// column stride M) on the N = M * 2^log_b points g * w_N^j in natural order
// (column stride N) in one pass, without scratch: a forward transform of the
// zero-padded coefficients times g^k, as ntt_batch computes it with `pre`.
// Needs ntt_coset_eval_ok(log_m, log_b): log_m <= 12 and at least as many
// cosets as a pass's lanes per CTA.
bool ntt_coset_eval_ok(int log_m, int log_b);
cudaError_t ntt_coset_eval(const NttTables& t, const uint64_t* coef, uint64_t* out, uint32_t n_cols, int log_m,
                           int log_b, cudaStream_t s, const PowSpec* pre = nullptr);

// Forward transform of w zero-padded columns (as ntt_batch with in_stride and
// n_valid) whose last pass, a 2^7-point DFT, hashes the rows of the result into
// Merkle leaves instead of storing them: leaf r (kc::kDigestLanes lanes at
// leaves + r * kDigestLanes) = SHA3 of the build's profile of
// {arity0, 0xFFFFFFFF, r, label} || row r of the w columns. Only the first
// keep_cols columns of the result are written (to out, column stride 2^log_n).
// Needs lde_leaf_ok (w a multiple of 16, 2^9 <= N <= 2^31) and
// lde_leaf_scratch_elems(w, log_n) elements of scratch.
bool lde_leaf_ok(uint32_t w, int log_n);
uint64_t lde_leaf_scratch_elems(uint32_t w, int log_n);
cudaError_t lde_leaf_transform(const NttTables& t, const uint64_t* in, uint64_t in_stride, uint32_t w, int log_n,
                               uint64_t n_valid, const PowSpec* pre, uint64_t* scratch, uint64_t arity0,
                               uint64_t label, uint64_t* leaves, uint64_t* out, uint32_t keep_cols, cudaStream_t s);
// lde_leaf_transform in two steps: the passes before the fused one for columns
// c0 .. c0 + wc - 1 (column by column, so chunks can go as they arrive), then the
// fused pass over all w columns.
cudaError_t lde_leaf_prepasses(const NttTables& t, const uint64_t* in, uint64_t in_stride, uint32_t w, uint32_t c0,
                               uint32_t wc, int log_n, uint64_t n_valid, const PowSpec* pre, uint64_t* scratch,
                               cudaStream_t s);
cudaError_t lde_leaf_final(const NttTables& t, uint32_t w, int log_n, const uint64_t* scratch, uint64_t arity0,
                           uint64_t label, uint64_t* leaves, uint64_t* out, uint32_t keep_cols, cudaStream_t s);

}  // namespace sg

#if defined(__CUDACC__)
#include "gl.cuh"
namespace sg {
// w_N^e for N = 2^log_n <= 2^28 (any e; reduced mod N) from the two-level tables.
__device__ __forceinline__ uint64_t tw_pow(const uint64_t* lo, const uint64_t* hi, uint64_t e, int log_n) {
  const uint64_t E = (e << (kTwBaseLog - log_n)) & ((1ull << kTwBaseLog) - 1);
  return gl::mul(__ldg(lo + (E & (kTwEntries - 1))), __ldg(hi + (E >> kTwSplit)));
}
__device__ __forceinline__ uint64_t pow_at(const PowSpec& p, uint64_t k) {
  if (p.tab) return __ldg(p.tab + k);
  const uint64_t E = ((k * p.mult) << p.shl) & ((1ull << kTwBaseLog) - 1);
  return gl::mul(__ldg(p.lo + (E & (kTwEntries - 1))), __ldg(p.hi + (E >> kTwSplit)));
}
}  // namespace sg
#endif

// stir.cu — STIR out-of-domain evaluation and fold kernels.
#include "dft.cuh"
#include "keccak.cuh"
#include "ntt.cuh"
#include "stir.cuh"
#include "counters.hpp"

namespace sg {
namespace {

constexpr int kOodThreads = 256;

__device__ __forceinline__ uint64_t warp_sum(uint64_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = gl::add(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

// Groups of M coefficients per thread: enough threads to fill the GPU (2^17),
// and at most 16 groups each. Small layers thus spread over many CTAs instead of
// running a long serial loop on a few.
inline uint64_t ood_blocks(uint64_t n, int m) {
  const uint64_t groups = n / m;
  uint64_t gpt = groups >> 17;
  gpt = gpt < 1 ? 1 : gpt > 16 ? 16 : gpt;
  const uint64_t threads = (groups + gpt - 1) / gpt;
  const uint64_t b = (threads + kOodThreads - 1) / kOodThreads;
  return b ? b : 1;
}

// Thread tid accumulates T_r over groups t = tid, tid + S, ... (S = all threads),
// starting from w^tid = w^(256 block) w^(tid mod 256) and stepping by w^S:
// consecutive threads read consecutive groups of M coefficients. The factors come
// from the scalars' tables (three products deep).
// Proof groups (grid.y = proof g): with sc set, proof g's scalars are sc[g] and its
// coefficients / partials start g_c / g_p elements further on; else they are `one`.
template <int M, bool BASE>
__global__ void __launch_bounds__(kOodThreads) ood_partial_kernel(const uint64_t* c, uint64_t n,
                                                                   const OodScalars one, uint64_t* partials,
                                                                   const OodScalars* sc, uint64_t g_c,
                                                                   uint64_t g_p) {
  static_assert(kOodThreads == 256, "the factor tables cover 256 threads");
  const uint32_t b = blockIdx.x, t = threadIdx.x;
  gl::Fp6 tl, tm, bl, bm, w_stride, w64;
  if (sc) {
    const uint32_t g = blockIdx.y;
    const OodScalars& S = sc[g];
    tl = S.lo[t & 15], tm = S.mid[t >> 4], bl = S.blo[b & 15], bm = S.bmid[(b >> 4) & 15];
    w_stride = S.ws, w64 = S.w65536;
    c += g * g_c;
    partials += g * g_p;
  } else {
    tl = one.lo[t & 15], tm = one.mid[t >> 4], bl = one.blo[b & 15], bm = one.bmid[(b >> 4) & 15];
    w_stride = one.ws, w64 = one.w65536;
  }
  const uint64_t n_groups = n / M;
  const uint64_t S = (uint64_t)gridDim.x * kOodThreads;
  const uint64_t tid = (uint64_t)b * kOodThreads + t;
  // the start powers go through one out-of-line product: each runs once, and a
  // single shared copy of its code is fetched once (inlined copies cost more in
  // instruction fetch than the calls save)
  gl::Fp6 bf = gl::e_mul_call(bl, bm);
  if (b >= 256) bf = gl::e_mul_call(bf, gl::e_pow_call(w64, b >> 8));
  gl::Fp6 wt = gl::e_mul_call(bf, gl::e_mul_call(tl, tm));
  uint64_t acc[M][6];
#pragma unroll
  for (int r = 0; r < M; ++r)
#pragma unroll
    for (int q = 0; q < 6; ++q) acc[r][q] = 0;
  for (uint64_t t = tid; t < n_groups; t += S) {
#pragma unroll
    for (int r = 0; r < M; ++r) {
      const uint64_t k = t * M + r;
      if constexpr (BASE) {
        const uint64_t ck = __ldg(c + k);
#pragma unroll
        for (int q = 0; q < 6; ++q) acc[r][q] = gl::add(acc[r][q], gl::mul(wt.c[q], ck));
      } else {
        gl::Fp6 ck;
#pragma unroll
        for (int q = 0; q < 6; ++q) ck.c[q] = __ldg(c + (uint64_t)q * n + k);
        gl::Fp6 p = gl::e_mul(ck, wt);
#pragma unroll
        for (int q = 0; q < 6; ++q) acc[r][q] = gl::add(acc[r][q], p.c[q]);
      }
    }
    wt = gl::e_mul(wt, w_stride);
  }
  __shared__ uint64_t red[kOodThreads / 32][M * 6];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int r = 0; r < M; ++r)
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      uint64_t v = warp_sum(acc[r][q]);
      if (lane == 0) red[warp][r * 6 + q] = v;
    }
  __syncthreads();
  if (threadIdx.x < M * 6) {
    uint64_t v = 0;
#pragma unroll
    for (int wi = 0; wi < kOodThreads / 32; ++wi) v = gl::add(v, red[wi][threadIdx.x]);
    partials[(uint64_t)blockIdx.x * M * 6 + threadIdx.x] = v;
  }
}

// evals[j] = sum_r w_M^{jr} z^r T_r for j < M, with T (M x 6 words) in shared
// memory: thread r < M forms z^r T_r into U (zt = its z^r), then thread j adds
// the M terms times powers of two (w_M = 2^EM).
// Every thread of the block calls it (it holds a barrier).
template <int M>
__device__ __forceinline__ void ood_evals(const uint64_t* T, uint64_t* U, const gl::Fp6& zt, uint64_t* evals) {
  const int t = threadIdx.x;
  if (t < M) {
    gl::Fp6 tr;
#pragma unroll
    for (int q = 0; q < 6; ++q) tr.c[q] = T[t * 6 + q];
    const gl::Fp6 u = gl::e_mul_call(zt, tr);
#pragma unroll
    for (int q = 0; q < 6; ++q) U[t * 6 + q] = u.c[q];
  }
  __syncthreads();
  if (t >= M) return;
  constexpr unsigned EM = (exp16(false) * (16 / M)) % 192;
  gl::Fp6 acc = gl::e_zero();
#pragma unroll
  for (int r = 0; r < M; ++r) {
    const unsigned e = (EM * (unsigned)((t * r) % M)) % 192u;
#pragma unroll
    for (int q = 0; q < 6; ++q) acc.c[q] = gl::add(acc.c[q], gl::mul_pow2(U[r * 6 + q], e));
  }
#pragma unroll
  for (int q = 0; q < 6; ++q) evals[t * 6 + q] = acc.c[q];
}

// Small layers (at most kOodSmallGroups groups): one CTA of M warps. Warp r sums
// T_r = sum_t c_{tM+r} w^t with its lanes striding over t, then ood_evals forms
// evals[j] = sum_r w_M^{jr} z^r T_r. The kernel runs once on a few warps, so its
// time is mostly instruction fetch: its Fp6 products share one out-of-line copy
// (e_mul_call), 18 % faster than inlined copies on a 64-byte SHA-256 proof.
// Each lane's loop waits on its loads every iteration with only M warps on the SM,
// so the bound is kept at 8 iterations: a 4096-group layer took 0.14 ms here and
// takes a few microseconds through the partial and finish kernels.
constexpr uint64_t kOodSmallGroups = 256;  // the power tables cover w^t, t < 256
static_assert(kOodSmallGroups <= 256, "ood_small_kernel forms w^t from 16 x 16 tables");
template <int M, bool BASE>
__global__ void __launch_bounds__(M * 32) ood_small_kernel(const uint64_t* c, uint64_t n, const OodScalars one,
                                                           uint64_t* evals, const OodScalars* sc, uint64_t g_c,
                                                           uint64_t g_e) {
  const int t0 = threadIdx.x < M ? threadIdx.x : 0;
  const OodScalars* S = sc ? sc + blockIdx.x : nullptr;  // one CTA per proof
  if (sc) {
    c += blockIdx.x * g_c;
    evals += blockIdx.x * g_e;
  }
  const gl::Fp6 zt = S ? S->zr[t0] : one.zr[t0];
  const int lane = threadIdx.x & 31, r = threadIdx.x >> 5;
  const uint64_t n_groups = n / M;  // at most kOodSmallGroups = 256
  __shared__ uint64_t T[M * 6];
  uint64_t acc[6] = {0, 0, 0, 0, 0, 0};
  // w^t = lo[t & 15] mid[t >> 4] for t < 256: the steps share no product chain
#pragma unroll 2
  for (uint64_t t = lane; t < n_groups; t += 32) {
    gl::Fp6 lo, mid;
    if (S) {
      lo = S->lo[t & 15];
      mid = S->mid[t >> 4];
    } else {
      lo = one.lo[t & 15];
      mid = one.mid[t >> 4];
    }
    const gl::Fp6 wt = gl::e_mul_call(lo, mid);
    const uint64_t k = t * M + r;
    if constexpr (BASE) {
      const uint64_t ck = __ldg(c + k);
#pragma unroll
      for (int q = 0; q < 6; ++q) acc[q] = gl::add(acc[q], gl::mul(wt.c[q], ck));
    } else {
      gl::Fp6 ck;
#pragma unroll
      for (int q = 0; q < 6; ++q) ck.c[q] = __ldg(c + (uint64_t)q * n + k);
      const gl::Fp6 p = gl::e_mul_call(ck, wt);
#pragma unroll
      for (int q = 0; q < 6; ++q) acc[q] = gl::add(acc[q], p.c[q]);
    }
  }
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const uint64_t v = warp_sum(acc[q]);
    if (lane == 0) T[r * 6 + q] = v;
  }
  __syncthreads();
  __shared__ uint64_t U[M * 6];
  ood_evals<M>(T, U, zt, evals);
}

// Sum block partials into T_r, then evals[j] = sum_r w_M^{jr} z^r T_r.
template <int M>
__global__ void ood_finish_kernel(const uint64_t* partials, uint64_t n_blocks, const OodScalars one,
                                  uint64_t* evals, const OodScalars* sc, uint64_t g_p, uint64_t g_e) {
  const int t0 = threadIdx.x < M ? threadIdx.x : 0;
  gl::Fp6 zt;
  if (sc) {
    const uint32_t g = blockIdx.x;  // one CTA per proof
    zt = sc[g].zr[t0];
    partials += g * g_p;
    evals += g * g_e;
  } else {
    zt = one.zr[t0];
  }
  __shared__ uint64_t T[M * 6];
  // one warp per element: the lanes stride over the block partials
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, n_warps = blockDim.x >> 5;
  for (int e = warp; e < M * 6; e += n_warps) {
    uint64_t v = 0;
    for (uint64_t b = lane; b < n_blocks; b += 32) v = gl::add(v, partials[b * M * 6 + e]);
    v = warp_sum(v);
    if (lane == 0) T[e] = v;
  }
  __syncthreads();
  __shared__ uint64_t U[M * 6];
  ood_evals<M>(T, U, zt, evals);
}

// proof g = blockIdx.y of a group: its buffers and challenge (FoldArgs' g_* strides)
__device__ __forceinline__ void fold_select(FoldArgs& a) {
  const uint32_t g = blockIdx.y;
  if (g == 0 && !a.alphas) return;
  a.f += g * a.g_f;
  if (a.next) a.next += g * a.g_next;
  if (a.tuples) a.tuples += g * a.g_tuples;
  if (a.leaves) a.leaves += g * a.g_leaves;
  if (a.alphas) a.alpha = a.alphas[g];
}

template <int M, bool BASE>
__global__ void fold_kernel(FoldArgs a) {
  constexpr int LM = M == 2 ? 1 : M == 4 ? 2 : M == 8 ? 3 : 4;
  const uint64_t nn = a.n / M;
  const uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (b >= nn) return;
  fold_select(a);
  constexpr int NC = BASE ? 1 : 6;
  uint64_t x[NC][M];
#pragma unroll
  for (int q = 0; q < NC; ++q) {
#pragma unroll
    for (int j = 0; j < M; ++j) x[q][j] = __ldg(a.f + (uint64_t)q * a.n + b + (uint64_t)j * nn);
    dft_reg<M, true>(x[q]);
  }
  // w_n^{-b}
  const uint64_t obinv = tw_pow(a.tw_inv_lo, a.tw_inv_hi, b, a.log_n);
  constexpr unsigned MINV = 192u - LM;  // 1/M = 2^{-LM} = 2^{192-LM}
  if (a.tuples) {
    uint64_t p = 1;
#pragma unroll
    for (int k = 0; k < M; ++k) {
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        uint64_t v = q < NC ? gl::mul(gl::mul_pow2(x[q][k], MINV), p) : 0;
        a.tuples[(uint64_t)(k * 6 + q) * nn + b] = v;
      }
      p = gl::mul(p, obinv);
    }
  }
  if (!a.next) return;
  const gl::Fp6 beta = gl::e_scale(a.alpha, obinv);
  gl::Fp6 acc;
#pragma unroll
  for (int q = 0; q < 6; ++q) acc.c[q] = q < NC ? x[q][M - 1] : 0;
#pragma unroll
  for (int k = M - 2; k >= 0; --k) {
    acc = gl::e_mul(acc, beta);
#pragma unroll
    for (int q = 0; q < NC; ++q) acc.c[q] = gl::add(acc.c[q], x[q][k]);
  }
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    acc.c[q] = gl::mul_pow2(acc.c[q], MINV);
    a.next[(uint64_t)q * nn + b] = acc.c[q];
  }
  if (a.leaves) {
    kc::LaneSponge sp;
    sp.init();
    sp.lane(a.leaf_arity0);
    sp.lane(0xFFFFFFFFull);
    sp.lane(b);
    sp.lane(a.leaf_label);
#pragma unroll
    for (int q = 0; q < 6; ++q) sp.lane(acc.c[q]);
    uint64_t d[kc::kDigestLanes];
    sp.finish(d);
#pragma unroll
    for (int i = 0; i < kc::kDigestLanes; ++i) a.leaves[kc::kDigestLanes * b + i] = d[i];
  }
}

// The fold for small layers (at most kFoldSmall cosets): the same arithmetic with
// the per-component DFT in a rolled loop (results in a local array) and the Horner
// products as calls, so a launch that runs once does not stream a large body of
// inlined code through the instruction cache.
constexpr uint64_t kFoldSmall = 4096;
template <int M, bool BASE>
__global__ void fold_small_kernel(FoldArgs a) {
  constexpr int LM = M == 2 ? 1 : M == 4 ? 2 : M == 8 ? 3 : 4;
  const uint64_t nn = a.n / M;
  const uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (b >= nn) return;
  fold_select(a);
  constexpr int NC = BASE ? 1 : 6;
  uint64_t xs[NC][M];
#pragma unroll 1
  for (int q = 0; q < NC; ++q) {
    uint64_t y[M];
#pragma unroll
    for (int j = 0; j < M; ++j) y[j] = __ldg(a.f + (uint64_t)q * a.n + b + (uint64_t)j * nn);
    dft_reg<M, true>(y);
#pragma unroll
    for (int j = 0; j < M; ++j) xs[q][j] = y[j];
  }
  const uint64_t obinv = tw_pow(a.tw_inv_lo, a.tw_inv_hi, b, a.log_n);  // w_n^{-b}
  constexpr unsigned MINV = 192u - LM;                                     // 1/M = 2^{-LM}
  if (a.tuples) {
    uint64_t p = 1;
#pragma unroll 1
    for (int k = 0; k < M; ++k) {
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        const uint64_t v = q < NC ? gl::mul(gl::mul_pow2(xs[q][k], MINV), p) : 0;
        a.tuples[(uint64_t)(k * 6 + q) * nn + b] = v;
      }
      p = gl::mul(p, obinv);
    }
  }
  if (!a.next) return;
  const gl::Fp6 beta = gl::e_scale(a.alpha, obinv);
  gl::Fp6 acc;
#pragma unroll
  for (int q = 0; q < 6; ++q) acc.c[q] = q < NC ? xs[q][M - 1] : 0;
#pragma unroll 1
  for (int k = M - 2; k >= 0; --k) {
    acc = gl::e_mul_call(acc, beta);
#pragma unroll
    for (int q = 0; q < NC; ++q) acc.c[q] = gl::add(acc.c[q], xs[q][k]);
  }
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    acc.c[q] = gl::mul_pow2(acc.c[q], MINV);
    a.next[(uint64_t)q * nn + b] = acc.c[q];
  }
  if (a.leaves) {
    kc::LaneSponge sp;
    sp.init();
    sp.lane(a.leaf_arity0);
    sp.lane(0xFFFFFFFFull);
    sp.lane(b);
    sp.lane(a.leaf_label);
#pragma unroll
    for (int q = 0; q < 6; ++q) sp.lane(acc.c[q]);
    uint64_t d[kc::kDigestLanes];
    sp.finish(d);
#pragma unroll
    for (int i = 0; i < kc::kDigestLanes; ++i) a.leaves[kc::kDigestLanes * b + i] = d[i];
  }
}

template <int M>
__global__ void fold_tuples_kernel(const uint64_t* tup, uint64_t nf, gl::Fp6 alpha, uint64_t* next,
                                   const gl::Fp6* alphas, uint64_t g_tup, uint64_t g_next) {
  const uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (b >= nf) return;
  if (alphas) {
    const uint32_t g = blockIdx.y;
    alpha = alphas[g];
    tup += g * g_tup;
    next += g * g_next;
  }
  gl::Fp6 acc;
#pragma unroll
  for (int q = 0; q < 6; ++q) acc.c[q] = tup[(uint64_t)((M - 1) * 6 + q) * nf + b];
#pragma unroll
  for (int k = M - 2; k >= 0; --k) {
    acc = gl::e_mul(acc, alpha);
#pragma unroll
    for (int q = 0; q < 6; ++q) acc.c[q] = gl::add(acc.c[q], tup[(uint64_t)(k * 6 + q) * nf + b]);
  }
#pragma unroll
  for (int q = 0; q < 6; ++q) next[(uint64_t)q * nf + b] = acc.c[q];
}

// One proof (sc null: its scalars built here from z and passed by value) or a
// group of G proofs (sc set: their scalars in device memory).
template <int M>
cudaError_t ood_launch(const uint64_t* c, uint64_t g_c, bool base, uint64_t n, const gl::Fp6& z,
                       const OodScalars* sc, uint64_t* partials, uint64_t* evals, uint64_t g_e, uint32_t G,
                       cudaStream_t s) {
  const OodScalars one = sc ? OodScalars{} : ood_scalars(z, n, M);
  if (n / M <= kOodSmallGroups) {
    SG_LAUNCH_SCOPE("stir_ood", s);
    if (base)
      ood_small_kernel<M, true><<<G, M * 32, 0, s>>>(c, n, one, evals, sc, g_c, g_e);
    else
      ood_small_kernel<M, false><<<G, M * 32, 0, s>>>(c, n, one, evals, sc, g_c, g_e);
    return cudaGetLastError();
  }
  const uint64_t blocks = ood_blocks(n, M), g_p = blocks * M * 6;
  if (blocks > 65535) return cudaErrorInvalidValue;
  {
    SG_LAUNCH_SCOPE("stir_ood", s);
    if (base)
      ood_partial_kernel<M, true><<<dim3((unsigned)blocks, G), kOodThreads, 0, s>>>(c, n, one, partials, sc, g_c,
                                                                                     g_p);
    else
      ood_partial_kernel<M, false><<<dim3((unsigned)blocks, G), kOodThreads, 0, s>>>(c, n, one, partials, sc,
                                                                                      g_c, g_p);
  }
  SG_LAUNCH_SCOPE("stir_ood_finish", s);
  ood_finish_kernel<M><<<G, 256, 0, s>>>(partials, blocks, one, evals, sc, g_p, g_e);
  return cudaGetLastError();
}

template <int M>
cudaError_t fold_launch(const FoldArgs& a, cudaStream_t s) {
  const uint64_t nn = a.n / M;
  const unsigned T = 128;
  const unsigned blocks = (unsigned)((nn + T - 1) / T);
  const dim3 grid(blocks, a.n_proofs ? a.n_proofs : 1);
  SG_LAUNCH_SCOPE("stir_fold", s);
  if (nn <= kFoldSmall) {
    if (a.base)
      fold_small_kernel<M, true><<<grid, T, 0, s>>>(a);
    else
      fold_small_kernel<M, false><<<grid, T, 0, s>>>(a);
  } else if (a.base) {
    fold_kernel<M, true><<<grid, T, 0, s>>>(a);
  } else {
    fold_kernel<M, false><<<grid, T, 0, s>>>(a);
  }
  return cudaGetLastError();
}

}  // namespace

uint64_t ood_partials_len(uint64_t n, int m) { return ood_blocks(n, m) * (uint64_t)m * 6; }

cudaError_t ood_evaluate(const uint64_t* coeffs, bool base, uint64_t n, int m, const gl::Fp6& z,
                         uint64_t* partials, uint64_t* evals, cudaStream_t s) {
  if (n % m) return cudaErrorInvalidValue;
  switch (m) {
    case 2: return ood_launch<2>(coeffs, 0, base, n, z, nullptr, partials, evals, 0, 1, s);
    case 4: return ood_launch<4>(coeffs, 0, base, n, z, nullptr, partials, evals, 0, 1, s);
    case 8: return ood_launch<8>(coeffs, 0, base, n, z, nullptr, partials, evals, 0, 1, s);
    case 16: return ood_launch<16>(coeffs, 0, base, n, z, nullptr, partials, evals, 0, 1, s);
    default: return cudaErrorInvalidValue;
  }
}

OodScalars ood_scalars(const gl::Fp6& z, uint64_t n, int m) {
  OodScalars r;
  r.z = z;
  // t-th powers of x for t < 16, and x^16
  auto powers = [](const gl::Fp6& x, gl::Fp6* out) {
    out[0] = gl::e_one();
    for (int t = 1; t < 16; ++t) out[t] = gl::e_mul(out[t - 1], x);
    return gl::e_mul(out[15], x);
  };
  const gl::Fp6 z16 = powers(z, r.zr);
  r.w = m == 16 ? z16 : r.zr[m];
  const gl::Fp6 w16 = powers(r.w, r.lo);
  const gl::Fp6 w256 = powers(w16, r.mid);
  const gl::Fp6 w4096 = powers(w256, r.blo);
  r.w65536 = powers(w4096, r.bmid);
  r.w32 = r.mid[2];
  const uint64_t S = ood_blocks(n, m) * kOodThreads;  // w^S = w^(256 b) for b = S / 256 blocks
  r.ws = gl::e_mul(gl::e_mul(r.blo[(S >> 8) & 15], r.bmid[(S >> 12) & 15]), gl::e_pow(r.w65536, S >> 16));
  return r;
}

cudaError_t ood_evaluate_group(const uint64_t* coeffs, uint64_t g_c, bool base, uint64_t n, int m,
                               const OodScalars* sc, uint64_t* partials, uint64_t* evals, uint64_t g_e,
                               uint32_t n_proofs, cudaStream_t s) {
  if (n % m || !sc || n_proofs == 0 || n_proofs > 65535) return cudaErrorInvalidValue;
  const gl::Fp6 z = gl::e_zero();
  switch (m) {
    case 2: return ood_launch<2>(coeffs, g_c, base, n, z, sc, partials, evals, g_e, n_proofs, s);
    case 4: return ood_launch<4>(coeffs, g_c, base, n, z, sc, partials, evals, g_e, n_proofs, s);
    case 8: return ood_launch<8>(coeffs, g_c, base, n, z, sc, partials, evals, g_e, n_proofs, s);
    case 16: return ood_launch<16>(coeffs, g_c, base, n, z, sc, partials, evals, g_e, n_proofs, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t stir_fold(const FoldArgs& a, cudaStream_t s) {
  if (a.n % a.m || a.log_n > kMaxLogN || a.n_proofs > 65535) return cudaErrorInvalidValue;
  switch (a.m) {
    case 2: return fold_launch<2>(a, s);
    case 4: return fold_launch<4>(a, s);
    case 8: return fold_launch<8>(a, s);
    case 16: return fold_launch<16>(a, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t fold_tuples(const uint64_t* tuples, uint64_t n_final, int m, const gl::Fp6& alpha, uint64_t* next,
                        cudaStream_t s) {
  const unsigned blocks = (unsigned)((n_final + 127) / 128);
  SG_LAUNCH_SCOPE("stir_fold_tuples", s);
  switch (m) {
    case 2: fold_tuples_kernel<2><<<blocks, 128, 0, s>>>(tuples, n_final, alpha, next, nullptr, 0, 0); break;
    case 4: fold_tuples_kernel<4><<<blocks, 128, 0, s>>>(tuples, n_final, alpha, next, nullptr, 0, 0); break;
    case 8: fold_tuples_kernel<8><<<blocks, 128, 0, s>>>(tuples, n_final, alpha, next, nullptr, 0, 0); break;
    case 16: fold_tuples_kernel<16><<<blocks, 128, 0, s>>>(tuples, n_final, alpha, next, nullptr, 0, 0); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t fold_tuples_group(const uint64_t* tuples, uint64_t g_tup, uint64_t n_final, int m,
                              const gl::Fp6* alphas, uint64_t* next, uint64_t g_next, uint32_t n_proofs,
                              cudaStream_t s) {
  if (!alphas || n_proofs == 0 || n_proofs > 65535) return cudaErrorInvalidValue;
  const dim3 grid((unsigned)((n_final + 127) / 128), n_proofs);
  const gl::Fp6 z = gl::e_zero();
  SG_LAUNCH_SCOPE("stir_fold_tuples", s);
  switch (m) {
    case 2: fold_tuples_kernel<2><<<grid, 128, 0, s>>>(tuples, n_final, z, next, alphas, g_tup, g_next); break;
    case 4: fold_tuples_kernel<4><<<grid, 128, 0, s>>>(tuples, n_final, z, next, alphas, g_tup, g_next); break;
    case 8: fold_tuples_kernel<8><<<grid, 128, 0, s>>>(tuples, n_final, z, next, alphas, g_tup, g_next); break;
    case 16: fold_tuples_kernel<16><<<grid, 128, 0, s>>>(tuples, n_final, z, next, alphas, g_tup, g_next); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace sg

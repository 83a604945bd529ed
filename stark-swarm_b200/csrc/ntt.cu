// ntt.cu — batched Goldilocks NTT for sm_100a.
//
// Global structure: a transform of N = 2^n <= 2^12 is one pass; up to 2^24 it
// is a four-step split N = N1 * N2 (N1 <= N2 <= 2^12) done as two passes:
//   pass 1: for each k1 < N1, DFT_{N2} over k2 of x[k2*N1 + k1], times w_N^{i2*k1},
//           stored transposed at i2*N1 + k1;
//   pass 2: for each i2 < N2, DFT_{N1} over the contiguous row, stored at i1*N2 + i2.
// Up to 2^28 the second step is itself split (N = A*B*C, three passes):
//   pass 1 as above with N1 = A*B, N2 = C;
//   pass 2: inside each block i3, DFT_B over k2 of rows k1 < A, times
//           w_{AB}^{i2*k1}, written to row (i2*C + i3) so that
//   pass 3: DFT_A over each contiguous row, stored at i1*BC + (i2*C + i3).
// A CTA owns K "lanes" (independent sub-DFTs with adjacent addresses, so every
// global row access is K*8 contiguous bytes) x M points in shared memory.
// Inside the CTA the M-point DFT is a Stockham autosort sequence of radix-16
// (and one smaller) stages: each thread holds 16 values in registers, reads
// them, barrier, writes them to their permuted slots, barrier. Shared memory
// is padded one word per 16 so every stage's stride pattern is conflict-free.
// The radix-R butterflies use only powers of w_R <= w_16, which in Goldilocks
// are powers of two (w_16 = 2^156 for ark's root chain).
#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>
#include <vector>

#include "counters.hpp"
#include "dft.cuh"
#include "gl.cuh"
#include "keccak.cuh"
#include "ntt.cuh"

namespace sg {
namespace {

__device__ __forceinline__ int padi(int m) { return m + (m >> 4); }

// Lanes per CTA (2^pass_log_k): at least 4 (32-byte global rows), about 8192
// elements per CTA, at most 1024 threads.
__host__ __device__ constexpr int pass_log_k(int log_m) {
  int lk = log_m >= 11 ? 2 : 13 - log_m;
  while (((1 << lk) << log_m) / (log_m < 4 ? (1 << log_m) : 16) > 1024) --lk;
  return lk;
}
// Shared-memory words between the rows of two lanes. Inside a row, one word of
// padding per 16 keeps every Stockham stage conflict-free. The load and store
// phases walk the lanes fastest (a half-warp covers K lanes x 16/K points), so
// for M >= 256 the row stride is also padded to 16/K (mod 16) words; below that
// a half-warp's stage accesses span several rows and the plain stride is kept.
__host__ __device__ constexpr int row_stride(int log_m) {
  const int M = 1 << log_m, Mp = M + (M >> 4), K = 1 << pass_log_k(log_m);
  return M >= 256 ? Mp + (K < 16 ? 16 / K : 1) : Mp;
}

// Twiddles staged in shared memory after the tile. Stage twiddles w_M^j (j < M)
// pay off while the tile is small (M <= 2^10); for the 2^11 and 2^12 passes the
// extra 16-32 KB costs more residency than the L1-cached table loads it saves.
// The pass twiddle w^{lane i} is the product of per-lane factors w^{lane (i mod 64)}
// and w^{64 lane (i / 64)}, built once per CTA from the global w28 tables.
__host__ __device__ constexpr bool stage_tw_in_smem(int log_m) { return log_m >= 5 && log_m <= 10; }
// Pass-twiddle factors for the 2^11 and 2^12 passes (K = 4 lanes); below that the
// per-lane build costs more than the table loads it replaces. A lane's factors
// are padded to 16/K (mod 16) words, so the K lanes a half-warp's stores cover
// start in distinct banks.
__host__ __device__ constexpr bool pass_tw_in_smem(int log_m) { return log_m >= 11; }
__host__ __device__ constexpr int pass_tw_stride(int log_m) {
  const int K = 1 << pass_log_k(log_m), n = 64 + ((1 << log_m) >> 6), want = K < 16 ? 16 / K : 0;
  return n + (((want - n) % 16) + 16) % 16;
}
__host__ __device__ constexpr size_t pass_table_bytes(int log_m) {
  const int M = 1 << log_m, K = 1 << pass_log_k(log_m);
  return 8 * ((stage_tw_in_smem(log_m) ? M : 0) + (pass_tw_in_smem(log_m) ? K * pass_tw_stride(log_m) : 0));
}

struct PassArgs {
  const uint64_t* in;
  uint64_t* out;
  // grid row y = blockIdx.y + y_base -> (c, s) = (y / y_sub, y % y_sub); the
  // tile's base is in + c*in_col + s*in_sub (same for out)
  uint64_t in_col, out_col, in_sub, out_sub;
  uint32_t y_sub;
  uint32_t y_base;
  uint64_t in_lane, in_m;     // input address of (lane, m)
  uint64_t out_lane, out_i;   // output address of (lane, i)
  uint64_t n_lanes;           // valid lanes
  // zero padding: the input element's flat index inside its column is
  // m*in_m + lane*flat_lane; indices >= in_valid are zero and never read
  uint64_t flat_lane;
  uint64_t in_valid;
  // 1 or 2 when only the first `sparse_nz` of the 16 inputs of every first-stage
  // radix-16 group can be non-zero (zero-padded forward transform); 0 = dense
  int sparse_nz;
  int tw_log;                 // > 0: output (lane, i) *= w_{2^tw_log}^(i*lane)
  const uint64_t* tw_tab;     // if set, that twiddle is tw_tab[i * n_lanes + lane]
  // grid x = grid row (column), y = lane group: the CTAs of one lane group run
  // back to back over all columns, so they share its tw_tab entries through L2
  bool cols_fast;
  int in_tw_log;              // > 0: input (lane, m) *= w_{2^in_tw_log}^(m*lane)
  const uint64_t* in_tw_tab;  // if set, that twist is in_tw_tab[m * lane] (m * lane < 2^in_tw_log)
  int out_i_log;              // coset evaluation: out_i = 2^out_i_log
  uint64_t scale;             // != 1: outputs *= scale
  const uint64_t* tw_st;      // w_4096^i (direction of the transform)
  const uint64_t* tw_lo;      // w28^i
  const uint64_t* tw_hi;      // w28^(2^14 i)
  PowSpec pre;                // lo != nullptr: input at flat index k times g^k
};

// One Stockham stage of radix R over all K lanes of the tile.
// Each thread holds V values = V/R groups; group g -> lane g / G, j = g % G.
template <int R, int V, bool INV, int TWL, bool TW_SM>
__device__ __forceinline__ void stockham_stage(uint64_t* sm, int t, int T, int log_m, int Mp, int log_ns,
                                               const uint64_t* tw_st) {
  constexpr int GPT = V / R;
  constexpr int LR = R == 2 ? 1 : R == 4 ? 2 : R == 8 ? 3 : 4;
  const int log_g = log_m - LR;
  const int G = 1 << log_g;
  const int Ns = 1 << log_ns;
  // Padded offsets as base + r * stride: when G (or Ns) is a multiple of 16,
  // padi(j + r G) = padi(j) + r (G + G/16), so the R accesses of a group are one
  // address and R immediate (or one-register) offsets.
  const int gstride = G + (G >> 4);
  uint64_t v[V];
#pragma unroll
  for (int q = 0; q < GPT; ++q) {
    int g = t + q * T;
    int l = g >> log_g, j = g & (G - 1);
    uint64_t* row = sm + l * Mp;
    if (G % 16 == 0) {
      const uint64_t* p = row + padi(j);
#pragma unroll
      for (int r = 0; r < R; ++r) v[q * R + r] = p[r * gstride];
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) v[q * R + r] = row[padi(j + r * G)];
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < GPT; ++q) {
    int g = t + q * T;
    int l = g >> log_g, j = g & (G - 1);
    int k = j & (Ns - 1);
    if (log_ns > 0) {
      // w_{Ns R}^{rk} = w_{2^TWL}^{rk 2^TWL/(Ns R)}; r k < Ns R, so the index
      // r (k << sh) stays below 2^TWL
      const int kk = k << (TWL - log_ns - LR);
      int ix = 0;
#pragma unroll
      for (int r = 1; r < R; ++r) {
        ix += kk;
        v[q * R + r] = gl::mul(v[q * R + r], TW_SM ? tw_st[ix] : __ldg(tw_st + ix));
      }
    }
    dft_reg<R, INV>(v + q * R);
    int idx = ((j >> log_ns) << (log_ns + LR)) + k;
    uint64_t* row = sm + l * Mp;
    // stages run with Ns = 1 (idx a multiple of R, the R outputs in one padded
    // 16-word block) or Ns >= 16 (every r Ns a multiple of 16)
    if (log_ns == 0 || log_ns >= 4) {
      uint64_t* p = row + padi(idx);
      const int ostride = log_ns == 0 ? 1 : Ns + (Ns >> 4);
#pragma unroll
      for (int r = 0; r < R; ++r) p[r * ostride] = v[q * R + r];
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) row[padi(idx + r * Ns)] = v[q * R + r];
    }
  }
  __syncthreads();
}

// First Stockham stage (Ns = 1, radix 16) when only inputs r < NZ of each group
// can be non-zero: X[k] = sum_{r<NZ} x_r w_16^{rk}. NZ = 1 is a broadcast,
// NZ = 2 is X[k], X[k+8] = x0 +- w_16^k x1 (7 shift-multiplies, no full DFT).
template <int NZ, bool INV>
__device__ __forceinline__ void stockham_first_sparse(uint64_t* sm, int t, int T, int K, int log_m, int Mp) {
  const int log_g = log_m - 4, G = 1 << log_g;
  const int groups = K << log_g;
  constexpr unsigned E16 = exp16(INV);
  for (int g0 = 0; g0 < groups; g0 += T) {
    const int g = g0 + t;
    uint64_t x0 = 0, x1 = 0;
    int l = 0, j = 0;
    if (g < groups) {
      l = g >> log_g;
      j = g & (G - 1);
      x0 = sm[l * Mp + padi(j)];
      if (NZ == 2) x1 = sm[l * Mp + padi(j + G)];
    }
    __syncthreads();
    if (g < groups) {
      uint64_t* row = sm + l * Mp;
      const int base = j << 4;
      if (NZ == 1) {
#pragma unroll
        for (int k = 0; k < 16; ++k) row[padi(base + k)] = x0;
      } else {
        row[padi(base)] = gl::add(x0, x1);
        row[padi(base + 8)] = gl::sub(x0, x1);
#pragma unroll
        for (int k = 1; k < 8; ++k) {
          const uint64_t w = gl::mul_pow2(x1, (E16 * (unsigned)k) % 192u);
          row[padi(base + k)] = gl::add(x0, w);
          row[padi(base + k + 8)] = gl::sub(x0, w);
        }
      }
    }
    __syncthreads();
  }
}

// COSET: the input twist w_{2^in_tw_log}^(m*lane) of ntt_coset_eval (a separate
// instantiation, so the other passes' register allocation does not carry it).
template <int LOG_M, bool INV, bool COSET = false>
__global__ void __launch_bounds__(1024) ntt_pass_kernel(PassArgs a) {
  constexpr int M = 1 << LOG_M;
  constexpr int V = M < 16 ? M : 16;
  constexpr int Mp = row_stride(LOG_M);
  constexpr int LOG_K = pass_log_k(LOG_M);
  extern __shared__ uint64_t sm[];
  constexpr int K = 1 << LOG_K;
  constexpr int E = K * M;
  constexpr int T = E / V;  // blockDim.x (launch_pass); every thread owns V elements
  const int t = threadIdx.x;
  // the launch has exactly T threads: with t < T known, the (lane, point) split of
  // t + q T folds into per-thread constants plus compile-time offsets
  __builtin_assume(t < T);
  const uint64_t lane0 = (uint64_t)(a.cols_fast ? blockIdx.y : blockIdx.x) << LOG_K;
  const uint64_t y = (uint64_t)(a.cols_fast ? blockIdx.x : blockIdx.y) + a.y_base;
  const uint64_t yc = y / a.y_sub, ys = y - yc * a.y_sub;
  const uint64_t* in = a.in + yc * a.in_col + ys * a.in_sub;
  uint64_t* out = a.out + yc * a.out_col + ys * a.out_sub;
  constexpr bool STW = stage_tw_in_smem(LOG_M);
  constexpr bool PTW = pass_tw_in_smem(LOG_M);
  constexpr int PT_PER = pass_tw_stride(LOG_M), PT_N = 64 + (M >> 6);
  uint64_t* stw = sm + K * Mp;
  uint64_t* ptw = stw + (STW ? M : 0);
  if constexpr (STW)
    for (int j = t; j < M; j += T) stw[j] = __ldg(a.tw_st + (j << (12 - LOG_M)));
  if constexpr (PTW) {
    if (a.tw_log > 0 && !a.tw_tab)
      for (int x = t; x < K * PT_N; x += T) {
        const int l = x / PT_N, r = x - l * PT_N;
        const uint64_t lane = lane0 + l;
        const uint64_t e = r < 64 ? lane * (uint64_t)r : lane * (uint64_t)(r - 64) * 64;
        ptw[l * PT_PER + r] = tw_pow(a.tw_lo, a.tw_hi, e, a.tw_log);
      }
  }

  const bool lane_fast_in = a.in_lane == 1;
  // a sparse first stage reads only points m < nz * M/16: skip the rest
  const int sparse = (LOG_M >= 4 && lane_fast_in) ? a.sparse_nz : 0;
  const int E_load = sparse ? K * sparse * (M >> 4) : E;
  // Global loads go out in batches of B before the batch's shared stores (a
  // generic load may not pass a shared store, so the split is explicit).
  constexpr int B = V < 8 ? V : 8;
  // element e of the tile -> (lane l, point m): lanes fastest or points fastest
  auto in_pos = [&](auto lf_c, int e, int& l, int& m) {
    if constexpr (decltype(lf_c)::value) {
      l = e & (K - 1);
      m = e >> LOG_K;
    } else {
      m = e & (M - 1);
      l = e >> LOG_M;
    }
  };
  // The uniform choices (pre-multiplication, a tile with every lane valid and no
  // zero padding) are taken once per CTA outside the element loops, so that each
  // loop is straight-line code without per-element predicates or selects.
  auto load_tile = [&](auto pre_c, auto full_c, auto lf_c) {
    constexpr bool PRE = decltype(pre_c)::value, FULL = decltype(full_c)::value;
#pragma unroll
    for (int q0 = 0; q0 < V; q0 += B) {
      uint64_t x[B];
#pragma unroll
      for (int q = 0; q < B; ++q) {
        const int e = t + (q0 + q) * T;
        int l, m;
        in_pos(lf_c, e, l, m);
        const uint64_t lane = lane0 + l;
        x[q] = 0;
        if constexpr (COSET) {
          // one column's cosets: point m of every lane is in[m], all lanes valid
          // (ntt_coset_eval launches exactly B / K CTAs per column)
          x[q] = __ldg(in + m);
          if (PRE) x[q] = gl::mul(x[q], pow_at(a.pre, (uint64_t)m));
          // w_N^e for N <= 2^14 is one entry of the hi table (hi[j] = w_{2^14}^j); above,
          // one entry of the per-size table when there is one
          const uint64_t ex = (uint64_t)m * lane;
          x[q] = gl::mul(x[q], a.in_tw_log <= kTwSplit
                                   ? __ldg(a.tw_hi + ((ex << (kTwSplit - a.in_tw_log)) & (kTwEntries - 1)))
                               : a.in_tw_tab ? __ldg(a.in_tw_tab + ex)
                                             : tw_pow(a.tw_lo, a.tw_hi, ex, a.in_tw_log));
        } else {
          const uint64_t flat = (uint64_t)m * a.in_m + lane * a.flat_lane;
          if (FULL || (e < E_load && lane < a.n_lanes && flat < a.in_valid)) {
            x[q] = __ldg(in + lane * a.in_lane + (uint64_t)m * a.in_m);
            if (PRE) x[q] = gl::mul(x[q], pow_at(a.pre, flat));
          }
        }
      }
#pragma unroll
      for (int q = 0; q < B; ++q) {
        const int e = t + (q0 + q) * T;
        int l, m;
        in_pos(lf_c, e, l, m);
        if (FULL || e < E_load) sm[l * Mp + padi(m)] = x[q];
      }
    }
  };
  using yes = std::true_type;
  using no = std::false_type;
  auto load_dispatch = [&](auto lf_c) {
    if (a.pre.active()) {
      load_tile(yes{}, no{}, lf_c);
    } else {
      // largest flat index of the tile: point M-1 of its last lane
      const uint64_t flat_max = (uint64_t)(M - 1) * a.in_m + (lane0 + K - 1) * a.flat_lane;
      if (!COSET && E_load == E && lane0 + K <= a.n_lanes && flat_max < a.in_valid)
        load_tile(no{}, yes{}, lf_c);
      else
        load_tile(no{}, no{}, lf_c);
    }
  };
  if (lane_fast_in)
    load_dispatch(yes{});
  else
    load_dispatch(no{});
  __syncthreads();

  // Stage sequence: radix-16 stages, then one radix 2/4/8 stage for the remainder.
  constexpr int N16 = LOG_M / 4, REM = LOG_M % 4;
  int log_ns = 0;
  if constexpr (LOG_M >= 4) {
    int st0 = 0;
    if (sparse == 1 || sparse == 2) {
      if (sparse == 1)
        stockham_first_sparse<1, INV>(sm, t, T, K, LOG_M, Mp);
      else
        stockham_first_sparse<2, INV>(sm, t, T, K, LOG_M, Mp);
      log_ns = 4;
      st0 = 1;
    }
    constexpr int TWL = STW ? LOG_M : 12;
    const uint64_t* tws = STW ? stw : a.tw_st;
#pragma unroll 1
    for (int st = st0; st < N16; ++st) {
      stockham_stage<16, V, INV, TWL, STW>(sm, t, T, LOG_M, Mp, log_ns, tws);
      log_ns += 4;
    }
  }
  {
    constexpr int TWL = STW ? LOG_M : 12;
    const uint64_t* tws = STW ? stw : a.tw_st;
    if constexpr (REM == 1) stockham_stage<2, V, INV, TWL, STW>(sm, t, T, LOG_M, Mp, log_ns, tws);
    if constexpr (REM == 2) stockham_stage<4, V, INV, TWL, STW>(sm, t, T, LOG_M, Mp, log_ns, tws);
    if constexpr (REM == 3) stockham_stage<8, V, INV, TWL, STW>(sm, t, T, LOG_M, Mp, log_ns, tws);
  }

  const bool lane_fast_out = a.out_lane == 1;
  auto out_pos = [&](auto lf_c, int e, int& l, int& i) {
    if constexpr (decltype(lf_c)::value) {
      l = e & (K - 1);
      i = e >> LOG_K;
    } else {
      i = e & (M - 1);
      l = e >> LOG_M;
    }
  };
  // shared reads and pass-twiddle loads of a batch before its global stores;
  // the twiddle / scale choice is uniform and taken outside the loops
  auto store_tile = [&](auto tw_c, auto sc_c, auto lf_c, auto tab_c) {
    constexpr bool TW = decltype(tw_c)::value, SC = decltype(sc_c)::value, TAB = decltype(tab_c)::value;
#pragma unroll
    for (int q0 = 0; q0 < V; q0 += B) {
      uint64_t x[B];
#pragma unroll
      for (int q = 0; q < B; ++q) {
        int l, i;
        out_pos(lf_c, t + (q0 + q) * T, l, i);
        x[q] = sm[l * Mp + padi(i)];
        if constexpr (TW) {
          uint64_t w;
          if constexpr (PTW && !TAB) {
            w = gl::mul(ptw[l * PT_PER + (i & 63)], ptw[l * PT_PER + 64 + (i >> 6)]);
          } else {
            // (a CTA's lanes past n_lanes store nothing and read no table entry)
            if (TAB || a.tw_tab)
              w = lane0 + l < a.n_lanes ? __ldg(a.tw_tab + (uint64_t)i * a.n_lanes + lane0 + l) : 0;
            else
              w = tw_pow(a.tw_lo, a.tw_hi, (uint64_t)i * (lane0 + l), a.tw_log);
          }
          x[q] = gl::mul(x[q], w);
        }
        if constexpr (SC) x[q] = gl::mul(x[q], a.scale);
      }
#pragma unroll
      for (int q = 0; q < B; ++q) {
        int l, i;
        out_pos(lf_c, t + (q0 + q) * T, l, i);
        const uint64_t lane = lane0 + l;
        if constexpr (COSET)
          out[lane + ((uint64_t)i << a.out_i_log)] = x[q];  // point B i + t of the column
        else if (lane < a.n_lanes)
          out[lane * a.out_lane + (uint64_t)i * a.out_i] = x[q];
      }
    }
  };
  auto store_dispatch = [&](auto lf_c) {
    if (a.tw_log > 0) {
      if (a.scale != 1)
        store_tile(yes{}, yes{}, lf_c, no{});
      else if (PTW && a.tw_tab)  // (smaller passes take the table inside the one variant)
        store_tile(yes{}, no{}, lf_c, yes{});
      else
        store_tile(yes{}, no{}, lf_c, no{});
    } else if (a.scale != 1) {
      store_tile(no{}, yes{}, lf_c, no{});
    } else {
      store_tile(no{}, no{}, lf_c, no{});
    }
  };
  if (lane_fast_out)
    store_dispatch(yes{});
  else
    store_dispatch(no{});
}

template <int LOG_M>
cudaError_t launch_pass(const PassArgs& a0, bool inv, uint64_t n_rows, cudaStream_t s) {
  constexpr int M = 1 << LOG_M;
  constexpr int V = M < 16 ? M : 16;
  const PassArgs& a = a0;
  constexpr int K = 1 << pass_log_k(LOG_M);
  constexpr int T = K * M / V;
  static_assert(T <= 1024, "too many threads per CTA");
  const size_t smem = (size_t)K * row_stride(LOG_M) * sizeof(uint64_t) + pass_table_bytes(LOG_M);
  const uint64_t blocks = (a.n_lanes + K - 1) / K;
  auto kern = a.in_tw_log > 0 ? ntt_pass_kernel<LOG_M, false, true>
                              : inv ? ntt_pass_kernel<LOG_M, true> : ntt_pass_kernel<LOG_M, false>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  if (a.cols_fast) {
    // rows on grid x (up to 2^31 - 1), lane groups on grid y
    if (blocks > 65535 || n_rows > 0x7FFFFFFFull) return cudaErrorInvalidValue;
    PassArgs b = a;
    b.y_base = 0;
    SG_LAUNCH_SCOPE("ntt_pass", s);
    kern<<<dim3((unsigned)n_rows, (unsigned)blocks), T, smem, s>>>(b);
    return cudaGetLastError();
  }
  for (uint64_t y0 = 0; y0 < n_rows; y0 += 65535) {
    const uint32_t ny = (uint32_t)(n_rows - y0 < 65535 ? n_rows - y0 : 65535);
    PassArgs b = a;
    b.y_base = (uint32_t)y0;
    SG_LAUNCH_SCOPE("ntt_pass", s);
    kern<<<dim3((unsigned)blocks, ny), T, smem, s>>>(b);
  }
  return cudaGetLastError();
}

cudaError_t launch_pass_dyn(int log_m, const PassArgs& a, bool inv, uint64_t n_rows, cudaStream_t s) {
  switch (log_m) {
    case 1: return launch_pass<1>(a, inv, n_rows, s);
    case 2: return launch_pass<2>(a, inv, n_rows, s);
    case 3: return launch_pass<3>(a, inv, n_rows, s);
    case 4: return launch_pass<4>(a, inv, n_rows, s);
    case 5: return launch_pass<5>(a, inv, n_rows, s);
    case 6: return launch_pass<6>(a, inv, n_rows, s);
    case 7: return launch_pass<7>(a, inv, n_rows, s);
    case 8: return launch_pass<8>(a, inv, n_rows, s);
    case 9: return launch_pass<9>(a, inv, n_rows, s);
    case 10: return launch_pass<10>(a, inv, n_rows, s);
    case 11: return launch_pass<11>(a, inv, n_rows, s);
    case 12: return launch_pass<12>(a, inv, n_rows, s);
    default: return cudaErrorInvalidValue;
  }
}

__global__ void copy_cols_kernel(const uint64_t* in, uint64_t* out, uint32_t n_cols, uint64_t in_stride,
                                 uint64_t out_stride, uint64_t n) {
  uint64_t total = (uint64_t)n_cols * n;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total; e += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t c = e / n, k = e - c * n;
    out[c * out_stride + k] = in[c * in_stride + k];
  }
}

PassArgs base_args(const NttTables& t, bool inverse) {
  PassArgs a{};
  a.tw_st = inverse ? t.d_inv_st : t.d_fwd_st;
  a.tw_lo = inverse ? t.d_inv_lo : t.d_fwd_lo;
  a.tw_hi = inverse ? t.d_inv_hi : t.d_fwd_hi;
  a.y_sub = 1;
  a.scale = 1;
  return a;
}

// sparse first stage for pass 1 over k_hi: points m >= ceil(n_valid / n_lo) are zero
__global__ void pass_tw_kernel(const uint64_t* lo, const uint64_t* hi, int log_n, int log_n1, uint64_t* out) {
  const uint64_t total = 1ull << log_n, n1 = 1ull << log_n1;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total;
       e += (uint64_t)gridDim.x * blockDim.x)
    out[e] = tw_pow(lo, hi, (e >> log_n1) * (e & (n1 - 1)), log_n);
}

// Pass-1 twiddles w_N^{i k} of the split N = N1 N2 as a table [i < N2][k < N1],
// built once per (device, size, split, direction) and kept for the process: one
// load per element instead of two table loads and a product, for first passes of
// at most 2^10 points (8 MB for a 2^20 transform). Larger first passes keep their
// per-CTA factor tables in shared memory: with a global table the 2^12 pass spilled
// and read 64 MB per column, and the 64 x 2^23 LDE went from 16.3 to 18.0 ms.
const uint64_t* pass_twiddle_table(const NttTables& t, int log_n, int log_n1, bool inverse, cudaStream_t s) {
  static std::mutex mu;
  static std::map<std::tuple<int, int, int, int>, uint64_t*> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> g(mu);
  const auto key = std::make_tuple(dev, log_n, log_n1, inverse ? 1 : 0);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  uint64_t* d = nullptr;
  if (cudaMalloc(&d, 8ull << log_n) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;  // no room: the pass forms its twiddles itself
  }
  pass_tw_kernel<<<148 * 8, 256, 0, s>>>(inverse ? t.d_inv_lo : t.d_fwd_lo, inverse ? t.d_inv_hi : t.d_fwd_hi, log_n,
                                          log_n1, d);
  if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) {
    cudaFree(d);
    return nullptr;
  }
  cache[key] = d;
  return d;
}

__global__ void pow_table_kernel(const uint64_t* lo, const uint64_t* hi, uint64_t mult, int log_n, uint64_t len,
                                 uint64_t* tab) {
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < len; k += (uint64_t)gridDim.x * blockDim.x)
    tab[k] = tw_pow(lo, hi, k * mult, log_n);
}

// w_N^j for j < N = 2^log_n (forward), built once per (device, size) and kept for
// the process: the coset twist w_N^(m t) of ntt_coset_eval above 2^14 points is then
// one load instead of two table loads and a product (m t < N). Up to 2^20 points
// (8 MB); none for table views of callers that must not allocate.
const uint64_t* coset_twist_table(const NttTables& t, int log_n, cudaStream_t s) {
  if (!t.pass_tables || log_n <= kTwSplit || log_n > 20) return nullptr;
  static std::mutex mu;
  static std::map<std::pair<int, int>, uint64_t*> cache;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> g(mu);
  const auto key = std::make_pair(dev, log_n);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  uint64_t* d = nullptr;
  if (cudaMalloc(&d, 8ull << log_n) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;  // no room: the pass forms its twist itself
  }
  const uint64_t len = 1ull << log_n;
  pow_table_kernel<<<(unsigned)std::min<uint64_t>((len + 255) / 256, 148 * 16), 256, 0, s>>>(t.d_fwd_lo, t.d_fwd_hi,
                                                                                          1, log_n, len, d);
  if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) {
    cudaFree(d);
    return nullptr;
  }
  cache[key] = d;
  return d;
}

// columns from which a 2^11 / 2^12 first pass reads its twiddles from the
// per-size table (shared through L2) instead of building per-CTA factors
constexpr uint32_t kPassTabMinCols = 8;

int sparse_nz_for(uint64_t n_valid, uint64_t N, uint64_t n_lo, uint64_t M) {
  if (n_valid >= N || M < 16) return 0;  // dense, or a pass without a radix-16 first stage
  const uint64_t m_nz = (n_valid + n_lo - 1) / n_lo, G = M / 16;
  const uint64_t nz = (m_nz + G - 1) / G;
  return (n_valid < N && M >= 16 && nz <= 2) ? (int)(nz ? nz : 1) : 0;
}

}  // namespace

void ntt_tables_host(uint64_t* out) {
  for (int dir = 0; dir < 2; ++dir) {
    uint64_t* st = out + dir * kTwDirElems;
    uint64_t* lo = st + 4096;
    uint64_t* hi = lo + kTwEntries;
    uint64_t w28 = gl::root_of_unity(kTwBaseLog);
    uint64_t w4096 = gl::root_of_unity(12);
    if (dir == 1) {
      w28 = gl::inv(w28);
      w4096 = gl::inv(w4096);
    }
    const uint64_t wstep = gl::pow(w28, kTwEntries);
    uint64_t a = 1, b = 1, c = 1;
    for (int i = 0; i < 4096; ++i) {
      st[i] = c;
      c = gl::mul(c, w4096);
    }
    for (int i = 0; i < kTwEntries; ++i) {
      lo[i] = a;
      a = gl::mul(a, w28);
      hi[i] = b;
      b = gl::mul(b, wstep);
    }
  }
}

void pow_tables_host(uint64_t g, uint64_t scale, uint64_t* out) {
  uint64_t* lo = out;
  uint64_t* hi = out + kTwEntries;
  const uint64_t gstep = gl::pow(g, kTwEntries);
  uint64_t a = scale % gl::P, b = 1;
  for (int i = 0; i < kTwEntries; ++i) {
    lo[i] = a;
    a = gl::mul(a, g);
    hi[i] = b;
    b = gl::mul(b, gstep);
  }
}

NttTables ntt_tables_view(uint64_t* dev) {
  NttTables t;
  t.d_fwd_st = dev;
  t.d_fwd_lo = dev + 4096;
  t.d_fwd_hi = dev + 4096 + kTwEntries;
  t.d_inv_st = dev + kTwDirElems;
  t.d_inv_lo = dev + kTwDirElems + 4096;
  t.d_inv_hi = dev + kTwDirElems + 4096 + kTwEntries;
  return t;
}

cudaError_t ntt_tables_init(NttTables* t) {
  std::vector<uint64_t> h(2 * kTwDirElems);
  ntt_tables_host(h.data());
  uint64_t* dev = nullptr;
  cudaError_t e = cudaMalloc(&dev, h.size() * 8);
  if (e != cudaSuccess) return e;
  e = cudaMemcpy(dev, h.data(), h.size() * 8, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(dev);
    return e;
  }
  *t = ntt_tables_view(dev);
  t->owned = true;
  t->pass_tables = true;
  return cudaSuccess;
}

void ntt_tables_free(NttTables* t) {
  if (t->owned && t->d_fwd_st) cudaFree(t->d_fwd_st);
  *t = NttTables{};
}

bool ntt_coset_eval_ok(int log_m, int log_b) {
  return log_m >= 1 && log_m <= 12 && log_b >= pass_log_k(log_m) && log_m + log_b <= kMaxLogN;
}

// Coset t < B of the evaluation domain is the DFT_M of c_m * g^m * w_N^{t m}:
// f(g w_N^{B i + t}) = sum_m c_m g^m w_N^{t m} w_M^{i m}. One pass with one lane
// per coset (a CTA's K lanes are K cosets of one column, so its stores of point
// i are K adjacent outputs B i + t) and grid.y over the columns; every lane
// reads the same M coefficients.
cudaError_t ntt_coset_eval(const NttTables& t, const uint64_t* coef, uint64_t* out, uint32_t n_cols, int log_m,
                           int log_b, cudaStream_t s, const PowSpec* pre) {
  if (!ntt_coset_eval_ok(log_m, log_b)) return cudaErrorInvalidValue;
  if (n_cols == 0) return cudaSuccess;
  const uint64_t M = 1ull << log_m, B = 1ull << log_b;
  PassArgs a = base_args(t, false);
  a.pre = pre ? *pre : PowSpec{};
  a.in = coef;
  a.out = out;
  a.in_col = M;
  a.out_col = M * B;
  a.in_lane = 0;
  a.in_m = 1;
  a.out_lane = 1;
  a.out_i = B;
  a.out_i_log = log_b;
  a.n_lanes = B;
  a.flat_lane = 0;
  a.in_valid = M;
  a.in_tw_log = log_m + log_b;
  a.in_tw_tab = coset_twist_table(t, log_m + log_b, s);
  return launch_pass_dyn(log_m, a, false, n_cols, s);
}

cudaError_t pow_table_device(const NttTables& t, uint64_t mult, int log_n, uint64_t len, uint64_t* tab,
                             cudaStream_t s) {
  if (len == 0) return cudaSuccess;
  if (log_n < 0 || log_n > kMaxLogN || !tab) return cudaErrorInvalidValue;
  SG_LAUNCH_SCOPE("pow_table", s);
  pow_table_kernel<<<(unsigned)std::min<uint64_t>((len + 255) / 256, 148 * 16), 256, 0, s>>>(
      t.d_fwd_lo, t.d_fwd_hi, mult, log_n, len, tab);
  return cudaGetLastError();
}

uint64_t ntt_scratch_elems(uint64_t n_cols, int log_n) {
  if (log_n <= 12) return 0;
  const uint64_t N = 1ull << log_n;
  return (log_n <= 24 ? 1 : 2) * n_cols * N;
}

// Four-step split per (log N, zero-padded input): log N1 of the second pass.
// 0 = the default, log N / 2; ntt_autotune stores measured choices.
namespace {
std::atomic<int> g_split[kMaxLogN + 1][2];
}

int ntt_split(int log_n, bool padded) {
  const int tuned = (log_n >= 0 && log_n <= kMaxLogN) ? g_split[log_n][padded ? 1 : 0].load() : 0;
  return tuned ? tuned : log_n / 2;
}

void ntt_set_split(int log_n, bool padded, int log_n1) {
  if (log_n >= 13 && log_n <= 24) g_split[log_n][padded ? 1 : 0].store(log_n1);
}

cudaError_t ntt_batch(const NttTables& t, const uint64_t* in, uint64_t* out, uint32_t n_cols, uint64_t in_stride,
                      uint64_t out_stride, int log_n, bool inverse, uint64_t n_valid, uint64_t* scratch,
                      cudaStream_t s, const PowSpec* pre) {
  if (n_cols == 0) return cudaSuccess;
  if (log_n < 0 || log_n > kMaxLogN) return cudaErrorInvalidValue;
  const uint64_t N = 1ull << log_n;
  if (n_valid > N) n_valid = N;
  if (log_n == 0 && !pre) {
    if (in == out) return cudaSuccess;
    SG_LAUNCH_SCOPE("copy_cols", s);
    copy_cols_kernel<<<64, 256, 0, s>>>(in, out, n_cols, in_stride, out_stride, 1);
    return cudaGetLastError();
  }
  const uint64_t ninv = inverse ? gl::inv(N) : 1;
  const PowSpec none{};
  if (log_n <= 12) {
    // one pass; the lanes are the columns (a length-1 "transform" is the identity
    // pass, used only to apply pre)
    PassArgs a = base_args(t, inverse);
    a.pre = pre ? *pre : none;
    a.in = in;
    a.out = out;
    a.in_lane = in_stride;
    a.in_m = 1;
    a.out_lane = out_stride;
    a.out_i = 1;
    a.n_lanes = n_cols;
    a.flat_lane = 0;  // lanes are whole columns
    a.in_valid = n_valid;
    a.scale = ninv;
    return log_n == 0 ? launch_pass<0>(a, inverse, 1, s) : launch_pass_dyn(log_n, a, inverse, 1, s);
  }
  if (!scratch) return cudaErrorInvalidValue;
  if (log_n <= 24) {
    const int l1 = ntt_split(log_n, n_valid < N), l2 = log_n - l1;
    const uint64_t N1 = 1ull << l1, N2 = 1ull << l2;
    // pass 1: DFT_{N2} over k2 (stride N1), lanes k1; transposed store into scratch
    PassArgs a = base_args(t, inverse);
    a.in = in;
    a.out = scratch;
    a.in_col = in_stride;
    a.out_col = N;
    a.in_lane = 1;
    a.in_m = N1;
    a.out_lane = 1;
    a.out_i = N1;
    a.n_lanes = N1;
    a.flat_lane = 1;  // flat index k = k2*N1 + k1
    a.in_valid = n_valid;
    a.sparse_nz = sparse_nz_for(n_valid, N, N1, N2);
    a.tw_log = log_n;
    // Passes of 2^11 and 2^12 build their twiddle factors in shared memory, unless
    // enough columns share the table: then the CTAs of one lane group run over all
    // columns back to back and read its entries from L2 (one load and one product
    // per element instead of two shared loads and two products).
    if (t.pass_tables && (!pass_tw_in_smem(l2) || n_cols >= kPassTabMinCols)) {
      a.tw_tab = pass_twiddle_table(t, log_n, l1, inverse, s);
      a.cols_fast = a.tw_tab && pass_tw_in_smem(l2) && (N1 >> pass_log_k(l2)) <= 65535;
    }
    a.pre = pre ? *pre : none;
    cudaError_t e = launch_pass_dyn(l2, a, inverse, n_cols, s);
    if (e != cudaSuccess) return e;
    // pass 2: DFT_{N1} over contiguous rows, lanes i2; natural-order store
    PassArgs b = base_args(t, inverse);
    b.in = scratch;
    b.out = out;
    b.in_col = N;
    b.out_col = out_stride;
    b.in_lane = N1;
    b.in_m = 1;
    b.out_lane = 1;
    b.out_i = N2;
    b.n_lanes = N2;
    b.flat_lane = N1;
    b.in_valid = N;
    b.scale = ninv;
    return launch_pass_dyn(l1, b, inverse, n_cols, s);
  }
  // three passes: N = A * B * C
  const int lc = (log_n + 2) / 3, lb = (log_n - lc + 1) / 2, la = log_n - lc - lb;
  const uint64_t A = 1ull << la, B = 1ull << lb, C = 1ull << lc, AB = A * B, BC = B * C;
  uint64_t* s1 = scratch;
  uint64_t* s2 = scratch + (uint64_t)n_cols * N;
  // pass 1: DFT_C over k3 (stride AB), lanes k1' < AB, twiddle w_N^{i3 k1'} -> s1[i3*AB + k1']
  PassArgs a = base_args(t, inverse);
  a.in = in;
  a.out = s1;
  a.in_col = in_stride;
  a.out_col = N;
  a.in_lane = 1;
  a.in_m = AB;
  a.out_lane = 1;
  a.out_i = AB;
  a.n_lanes = AB;
  a.flat_lane = 1;
  a.in_valid = n_valid;
  a.sparse_nz = sparse_nz_for(n_valid, N, AB, C);
  a.tw_log = log_n;
  a.pre = pre ? *pre : none;
  cudaError_t e = launch_pass_dyn(lc, a, inverse, n_cols, s);
  if (e != cudaSuccess) return e;
  // pass 2: per (column, i3): DFT_B over k2 (stride A) of lanes k1 < A, twiddle
  // w_{AB}^{i2 k1}, stored at s2[col*N + (i2*C + i3)*A + k1]
  PassArgs b = base_args(t, inverse);
  b.in = s1;
  b.out = s2;
  b.y_sub = (uint32_t)C;
  b.in_col = N;
  b.in_sub = AB;
  b.out_col = N;
  b.out_sub = A;
  b.in_lane = 1;
  b.in_m = A;
  b.out_lane = 1;
  b.out_i = C * A;
  b.n_lanes = A;
  b.flat_lane = 1;
  b.in_valid = AB;
  b.tw_log = la + lb;
  e = launch_pass_dyn(lb, b, inverse, (uint64_t)n_cols * C, s);
  if (e != cudaSuccess) return e;
  // pass 3: DFT_A over each contiguous row h' = i2*C + i3, stored at i1*BC + h'
  PassArgs c = base_args(t, inverse);
  c.in = s2;
  c.out = out;
  c.in_col = N;
  c.out_col = out_stride;
  c.in_lane = A;
  c.in_m = 1;
  c.out_lane = 1;
  c.out_i = BC;
  c.n_lanes = BC;
  c.flat_lane = A;
  c.in_valid = N;
  c.scale = ninv;
  return launch_pass_dyn(la, c, inverse, n_cols, s);
}

// ------------------------------------------------------------------ fused LDE -> leaf hash
// The forward transform of a zero-padded (LDE) column set whose last pass is a
// 2^7-point DFT fused with the Merkle leaf hash of the LDE rows: leaf r =
// SHA3(DsLabel{arity0, level 0xFFFFFFFF, position r, label} || row r of all
// w columns) (merkle/src/lib.rs:95-113, 391-476 over trace_import.rs:251-281's
// LDE). A CTA owns 4 consecutive last-pass lanes h (rows i1 * BC + h, i1 < 128):
// 512 rows, one per thread, whose sponge states stay in registers while the CTA
// walks the columns 16 at a time: it stages the 64 lanes' last-pass inputs of 16
// columns in shared memory, runs the two Stockham stages (radix 16, radix 8) of
// the 128-point DFT, and each thread absorbs its row's 16 values. The LDE itself
// need not be written (only its first keep_cols columns are, e.g. the column a
// STIR proof takes next): the 8 + 64 bytes per row that reach the tree replace the
// LDE write and the leaf kernel's full re-read.
namespace {

constexpr int kFuseLogA = 7, kFuseA = 1 << kFuseLogA;
constexpr int kFuseLanes = 4, kFuseCols = 16;
constexpr int kFuseTileLanes = kFuseLanes * kFuseCols;          // 64 DFT lanes per tile
constexpr int kFuseThreads = kFuseTileLanes * kFuseA / 16;      // 512 = rows per CTA
constexpr int kFuseMp = kFuseA + (kFuseA >> 4);                 // padded lane stride in shared memory
static_assert(kFuseThreads == kFuseLanes * kFuseA, "one hashing thread per row");
static_assert(pass_log_k(kFuseLogA) == 6 && row_stride(kFuseLogA) == kFuseMp,
              "the tile has the shape of a 2^7 pass");

struct LeafFuse {
  const uint64_t* in;  // last-pass input: column c, lane h, point m at in + c * N + h * 128 + m
  uint64_t N, BC;      // LDE length; row of (i1, lane h) = i1 * BC + h
  uint32_t w, keep_cols;
  uint64_t arity0, label;
  uint64_t* leaves;  // N digests (level 0 of the tree)
  uint64_t* out;     // the LDE's first keep_cols columns (column stride N), or null
  const uint64_t* tw_st;
};

__global__ void __launch_bounds__(kFuseThreads, 1) lde_leaf_kernel(LeafFuse a) {
  extern __shared__ uint64_t sm[];
  uint64_t* stw = sm + kFuseTileLanes * kFuseMp;
  const int t = threadIdx.x;
  __builtin_assume(t < kFuseThreads);
  const uint64_t lane0 = (uint64_t)blockIdx.x * kFuseLanes;
  for (int j = t; j < kFuseA; j += kFuseThreads) stw[j] = __ldg(a.tw_st + (j << (12 - kFuseLogA)));
  // this thread's row: lane hl, point hi1 (consecutive threads: consecutive points,
  // conflict-free shared reads)
  const int hl = t / kFuseA, hi1 = t % kFuseA;
  const uint64_t row = (uint64_t)hi1 * a.BC + lane0 + hl;
  kc::LaneSponge sp;
  sp.init();
  sp.lane(a.arity0);
  sp.lane(0xFFFFFFFFull);
  sp.lane(row);
  sp.lane(a.label);
#pragma unroll 1
  for (uint32_t c0 = 0; c0 < a.w; c0 += kFuseCols) {
    // tile lane L = cc * 4 + l: column c0 + cc, last-pass lane lane0 + l (128 contiguous inputs)
#pragma unroll 4
    for (int e = t; e < kFuseTileLanes * kFuseA; e += kFuseThreads) {
      const int L = e >> kFuseLogA, m = e & (kFuseA - 1);
      const int cc = L / kFuseLanes, l = L % kFuseLanes;
      sm[L * kFuseMp + padi(m)] = __ldg(a.in + (uint64_t)(c0 + cc) * a.N + (lane0 + l) * kFuseA + m);
    }
    __syncthreads();
    stockham_stage<16, 16, false, kFuseLogA, true>(sm, t, kFuseThreads, kFuseLogA, kFuseMp, 0, stw);
    stockham_stage<8, 16, false, kFuseLogA, true>(sm, t, kFuseThreads, kFuseLogA, kFuseMp, 4, stw);
#pragma unroll 1
    for (int cc = 0; cc < kFuseCols; ++cc) {
      const uint64_t v = sm[(cc * kFuseLanes + hl) * kFuseMp + padi(hi1)];
      sp.lane(v);
      if (c0 + cc < a.keep_cols) a.out[(uint64_t)(c0 + cc) * a.N + row] = v;
    }
    __syncthreads();  // the next tile overwrites the shared rows
  }
  uint64_t d[kc::kDigestLanes];
  sp.finish(d);
#pragma unroll
  for (int q = 0; q < kc::kDigestLanes; ++q) a.leaves[(uint64_t)kc::kDigestLanes * row + q] = d[q];
}

}  // namespace

bool lde_leaf_ok(uint32_t w, int log_n) {
  return w >= kFuseCols && w % kFuseCols == 0 && log_n >= kFuseLogA + 2 && log_n <= kFuseLogA + 24;
}

uint64_t lde_leaf_scratch_elems(uint32_t w, int log_n) {
  const int r = log_n - kFuseLogA;
  return (r <= 12 ? 1ull : 2ull) * w * (1ull << log_n);
}

// The passes before the fused one, for columns c0 .. c0 + wc - 1 of a w-column
// transform (column c's input at in + c in_stride; scratch as lde_leaf_transform's).
// Every pass works column by column, so a host-input pipeline can run them
// chunk by chunk as the chunks arrive.
cudaError_t lde_leaf_prepasses(const NttTables& t, const uint64_t* in, uint64_t in_stride, uint32_t w, uint32_t c0,
                               uint32_t wc, int log_n, uint64_t n_valid, const PowSpec* pre, uint64_t* scratch,
                               cudaStream_t s) {
  if (!lde_leaf_ok(w, log_n) || !scratch || c0 + wc > w) return cudaErrorInvalidValue;
  if (wc == 0) return cudaSuccess;
  const uint64_t N = 1ull << log_n, A = kFuseA;
  if (n_valid > N) n_valid = N;
  const PowSpec none{};
  const int r = log_n - kFuseLogA;
  in += (uint64_t)c0 * in_stride;
  if (r <= 12) {
    // four-step with N1 = 2^7: pass 1 as ntt_batch's, transposed into scratch
    const uint64_t N2 = 1ull << r;
    PassArgs a = base_args(t, false);
    a.in = in;
    a.out = scratch;
    a.in_col = in_stride;
    a.out_col = N;
    a.in_lane = 1;
    a.in_m = A;
    a.out_lane = 1;
    a.out_i = A;
    a.n_lanes = A;
    a.flat_lane = 1;
    a.in_valid = n_valid;
    a.sparse_nz = sparse_nz_for(n_valid, N, A, N2);
    a.tw_log = log_n;
    a.pre = pre ? *pre : none;
    a.out = scratch + (uint64_t)c0 * N;
    return launch_pass_dyn(r, a, false, wc, s);
  } else {
    // three passes N = A * B * C, as ntt_batch's, with C and B as even as possible
    // (2^8 x 2^8 for a 2^23 domain): every pass then fills its CTAs' lanes, where
    // C = 2^12 would leave a 2^(r - 12)-point middle pass with mostly idle lanes
    const int lc = (r + 1) / 2, lb = r - lc;
    const uint64_t B = 1ull << lb, C = 1ull << lc, AB = A * B;
    uint64_t* s1 = scratch + (uint64_t)c0 * N;
    uint64_t* s2 = scratch + (uint64_t)w * N + (uint64_t)c0 * N;
    PassArgs a = base_args(t, false);
    a.in = in;
    a.out = s1;
    a.in_col = in_stride;
    a.out_col = N;
    a.in_lane = 1;
    a.in_m = AB;
    a.out_lane = 1;
    a.out_i = AB;
    a.n_lanes = AB;
    a.flat_lane = 1;
    a.in_valid = n_valid;
    a.sparse_nz = sparse_nz_for(n_valid, N, AB, C);
    a.tw_log = log_n;
    a.pre = pre ? *pre : none;
    cudaError_t e = launch_pass_dyn(lc, a, false, wc, s);
    if (e != cudaSuccess) return e;
    PassArgs b = base_args(t, false);
    b.in = s1;
    b.out = s2;
    b.y_sub = (uint32_t)C;
    b.in_col = N;
    b.in_sub = AB;
    b.out_col = N;
    b.out_sub = A;
    b.in_lane = 1;
    b.in_m = A;
    b.out_lane = 1;
    b.out_i = C * A;
    b.n_lanes = A;
    b.flat_lane = 1;
    b.in_valid = AB;
    b.tw_log = kFuseLogA + lb;
    return launch_pass_dyn(lb, b, false, (uint64_t)wc * C, s);
  }
}

// The fused last pass over all w columns, after lde_leaf_prepasses covered them.
cudaError_t lde_leaf_final(const NttTables& t, uint32_t w, int log_n, const uint64_t* scratch, uint64_t arity0,
                           uint64_t label, uint64_t* leaves, uint64_t* out, uint32_t keep_cols, cudaStream_t s) {
  if (!lde_leaf_ok(w, log_n) || !scratch || !leaves || keep_cols > w || (keep_cols && !out))
    return cudaErrorInvalidValue;
  const uint64_t N = 1ull << log_n;
  const int r = log_n - kFuseLogA;
  const uint64_t* last_in = r <= 12 ? scratch : scratch + (uint64_t)w * N;
  const uint64_t BC = N >> kFuseLogA;
  LeafFuse f{last_in, N, BC, w, keep_cols, arity0, label, leaves, out, t.d_fwd_st};
  const size_t smem = ((size_t)kFuseTileLanes * kFuseMp + kFuseA) * sizeof(uint64_t);
  cudaError_t e = cudaFuncSetAttribute(lde_leaf_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  SG_LAUNCH_SCOPE("lde_leaf", s);
  lde_leaf_kernel<<<(unsigned)(BC / kFuseLanes), kFuseThreads, smem, s>>>(f);
  return cudaGetLastError();
}

cudaError_t lde_leaf_transform(const NttTables& t, const uint64_t* in, uint64_t in_stride, uint32_t w, int log_n,
                               uint64_t n_valid, const PowSpec* pre, uint64_t* scratch, uint64_t arity0,
                               uint64_t label, uint64_t* leaves, uint64_t* out, uint32_t keep_cols, cudaStream_t s) {
  cudaError_t e = lde_leaf_prepasses(t, in, in_stride, w, 0, w, log_n, n_valid, pre, scratch, s);
  if (e != cudaSuccess) return e;
  return lde_leaf_final(t, w, log_n, scratch, arity0, label, leaves, out, keep_cols, s);
}

}  // namespace sg

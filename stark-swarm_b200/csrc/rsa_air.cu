// rsa_air.cu — device kernels of the RSA-2048 AIR: trace expansion from the
// per-row witnesses, and Phi = sum_j lambda_j C_j at the LDE points
// (deep_ali_merge_rsa_exp_multirow(_streaming) / deep_ali_merge_rsa_stacked_streaming,
// lib.rs:1694-2070, with lambda_j = j + 1 over the concatenated constraints).
//
// Phi layout: one CTA per (4 consecutive LDE points, record). The 4 points are
// one 32-byte sector of every column, so each cell load of the CTA is one
// sector for 4 threads; the points share their trace row (blowup >= 4). The
// limbs the slot identities convolve (acc, op2, q, n, c) and the 158 signed
// carries are staged in shared memory; every other constraint reads its cells
// directly. Each thread accumulates lambda_j C_j for one point; a warp shuffle
// and a shared-memory pass reduce the 256 partial sums to the 4 points.
#include "context.hpp"
#include "counters.hpp"
#include "gl.cuh"
#include "rsa_air.cuh"

namespace sg {
namespace {

using namespace rsa;

constexpr int kPts = 4, kThreads = 256;

__global__ void rsa_expand_kernel(const RecordW* recs, const RowW* rows, uint64_t n_records, uint64_t* trace) {
  const uint64_t total = n_records * WIDTH * N_TRACE;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t row = (uint32_t)(e % N_TRACE);
    const uint64_t gcol = e / N_TRACE, r = gcol / WIDTH;
    trace[e] = cell(recs[r], rows[r * N_TRACE + row], (uint32_t)(gcol - r * WIDTH));
  }
}

// lambda C summed in a field accumulator
struct Acc {
  uint64_t v = 0;
  __device__ __forceinline__ void put(uint64_t lambda, uint64_t c) { v = gl::add(v, gl::mul(lambda, c)); }
};

// sum_b 2^b x_b for b < nb (Horner from the top bit), over field cells
__device__ __forceinline__ uint64_t pack_bits(const uint64_t* col0, uint64_t n, uint32_t nb) {
  uint64_t s = 0;
  for (int b = (int)nb - 1; b >= 0; --b) s = gl::add(gl::add(s, s), __ldg(col0 + (uint64_t)b * n));
  return s;
}

__global__ void __launch_bounds__(kThreads) rsa_phi_kernel(const uint64_t* lde, uint64_t n, uint64_t blowup,
                                                           uint64_t n_trace, uint64_t* phi_part) {
  const uint64_t i0 = (uint64_t)blockIdx.x * kPts, rec = blockIdx.y;
  const uint64_t row = i0 / blowup;
  const bool trans = row + 1 < n_trace, out_row = row == OUTPUT_ROW;
  const uint64_t nx0 = (i0 + blowup) % n;  // next-row points: nx0 .. nx0 + 3 (blowup % 4 == 0)
  const uint64_t* L = lde + rec * (uint64_t)WIDTH * n;
  const uint64_t lam0 = rec * (uint64_t)CONSTRAINTS + 1;  // lambda_j = global index + 1
  const int t = threadIdx.x, p = t & (kPts - 1);
  auto cur = [&](uint32_t col) { return __ldg(L + (uint64_t)col * n + i0 + p); };
  auto nxt = [&](uint32_t col) { return __ldg(L + (uint64_t)col * n + nx0 + p); };

  __shared__ uint64_t sa[LIMBS][kPts], sb[LIMBS][kPts], sq[LIMBS][kPts], sn[LIMBS][kPts], sc[LIMBS][kPts];
  __shared__ uint64_t sk[CARRY_POS][kPts];  // signed carries sum_b 2^b bit - 2^39
  for (int e = t; e < (int)(LIMBS * kPts); e += kThreads) {
    const int i = e / kPts;
    sa[i][p] = cur(ACC + i);
    sb[i][p] = cur(OP2 + i);
    sq[i][p] = cur(Q + i);
    sn[i][p] = cur(N + i);
    sc[i][p] = cur(C + i);
  }
  for (int e = t; e < (int)(CARRY_POS * kPts); e += kThreads) {
    const int k = e / kPts;
    sk[k][p] = gl::sub(pack_bits(L + (uint64_t)(CARRY + k * CARRY_BITS) * n + i0 + p, n, CARRY_BITS),
                       CARRY_OFFSET);
  }
  __syncthreads();

  Acc acc;
  const uint64_t phase = cur(PHASE);
  if (t < kPts) acc.put(lam0 + K_PHASE, gl::mul(phase, gl::sub(1, phase)));
  // select
  for (int e = t; e < (int)(LIMBS * kPts); e += kThreads) {
    const int i = e / kPts;
    const uint64_t a = sa[i][p];
    const uint64_t target = gl::add(gl::mul(phase, gl::sub(cur(S + i), a)), a);
    acc.put(lam0 + K_SELECT + i, gl::sub(sb[i][p], target));
  }
  // booleanity of the c bits, q bits and carry bits
  for (int e = t; e < (int)(2 * LIMBS * LIMB_BITS * kPts); e += kThreads) {
    const int j = e / kPts;  // 0 .. 4159: c bits then q bits
    const bool is_c = j < (int)(LIMBS * LIMB_BITS);
    const uint32_t off = is_c ? j : j - LIMBS * LIMB_BITS;
    const uint64_t x = cur((is_c ? C_BITS : Q_BITS) + off);
    acc.put(lam0 + (is_c ? K_CBOOL : K_QBOOL) + off, gl::mul(x, gl::sub(1, x)));
  }
  for (int e = t; e < (int)(CARRY_POS * CARRY_BITS * kPts); e += kThreads) {
    const int j = e / kPts;
    const uint64_t x = cur(CARRY + j);
    acc.put(lam0 + K_CARRY + j, gl::mul(x, gl::sub(1, x)));
  }
  // limb packs
  for (int e = t; e < (int)(2 * LIMBS * kPts); e += kThreads) {
    const int j = e / kPts;
    const bool is_c = j < (int)LIMBS;
    const int i = is_c ? j : j - LIMBS;
    const uint64_t bits = pack_bits(L + (uint64_t)((is_c ? C_BITS : Q_BITS) + i * LIMB_BITS) * n + i0 + p, n,
                                    LIMB_BITS);
    acc.put(lam0 + (is_c ? K_CPACK : K_QPACK) + i, gl::sub(is_c ? sc[i][p] : sq[i][p], bits));
  }
  // slot identities: sum a_i b_{k-i} - sum q_i n_{k-i} - c_k + carry_{k-1} - 2^26 carry_k
  for (int e = t; e < (int)(SLOTS * kPts); e += kThreads) {
    const int k = e / kPts;
    const int lo = k >= (int)LIMBS - 1 ? k - (int)(LIMBS - 1) : 0, hi = k < (int)LIMBS - 1 ? k : LIMBS - 1;
    uint64_t ab = 0, qn = 0;
    for (int i = lo; i <= hi; ++i) {
      ab = gl::add(ab, gl::mul(sa[i][p], sb[k - i][p]));
      qn = gl::add(qn, gl::mul(sq[i][p], sn[k - i][p]));
    }
    uint64_t v = gl::sub(ab, qn);
    if (k < (int)LIMBS) v = gl::sub(v, sc[k][p]);
    if (k > 0) v = gl::add(v, sk[k - 1][p]);
    if (k < (int)CARRY_POS) v = gl::sub(v, gl::mul_pow2(sk[k][p], LIMB_BITS));
    acc.put(lam0 + K_SLOT + k, v);
  }
  // row-16 boundary and the transitions (zero elsewhere: no contribution)
  if (out_row)
    for (int e = t; e < (int)(LIMBS * kPts); e += kThreads) {
      const int i = e / kPts;
      acc.put(lam0 + K_EM + i, gl::sub(sc[i][p], cur(EM + i)));
    }
  if (trans)
    for (int e = t; e < (int)(4 * LIMBS * kPts); e += kThreads) {
      const int j = e / kPts, g = j / LIMBS, i = j - g * LIMBS;
      uint64_t v;
      if (g == 0)
        v = gl::sub(nxt(ACC + i), sc[i][p]);
      else {
        const uint32_t col = (g == 1 ? S : g == 2 ? N : EM) + i;
        v = gl::sub(nxt(col), cur(col));
      }
      acc.put(lam0 + K_TRANS + j, v);
    }

  // reduce the threads of each point: lanes l, l + 4, ... share a point
  uint64_t v = acc.v;
#pragma unroll
  for (int o = 16; o >= kPts; o >>= 1) v = gl::add(v, __shfl_down_sync(0xffffffffu, v, o));
  __shared__ uint64_t red[kThreads / 32][kPts];
  if ((t & 31) < kPts) red[t >> 5][p] = v;
  __syncthreads();
  if (t < kPts) {
    uint64_t s = 0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) s = gl::add(s, red[w][t]);
    phi_part[rec * n + i0 + t] = s;
  }
}

__global__ void sum_records_kernel(const uint64_t* part, uint64_t n, uint64_t n_records, uint64_t* phi) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint64_t s = 0;
  for (uint64_t r = 0; r < n_records; ++r) s = gl::add(s, part[r * n + i]);
  phi[i] = s;
}

}  // namespace

cudaError_t rsa_expand(const RecordW* d_recs, const RowW* d_rows, uint64_t n_records, uint64_t* d_trace,
                       cudaStream_t s) {
  const uint64_t total = n_records * WIDTH * N_TRACE;
  const unsigned blocks = (unsigned)std::min<uint64_t>((total + 255) / 256, 148ull * 16);
  SG_LAUNCH_SCOPE("rsa_expand", s);
  rsa_expand_kernel<<<blocks, 256, 0, s>>>(d_recs, d_rows, n_records, d_trace);
  return cudaGetLastError();
}

cudaError_t rsa_phi(const uint64_t* d_lde, uint64_t n_records, uint64_t n_trace, uint64_t blowup, uint64_t* d_part,
                    uint64_t* d_phi, cudaStream_t s) {
  const uint64_t n = n_trace * blowup;
  if (blowup % kPts || n % kPts || n_records == 0 || n_records > 65535) return cudaErrorInvalidValue;
  {
    SG_LAUNCH_SCOPE("rsa_phi", s);
    rsa_phi_kernel<<<dim3((unsigned)(n / kPts), (unsigned)n_records), kThreads, 0, s>>>(
        d_lde, n, blowup, n_trace, n_records == 1 ? d_phi : d_part);
  }
  if (n_records > 1) {
    SG_LAUNCH_SCOPE("rsa_phi_sum", s);
    sum_records_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(d_part, n, n_records, d_phi);
  }
  return cudaGetLastError();
}

}  // namespace sg

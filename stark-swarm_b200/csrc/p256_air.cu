// p256_air.cu — device kernels of the P-256 double-chain AIR: trace expansion
// from the row witnesses, and Phi = sum_j lambda_j C_j at every LDE point
// (deep_ali_merge_ecdsa_double_multirow_streaming, lambda_j = j + 1), evaluated
// gadget by gadget from the row's gadget table.
//
// Phi layout: one thread per LDE point, so each cell load of a warp reads 32
// consecutive points of one column (256 contiguous bytes). grid.y splits the
// row's 260 gadgets (and the 180 tail slots) into chunks of about equal
// constraint count; each (point block, chunk) CTA writes one partial sum per
// point, and a second kernel adds the chunks. Every constraint is folded into
// the accumulator as it is formed (its lambda is its index + 1), so no
// constraint vector is ever stored; range checks form booleanity and the limb
// pack in one pass over the bits.
#include <algorithm>

#include "context.hpp"
#include "counters.hpp"
#include "gl.cuh"
#include "p256_air.cuh"
#include "p256_cells.cuh"

namespace sg {
namespace {

using namespace p256;

__constant__ uint64_t kPT[NL] = {0x3FFFFFF, 0x3FFFFFF, 0x3FFFFFF, 0x003FFFF, 0, 0, 0, 0x0000400, 0x3FF0000, 0x03FFFFF};

__global__ void p256_expand_kernel(P256Dev d, uint64_t k, uint64_t* trace) {
  const uint64_t total = (uint64_t)d.width * k;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t col = e / k, row = e - col * k;
    trace[e] = cell_value(d.cell_code[col], d.table, d.rows[row], d.gw + row * d.n_gadgets, d.rproj, d.b);
  }
}

// Phi accumulates lam_j C_j (lam_j <= 155,775 < 2^32) in 128 bits and reduces
// once per chunk: a term is 7 instructions instead of a field product and add.
struct Ctx {
  const uint64_t* L;  // column 0 at this point: cell c is L[c * n]
  uint64_t n;
  gl::Acc128 acc;
  __device__ __forceinline__ uint64_t v(uint32_t c) const { return __ldg(L + (uint64_t)c * n); }
  __device__ __forceinline__ void put(uint64_t lam, uint64_t c) { acc.add_mul32((uint32_t)lam, c); }
};

// 128 threads and at most 128 registers: 4 CTAs (16 warps) per SM. Measured for
// n = 8192: 3.8 ms, against 4.0 ms at 3 CTAs (168 registers) and 4.1 ms at 5 (96).
constexpr int kPhiThreads = 128;

// Booleanity terms t_b (1 - t_b) with lambdas lam + b for the NB bit cells
// bits .. bits+NB-1, added into *acc, and the pack sum_b t_b 2^b (reduced). The
// loads of a batch go out together. One out-of-line copy serves every range
// check and carry: inlined at each, the unrolled bodies overflowed the
// instruction cache.
template <int NB>
__device__ __noinline__ uint64_t bits_pack(const uint64_t* L, uint64_t n, uint32_t bits, uint32_t lam,
                                           gl::Acc128* acc) {
  constexpr int H = NB > LB ? NB / 2 : NB;  // loads per batch: 26, or 2 x 18 for a 36-bit carry
  static_assert(NB % H == 0 && NB <= 64, "bit batch");
  gl::Acc128 a = *acc, s;
#pragma unroll
  for (int h = 0; h < NB / H; ++h) {
    uint64_t t[H];
#pragma unroll
    for (int j = 0; j < H; ++j) t[j] = __ldg(L + (uint64_t)(bits + h * H + j) * n);
#pragma unroll
    for (int j = 0; j < H; ++j) {
      const int b = h * H + j;
      a.add_mul32(lam + b, gl::mul(t[j], gl::sub(1, t[j])));
      if (b < 32)
        s.add_shl(t[j], b);
      else
        s.add_shl32(t[j], b - 32);
    }
  }
  *acc = a;
  return s.reduce();
}

// booleanity of the 260 bits at lam .. lam+259, limb packs at lam+260 .. lam+269
__device__ __forceinline__ void range(Ctx& x, uint32_t limbs, uint32_t bits, uint64_t lam) {
  gl::Acc128 a = x.acc;
#pragma unroll 1
  for (uint32_t i = 0; i < NL; ++i) {
    const uint64_t s = bits_pack<LB>(x.L, x.n, bits + i * LB, (uint32_t)(lam + i * LB), &a);
    a.add_mul32((uint32_t)(lam + NL * LB + i), gl::sub(x.v(limbs + i), s));
  }
  x.acc = a;
}

__device__ void eval_mul(Ctx& x, const Gadget& g, uint64_t lam) {
  const uint32_t a = g.p[0], b = g.p[1], c = g.p[2], q = g.p[4], cy = g.p[6];
  range(x, c, g.p[3], lam);
  range(x, q, g.p[5], lam + ELEM);
  // the 18 biased carries, staged per thread in shared memory so that the loop
  // over them stays rolled while the slot identities below index them statically
  __shared__ uint64_t s_carry[MUL_CP][kPhiThreads];
  const uint64_t lam_b = lam + 2 * ELEM + MUL_SP;
  {
    gl::Acc128 acc = x.acc;
#pragma unroll 1
    for (uint32_t k = 0; k < MUL_CP; ++k)
      s_carry[k][threadIdx.x] =
          gl::sub(bits_pack<MUL_CB>(x.L, x.n, cy + k * MUL_CB, (uint32_t)(lam_b + k * MUL_CB), &acc),
                  1ull << (MUL_CB - 1));
    x.acc = acc;
  }
  uint64_t al[NL], bl[NL], ql[NL];
#pragma unroll
  for (uint32_t i = 0; i < NL; ++i) {
    al[i] = x.v(a + i);
    bl[i] = x.v(b + i);
    ql[i] = x.v(q + i);
  }
#pragma unroll
  for (uint32_t k = 0; k < MUL_SP; ++k) {
    uint64_t ab = 0, qp = 0;
#pragma unroll
    for (uint32_t i = 0; i < NL; ++i) {
      if (i + NL - 1 < k || i > k) continue;
      ab = gl::add(ab, gl::mul(al[i], bl[k - i]));
      qp = gl::add(qp, gl::mul(ql[i], kPT[k - i]));
    }
    uint64_t v = gl::sub(ab, qp);
    if (k < NL) v = gl::sub(v, x.v(c + k));
    if (k > 0) v = gl::add(v, s_carry[k - 1][threadIdx.x]);
    if (k < MUL_CP) v = gl::sub(v, gl::mul_pow2(s_carry[k][threadIdx.x], LB));
    x.put(lam + 2 * ELEM + k, v);
  }
}

__device__ void eval_add(Ctx& x, const Gadget& g, uint64_t lam) {
  const uint32_t a = g.p[0], b = g.p[1], c = g.p[2], cr = g.p[4];
  range(x, c, g.p[3], lam);
  uint64_t prev = 0;
#pragma unroll 1
  for (uint32_t k = 0; k < NL; ++k) {
    const uint64_t ck = x.v(cr + k);
    const uint64_t v = gl::sub(gl::add(gl::add(x.v(a + k), x.v(b + k)), prev),
                               gl::add(x.v(c + k), gl::mul_pow2(ck, LB)));
    x.put(lam + ELEM + k, v);
    if (k + 1 < NL)
      x.put(lam + ELEM + NL + k, gl::mul(ck, gl::sub(1, ck)));
    else
      x.put(lam + ELEM + 2 * NL - 1, ck);
    prev = ck;
  }
}

// shared by sub (sign +1: a + P - b) and freeze (sign -1: a - P - diff)
__device__ void pos_neg_rules(Ctx& x, uint32_t pos, uint32_t neg, uint64_t lam) {
#pragma unroll 1
  for (uint32_t k = 0; k < NL; ++k) {
    const uint64_t cp = x.v(pos + k), cn = x.v(neg + k);
    x.put(lam + k, gl::mul(cp, gl::sub(1, cp)));
    x.put(lam + NL + k, gl::mul(cn, gl::sub(1, cn)));
    x.put(lam + 2 * NL + k, gl::mul(cp, cn));
  }
}

__device__ void eval_sub(Ctx& x, const Gadget& g, uint64_t lam) {
  const uint32_t a = g.p[0], b = g.p[1], c = g.p[2], pos = g.p[4], neg = g.p[5];
  range(x, c, g.p[3], lam);
  uint64_t prev = 0;
#pragma unroll 1
  for (uint32_t k = 0; k < NL; ++k) {
    const uint64_t net = gl::sub(x.v(pos + k), x.v(neg + k));
    const uint64_t v = gl::sub(gl::add(gl::sub(gl::add(x.v(a + k), kPT[k]), x.v(b + k)), prev),
                               gl::add(x.v(c + k), gl::mul_pow2(net, LB)));
    x.put(lam + ELEM + k, v);
    prev = net;
  }
  pos_neg_rules(x, pos, neg, lam + ELEM + NL);
  x.put(lam + ELEM + 4 * NL, gl::add(x.v(pos + NL - 1), x.v(neg + NL - 1)));
}

__device__ void eval_freeze(Ctx& x, const Gadget& g, uint64_t lam) {
  const uint32_t a = g.p[0], d = g.p[1], c = g.p[3], pos = g.p[5], neg = g.p[6];
  range(x, d, g.p[2], lam);
  range(x, c, g.p[4], lam + ELEM);
  uint64_t prev = 0;
#pragma unroll 1
  for (uint32_t k = 0; k < NL; ++k) {
    const uint64_t net = gl::sub(x.v(pos + k), x.v(neg + k));
    const uint64_t v = gl::sub(gl::add(gl::sub(x.v(a + k), kPT[k]), prev),
                               gl::add(x.v(d + k), gl::mul_pow2(net, LB)));
    x.put(lam + 2 * ELEM + k, v);
    prev = net;
  }
  pos_neg_rules(x, pos, neg, lam + 2 * ELEM + NL);
  x.put(lam + 2 * ELEM + 4 * NL, x.v(pos + NL - 1));
  const uint64_t n9 = x.v(neg + NL - 1);
#pragma unroll 1
  for (uint32_t k = 0; k < NL; ++k) {
    const uint64_t ak = x.v(a + k), dk = x.v(d + k);
    x.put(lam + 2 * ELEM + 4 * NL + 1 + k, gl::sub(gl::sub(x.v(c + k), dk), gl::mul(n9, gl::sub(ak, dk))));
  }
}

__device__ void eval_select(Ctx& x, const Gadget& g, uint64_t lam) {
  const uint32_t a = g.p[0], b = g.p[1], c = g.p[2];
  range(x, c, g.p[3], lam);
  const uint64_t s = x.v(g.p[4]);
#pragma unroll 1
  for (uint32_t k = 0; k < NL; ++k) {
    const uint64_t ak = x.v(a + k), bk = x.v(b + k);
    x.put(lam + ELEM + k, gl::sub(gl::sub(x.v(c + k), bk), gl::mul(s, gl::sub(ak, bk))));
  }
  x.put(lam + ELEM + NL, gl::mul(s, gl::sub(1, s)));
}

// boundary (last row) and transition (rows + 1 < n_trace) slots
__device__ void eval_tail(Ctx& x, const uint64_t* nxt, const uint32_t* tail, bool last, bool trans, uint64_t lam) {
  if (last) {
#pragma unroll 1
    for (uint32_t j = 0; j < 6; ++j) {
      const uint32_t c = tail[6 * (j / 3) + 3 + j % 3], r = tail[12 + j];
      for (uint32_t i = 0; i < NL; ++i) x.put(lam + NL * j + i, gl::sub(x.v(c + i), x.v(r + i)));
    }
  }
  if (trans) {
    auto nv = [&](uint32_t c) { return __ldg(nxt + (uint64_t)c * x.n); };
#pragma unroll 1
    for (uint32_t j = 0; j < 6; ++j) {
      const uint32_t acc = tail[6 * (j / 3) + j % 3], c = tail[6 * (j / 3) + 3 + j % 3];
      for (uint32_t i = 0; i < NL; ++i) x.put(lam + 60 + NL * j + i, gl::sub(nv(acc + i), x.v(c + i)));
    }
#pragma unroll 1
    for (uint32_t j = 0; j < 6; ++j) {
      const uint32_t r = tail[12 + j];
      for (uint32_t i = 0; i < NL; ++i) x.put(lam + 120 + NL * j + i, gl::sub(nv(r + i), x.v(r + i)));
    }
  }
}

__global__ void __launch_bounds__(kPhiThreads, 4) p256_phi_kernel(P256Phi a, uint64_t* part) {
  const uint64_t i = blockIdx.x * (uint64_t)kPhiThreads + threadIdx.x;
  if (i >= a.n) return;
  const uint32_t ch = blockIdx.y;
  Ctx x{a.lde + i, a.n, {}};
  const uint32_t g0 = a.chunk[ch], g1 = a.chunk[ch + 1];
  for (uint32_t gi = g0; gi < g1; ++gi) {
    const Gadget g = a.table[gi];
    const uint64_t lam = (uint64_t)a.lam_base[gi] + 1;
    switch (g.kind) {
      case G_MUL: eval_mul(x, g, lam); break;
      case G_ADD: eval_add(x, g, lam); break;
      case G_SUB: eval_sub(x, g, lam); break;
      case G_FREEZE: eval_freeze(x, g, lam); break;
      default: eval_select(x, g, lam); break;
    }
  }
  if (g1 == a.n_gadgets && ch + 1 == gridDim.y) {
    uint64_t row, nx;
    if (a.coset_len == 0) {
      row = i / a.blowup;
      nx = (i + a.blowup) % a.n;
    } else {
      const uint64_t c = i / a.coset_len, p = i - c * a.coset_len;
      row = p;
      nx = c * a.coset_len + (p + 1 == a.coset_len ? 0 : p + 1);
    }
    eval_tail(x, a.lde + nx, a.tail, row + 1 == a.n_trace, row + 1 < a.n_trace, (uint64_t)a.lam_tail + 1);
  }
  part[(uint64_t)ch * a.n + i] = x.acc.reduce();
}

__global__ void p256_sum_kernel(const uint64_t* part, uint64_t n, uint32_t chunks, uint64_t* phi, uint64_t coset_len,
                                uint64_t out_stride, uint64_t out_off) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint64_t s = 0;
  for (uint32_t c = 0; c < chunks; ++c) s = gl::add(s, part[(uint64_t)c * n + i]);
  if (coset_len == 0) {
    phi[i] = s;
  } else {
    const uint64_t c = i / coset_len;
    phi[out_off + c + out_stride * (i - c * coset_len)] = s;
  }
}

}  // namespace

std::vector<uint32_t> p256_chunks(uint32_t target_constraints) {
  const p256::Layout& L = p256::layout();
  std::vector<uint32_t> ch{0};
  uint32_t acc = 0;
  for (uint32_t gi = 0; gi < L.table.size(); ++gi) {
    acc += p256::gadget_constraints(L.table[gi].kind);
    if (acc >= target_constraints) {
      ch.push_back(gi + 1);
      acc = 0;
    }
  }
  if (ch.back() != L.table.size()) ch.push_back((uint32_t)L.table.size());
  return ch;
}

cudaError_t p256_expand(const P256Dev& d, uint64_t k, uint64_t* d_trace, cudaStream_t s) {
  const uint64_t total = (uint64_t)d.width * k;
  const unsigned blocks = (unsigned)std::min<uint64_t>((total + 255) / 256, 148ull * 32);
  SG_LAUNCH_SCOPE("p256_expand", s);
  p256_expand_kernel<<<blocks, 256, 0, s>>>(d, k, d_trace);
  return cudaGetLastError();
}

cudaError_t p256_phi(const P256Phi& a, uint32_t n_chunks, uint64_t* d_part, uint64_t* d_phi, cudaStream_t s) {
  if (a.blowup == 0 || a.n % (a.coset_len ? a.coset_len : a.blowup) || n_chunks == 0 || n_chunks > 65535)
    return cudaErrorInvalidValue;
  {
    SG_LAUNCH_SCOPE("p256_phi", s);
    p256_phi_kernel<<<dim3((unsigned)((a.n + kPhiThreads - 1) / kPhiThreads), n_chunks), kPhiThreads, 0, s>>>(
        a, d_part);
  }
  SG_LAUNCH_SCOPE("p256_phi_sum", s);
  p256_sum_kernel<<<(unsigned)((a.n + 255) / 256), 256, 0, s>>>(d_part, a.n, n_chunks, d_phi, a.coset_len,
                                                                 a.out_stride, a.out_off);
  return cudaGetLastError();
}

}  // namespace sg

// ed25519_air.cu — device kernels of the Ed25519 verify AIR: the trace expanded
// from per-row words and per-phase cell codes, and Phi = sum_j (j + 1) C_j at every
// LDE point (deep_ali_merge_ed25519_verify_streaming, lib.rs:854-974), each point
// evaluating only the blocks its row opens (eval_verify_air_v16_per_row emits zeros
// for the others, ed25519_verify_air.rs:4870-4960).
//
// Phi layout: one thread per LDE point, so a warp's cell loads read 32 consecutive
// points of one column. In the materialised LDE (blowup 32) a warp is the 32 points
// of one trace row and so of one class: the single-row classes (reduction,
// decompressions, residual, doublings, verdict) run without divergence. grid.y
// splits each class's blocks into chunks; a CTA writes one partial sum per point
// and chunk, and a second kernel adds them with the SHA-512 block's part.
#include <algorithm>
#include <map>

#include "context.hpp"
#include "counters.hpp"
#include "ed25519_air.cuh"
#include "gl.cuh"

namespace sg {
namespace {

using namespace ed25519;

__global__ void ed25519_expand_kernel(EdExpand d, uint64_t* trace) {
  const uint64_t total = (uint64_t)d.width * d.height;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t col = e / d.height, row = e - col * d.height;
    const uint32_t cd = __ldg(d.codes + (uint64_t)d.row_phase[row] * d.width + col);
    trace[e] = cell_value(cd, d.words + d.row_off[row], d.globals);
  }
}

constexpr int kPhiThreads = 128;
constexpr uint64_t kMulBias = 1ull << (MUL_CB - 1), kRedBias = 1ull << (RED_CB - 1);

struct Ctx {
  const uint64_t* L;  // cell c of this point at L[c * n]
  const uint64_t* N;  // the next row's point
  uint64_t n;
  gl::Acc128 acc;
  __device__ __forceinline__ uint64_t v(uint32_t c) const { return __ldg(L + (uint64_t)c * n); }
  __device__ __forceinline__ uint64_t w(uint32_t c) const { return __ldg(N + (uint64_t)c * n); }
  __device__ __forceinline__ void put(uint32_t lam, uint64_t x) { acc.add_mul32(lam, x); }
};

// Booleanity t_b (1 - t_b) with lambdas lam + b for the NB bit cells at bits ..,
// added into *acc, and their pack sum_b t_b 2^b (reduced). Loads go out in
// batches; one out-of-line copy per width keeps the instruction footprint small.
template <int NB>
__device__ __noinline__ uint64_t bits_pack(const uint64_t* L, uint64_t n, uint32_t bits, uint32_t lam,
                                           gl::Acc128* acc) {
  constexpr int H = NB > 26 ? NB / 2 : NB;
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

// 255 booleanity constraints at lam + 1 .., then the 10 limb packs at lam + 256 ..
__device__ __forceinline__ void range(Ctx& x, uint32_t limbs, uint32_t bits, uint32_t lam) {
  gl::Acc128 a = x.acc;
  uint32_t off = 0;
#pragma unroll 1
  for (uint32_t i = 0; i < NL; i += 2) {
    const uint64_t s0 = bits_pack<26>(x.L, x.n, bits + off, lam + 1 + off, &a);
    a.add_mul32(lam + 256 + i, gl::sub(x.v(limbs + i), s0));
    const uint64_t s1 = bits_pack<25>(x.L, x.n, bits + off + 26, lam + 1 + off + 26, &a);
    a.add_mul32(lam + 257 + i, gl::sub(x.v(limbs + i + 1), s1));
    off += 51;
  }
  x.acc = a;
}

__device__ __forceinline__ uint64_t mul_small(uint64_t x, uint32_t k) { return gl::mul(x, k); }

// eval_mul_gadget (ed25519_field_air.rs:1000-1076): range, 10 limb sums, 360 carry bits
__device__ void eval_mul(Ctx& x, const EdBlock& g) {
  const uint32_t a = g.p[0], b = g.p[1], c = g.p[2], cy = g.p[4], lam = g.lam;
  range(x, c, g.p[3], lam);
  __shared__ uint64_t s_carry[NL][kPhiThreads];
  {
    gl::Acc128 acc = x.acc;
#pragma unroll 1
    for (uint32_t k = 0; k < NL; ++k)
      s_carry[k][threadIdx.x] =
          gl::sub(bits_pack<MUL_CB>(x.L, x.n, cy + k * MUL_CB, lam + 276 + k * MUL_CB, &acc), kMulBias);
    x.acc = acc;
  }
  uint64_t al[NL], bl[NL];
#pragma unroll
  for (uint32_t i = 0; i < NL; ++i) {
    al[i] = x.v(a + i);
    bl[i] = x.v(b + i);
  }
  // diagonals: lo[k] = sum_{i+j=k} f a_i b_j, hi[k] = sum_{i+j=k+10} f a_i b_j, f = 2 for odd i, j
  uint64_t lo[NL], hi[NL];
#pragma unroll
  for (uint32_t k = 0; k < NL; ++k) lo[k] = hi[k] = 0;
#pragma unroll
  for (uint32_t i = 0; i < NL; ++i)
#pragma unroll
    for (uint32_t j = 0; j < NL; ++j) {
      uint64_t p = gl::mul(al[i], bl[j]);
      if ((i & 1) && (j & 1)) p = gl::add(p, p);
      if (i + j < NL)
        lo[i + j] = gl::add(lo[i + j], p);
      else
        hi[i + j - NL] = gl::add(hi[i + j - NL], p);
    }
#pragma unroll
  for (uint32_t k = 0; k < NL; ++k) {
    const uint64_t t = gl::add(lo[k], mul_small(hi[k], 19));
    const uint64_t cin = k == 0 ? mul_small(s_carry[NL - 1][threadIdx.x], 19) : s_carry[k - 1][threadIdx.x];
    const uint64_t v = gl::sub(gl::add(t, cin), gl::add(x.v(c + k), gl::mul_pow2(s_carry[k][threadIdx.x], (k & 1) ? 25u : 26u)));
    x.put(lam + 266 + k, v);
  }
}

// The loops below load a gadget's cells five limbs at a time before using them,
// so a warp has tens of loads in flight instead of waiting on each limb's few.
// Constraint values go into an exact 128-bit sum, so their order is free.

// eval_add_gadget (ed25519_field_air.rs:431-486)
__device__ void eval_add(Ctx& x, const EdBlock& g) {
  const uint32_t a = g.p[0], b = g.p[1], c = g.p[2], cr = g.p[4], lam = g.lam;
  range(x, c, g.p[3], lam);
  uint64_t ck[NL];
#pragma unroll
  for (uint32_t k = 0; k < NL; ++k) ck[k] = x.v(cr + k);
#pragma unroll
  for (uint32_t h = 0; h < NL; h += 5) {
    uint64_t av[5], bv[5], cv[5];
#pragma unroll
    for (uint32_t j = 0; j < 5; ++j) av[j] = x.v(a + h + j), bv[j] = x.v(b + h + j), cv[j] = x.v(c + h + j);
#pragma unroll
    for (uint32_t j = 0; j < 5; ++j) {
      const uint32_t k = h + j;
      const uint64_t prev = k == 0 ? mul_small(ck[NL - 1], 19) : ck[k - 1];
      const uint64_t v = gl::sub(gl::add(gl::add(av[j], bv[j]), prev), gl::add(cv[j], gl::mul_pow2(ck[k], (k & 1) ? 25u : 26u)));
      x.put(lam + 266 + k, v);
      x.put(lam + 276 + k, gl::mul(ck[k], gl::sub(1, ck[k])));
    }
  }
}

// eval_sub_gadget (ed25519_field_air.rs:672-730)
__device__ void eval_sub(Ctx& x, const EdBlock& g) {
  const uint32_t a = g.p[0], b = g.p[1], c = g.p[2], pos = g.p[4], neg = g.p[5], lam = g.lam;
  range(x, c, g.p[3], lam);
  uint64_t net[NL];
  {
    uint64_t cp[NL], cn[NL];
#pragma unroll
    for (uint32_t k = 0; k < NL; ++k) cp[k] = x.v(pos + k), cn[k] = x.v(neg + k);
#pragma unroll
    for (uint32_t k = 0; k < NL; ++k) {
      net[k] = gl::sub(cp[k], cn[k]);
      x.put(lam + 276 + k, gl::mul(cp[k], gl::sub(1, cp[k])));
      x.put(lam + 286 + k, gl::mul(cn[k], gl::sub(1, cn[k])));
      x.put(lam + 296 + k, gl::mul(cp[k], cn[k]));
    }
  }
#pragma unroll
  for (uint32_t h = 0; h < NL; h += 5) {
    uint64_t av[5], bv[5], cv[5];
#pragma unroll
    for (uint32_t j = 0; j < 5; ++j) av[j] = x.v(a + h + j), bv[j] = x.v(b + h + j), cv[j] = x.v(c + h + j);
#pragma unroll
    for (uint32_t j = 0; j < 5; ++j) {
      const uint32_t k = h + j;
      const uint64_t prev = k == 0 ? mul_small(net[NL - 1], 19) : net[k - 1];
      const uint64_t v = gl::add(gl::sub(gl::sub(gl::sub(av[j], bv[j]), prev), cv[j]),
                                 gl::mul_pow2(net[k], (k & 1) ? 25u : 26u));
      x.put(lam + 266 + k, v);
    }
  }
}

// eval_select_gadget (ed25519_field_air.rs:1457-1475)
__device__ void eval_sel(Ctx& x, const EdBlock& g) {
  const uint32_t a = g.p[0], b = g.p[1], c = g.p[3], lam = g.lam;
  const uint64_t s = x.v(g.p[2]);
  x.put(lam + 1, gl::mul(s, gl::sub(1, s)));
#pragma unroll
  for (uint32_t h = 0; h < NL; h += 5) {
    uint64_t av[5], bv[5], cv[5];
#pragma unroll
    for (uint32_t j = 0; j < 5; ++j) av[j] = x.v(a + h + j), bv[j] = x.v(b + h + j), cv[j] = x.v(c + h + j);
#pragma unroll
    for (uint32_t j = 0; j < 5; ++j)
      x.put(lam + 2 + h + j, gl::sub(gl::sub(cv[j], av[j]), gl::mul(s, gl::sub(bv[j], av[j]))));
  }
}

__device__ __forceinline__ uint64_t ref(const Ctx& x, uint64_t r) {
  const uint64_t src = r >> 62;
  const uint32_t v = (uint32_t)(r & 0xFFFFFFFFu);
  return src == SRC_CUR ? x.v(v) : src == SRC_NXT ? x.w(v) : (r & ((1ull << 62) - 1));
}

// Pairs go in batches of 8: the batch's 16 references (the same for the whole warp)
// are read first, then its up to 16 cells, then the 8 differences.
__device__ void eval_pairs(Ctx& x, const EdBlock& g, const uint64_t* pairs) {
  constexpr uint32_t kB = 8;
  const uint32_t off = g.p[0], cnt = g.p[1];
  uint32_t i = 0;
  for (; i + kB <= cnt; i += kB) {
    uint64_t r[2 * kB], v[2 * kB];
#pragma unroll
    for (uint32_t j = 0; j < 2 * kB; ++j) r[j] = __ldg(pairs + 2 * (off + i) + j);
#pragma unroll
    for (uint32_t j = 0; j < 2 * kB; ++j) v[j] = ref(x, r[j]);
#pragma unroll
    for (uint32_t j = 0; j < kB; ++j) x.put(g.lam + 1 + i + j, gl::sub(v[2 * j], v[2 * j + 1]));
  }
  for (; i < cnt; ++i) {
    const uint64_t ra = __ldg(pairs + 2 * (off + i)), rb = __ldg(pairs + 2 * (off + i) + 1);
    x.put(g.lam + 1 + i, gl::sub(ref(x, ra), ref(x, rb)));
  }
}

// eval_scalar_reduce_gadget (ed25519_scalar_air.rs:412-583); its 16 r + slack = L - 1
// slots are zero. Single row: plain code.
__device__ void eval_reduce(Ctx& x, const EdBlock& g) {
  const uint32_t in = g.p[0], lam = g.lam;
  const uint32_t limbs[3] = {g.p[1], g.p[3], g.p[5]}, bits[3] = {g.p[2], g.p[4], g.p[6]},
                 cnt[3] = {RED_Q, RED_R, RED_R}, base[3] = {0, 289, 561};
  for (int part = 0; part < 3; ++part)
    for (uint32_t i = 0; i < cnt[part]; ++i) {
      gl::Acc128 a = x.acc;
      const uint64_t s = bits_pack<RED_LB>(x.L, x.n, bits[part] + i * RED_LB, lam + 1 + base[part] + i * RED_LB, &a);
      x.acc = a;
      x.put(lam + 1 + base[part] + cnt[part] * RED_LB + i, gl::sub(x.v(limbs[part] + i), s));
    }
  constexpr uint32_t L16[RED_R] = {0xd3ed, 0x5cf5, 0x631a, 0x5812, 0x9cd6, 0xa2f7, 0xf9de, 0x14de,
                                   0,      0,      0,      0,      0,      0,      0,      0x1000};
  uint64_t prev = 0;
  for (uint32_t k = 0; k < RED_PROD; ++k) {
    gl::Acc128 a = x.acc;
    const uint64_t cy = gl::sub(bits_pack<RED_CB>(x.L, x.n, g.p[7] + k * RED_CB, lam + 1 + 882 + k * RED_CB, &a),
                                kRedBias);
    x.acc = a;
    uint64_t ql = 0;
    for (uint32_t i = 0; i < RED_Q; ++i)
      if (k >= i && k - i < RED_R && L16[k - i]) ql = gl::add(ql, gl::mul(x.v(g.p[1] + i), L16[k - i]));
    const uint64_t in_k = k < RED_IN ? x.v(in + k) : 0, r_k = k < RED_R ? x.v(g.p[3] + k) : 0;
    const uint64_t v = gl::sub(gl::add(gl::sub(gl::sub(in_k, ql), r_k), prev), gl::mul_pow2(cy, RED_LB));
    x.put(lam + 1 + 849 + k, v);
    prev = cy;
  }
}

// the v1 format conversion (ed25519_verify_air.rs:487-538). Single row.
__device__ void eval_format(Ctx& x, const EdBlock& g) {
  const uint32_t db = g.p[0], in = g.p[1], h0 = g.p[2], lam = g.lam;
  for (uint32_t k = 0; k < 8; ++k) {
    gl::Acc128 a = x.acc;
    const uint64_t lo = bits_pack<32>(x.L, x.n, db + 64 * k, lam + 1 + 64 * k, &a);
    const uint64_t hi = bits_pack<32>(x.L, x.n, db + 64 * k + 32, lam + 1 + 64 * k + 32, &a);
    x.acc = a;
    x.put(lam + 1 + 512 + 2 * k, gl::sub(x.v(h0 + 2 * k), lo));
    x.put(lam + 1 + 512 + 2 * k + 1, gl::sub(x.v(h0 + 2 * k + 1), hi));
  }
  for (uint32_t k = 0; k < 8; ++k)
    for (uint32_t m = 0; m < 4; ++m) {
      const uint32_t lb = 56 - 16 * m, hb = lb - 8;
      uint64_t s = 0;
      for (uint32_t j = 0; j < 8; ++j) {
        s = gl::add(s, gl::mul_pow2(x.v(db + 64 * k + lb + j), j));
        s = gl::add(s, gl::mul_pow2(x.v(db + 64 * k + hb + j), 8 + j));
      }
      x.put(lam + 1 + 528 + 4 * k + m, gl::sub(x.w(in + 4 * k + m), s));
    }
}

__global__ void __launch_bounds__(kPhiThreads, 4) ed25519_phi_kernel(EdPhi a, uint64_t* part) {
  const uint64_t i = blockIdx.x * (uint64_t)kPhiThreads + threadIdx.x;
  if (i >= a.n) return;
  uint64_t row, nx;
  if (a.coset_len == 0) {
    row = i / a.blowup;
    nx = (i + a.blowup) % a.n;
  } else {
    const uint64_t c = i / a.coset_len, p = i - c * a.coset_len;
    row = p;
    nx = c * a.coset_len + (p + 1 == a.coset_len ? 0 : p + 1);
  }
  const uint32_t cls = a.row_class[row], c0 = a.cls_chunk[cls], nch = a.cls_chunk[cls + 1] - c0;
  const uint32_t ch = blockIdx.y;
  if (ch >= nch) return;
  Ctx x{a.lde + i, a.lde + nx, a.n, {}};
  const uint32_t b0 = a.chunk_rng[2 * (c0 + ch)], b1 = a.chunk_rng[2 * (c0 + ch) + 1];
  for (uint32_t bi = b0; bi < b1; ++bi) {
    const EdBlock g = a.blocks[a.cls_list[bi]];
    switch (g.kind) {
      case B_MUL: eval_mul(x, g); break;
      case B_ADD: eval_add(x, g); break;
      case B_SUB: eval_sub(x, g); break;
      case B_SEL: eval_sel(x, g); break;
      case B_RANGE: range(x, g.p[0], g.p[1], g.lam); break;
      case B_SIGN: {
        const uint64_t sb = x.v(g.p[0]);
        x.put(g.lam + 1, gl::mul(sb, gl::sub(1, sb)));
        x.put(g.lam + 2, gl::sub(x.v(g.p[1]), sb));
        break;
      }
      case B_PAIRS: eval_pairs(x, g, a.pairs); break;
      case B_REDUCE: eval_reduce(x, g); break;
      case B_FORMAT: eval_format(x, g); break;
      default: break;
    }
  }
  part[(uint64_t)ch * a.n + i] = x.acc.reduce();
}

__global__ void ed25519_phi_sum(EdPhi a, const uint64_t* part, uint64_t* phi) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  uint64_t row, c = 0;
  if (a.coset_len == 0) {
    row = i / a.blowup;
  } else {
    c = i / a.coset_len;
    row = i - c * a.coset_len;
  }
  const uint32_t cls = a.row_class[row], nch = a.cls_chunk[cls + 1] - a.cls_chunk[cls];
  uint64_t s = 0;
  for (uint32_t ch = 0; ch < nch; ++ch) s = gl::add(s, part[(uint64_t)ch * a.n + i]);
  if (a.phi_sha && row < a.sha_rows) s = gl::add(s, a.phi_sha[i]);
  if (a.coset_len == 0)
    phi[i] = s;
  else
    phi[a.out_off + c + a.out_stride * row] = s;
}

// L_r(x) = w_n^r (x^n - 1) / (n (x - w_n^r)) at x = w_N^(a B + j); on the trace
// domain (j = 0) it is 1 when a = r and 0 otherwise.
__global__ void ed25519_lagrange_kernel(const uint32_t* ar, uint32_t n_pairs, uint64_t B, unsigned log_n0,
                                        uint64_t n_trace, uint64_t* lval) {
  const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (t >= (uint64_t)n_pairs * B) return;
  const uint64_t p = t / B, j = t - p * B;
  const uint64_t a = ar[2 * p], r = ar[2 * p + 1];
  if (j == 0) {
    lval[t] = a == r;
    return;
  }
  const uint64_t wN = gl::root_of_unity(log_n0);
  const uint64_t x = gl::pow(wN, a * B + j), wr = gl::pow(wN, r * B);
  const uint64_t num = gl::mul(gl::mul(wr, gl::inv(n_trace % gl::P)), gl::sub(gl::pow(x, n_trace), 1));
  lval[t] = gl::mul(num, gl::inv(gl::sub(x, wr)));
}

// one CTA per task: the B points of read row a of column c
__global__ void ed25519_sparse_fill_kernel(EdLdeFill f, const uint64_t* trace, uint64_t H, uint64_t B,
                                           const uint64_t* lval, uint64_t* lde) {
  const uint32_t* t = f.tasks + 5 * (uint64_t)blockIdx.x;
  const uint64_t c = t[0], a = t[1], lb = t[2], off = t[3], nnz = t[4], n0 = H * B;
  for (uint64_t j = threadIdx.x; j < B; j += blockDim.x) {
    uint64_t v = 0;
    for (uint64_t k = 0; k < nnz; ++k)
      v = gl::add(v, gl::mul(__ldg(trace + c * H + f.nz_rows[off + k]), __ldg(lval + (lb + k) * B + j)));
    lde[c * n0 + a * B + j] = v;
  }
}

__global__ void ed25519_const_fill_kernel(EdLdeFill f, const uint64_t* trace, uint64_t H, uint64_t n0,
                                          uint64_t* lde) {
  const uint64_t total = (uint64_t)f.n_const * n0;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = e / n0, c = f.const_cols[k];
    lde[c * n0 + (e - k * n0)] = __ldg(trace + c * H);
  }
}

}  // namespace

EdPhiPlan ed25519_phi_plan(const Program& prog, uint32_t n_trace, uint32_t chunk_constraints) {
  EdPhiPlan P;
  std::vector<uint32_t> dev_index(prog.blocks.size(), ~0u), count;
  for (size_t b = 0; b < prog.blocks.size(); ++b) {
    const Block& B = prog.blocks[b];
    if (B.kind == B_SHA512) continue;  // evaluated by the SHA-512 kernel
    dev_index[b] = (uint32_t)P.blocks.size();
    EdBlock e{B.kind, B.lam, {0}};
    for (int j = 0; j < 8; ++j) e.p[j] = B.p[j];
    P.blocks.push_back(e);
    count.push_back(B.count);
  }
  std::map<std::vector<uint32_t>, uint32_t> classes;
  P.row_class.assign(n_trace, 0);
  P.cls_chunk.push_back(0);
  for (uint32_t row = 0; row < n_trace; ++row) {
    std::vector<uint32_t> open;
    for (size_t b = 0; b < prog.blocks.size(); ++b)
      if (dev_index[b] != ~0u && gate_open(prog.blocks[b], row)) open.push_back(dev_index[b]);
    auto it = classes.find(open);
    if (it == classes.end()) {
      const uint32_t id = (uint32_t)classes.size();
      require(id < 255, "ed25519: too many row classes");
      it = classes.emplace(open, id).first;
      // the class's blocks grouped by kind (program order within a kind), cut into chunks
      // of about chunk_constraints: most chunks then run one gadget evaluator, so a CTA's
      // instruction footprint is one evaluator's code. Every block carries its own
      // lambda and the sum is exact, so the order changes no value.
      std::vector<uint32_t> order(open);
      std::stable_sort(order.begin(), order.end(),
                       [&](uint32_t x, uint32_t y) { return P.blocks[x].kind < P.blocks[y].kind; });
      const uint32_t start = (uint32_t)P.cls_list.size();
      uint32_t first = start, acc = 0;
      for (uint32_t bi : order) {
        P.cls_list.push_back(bi);
        acc += count[bi];
        if (acc >= chunk_constraints) {
          P.chunk_rng.push_back(first);
          P.chunk_rng.push_back((uint32_t)P.cls_list.size());
          first = (uint32_t)P.cls_list.size();
          acc = 0;
        }
      }
      if (first < P.cls_list.size() || P.cls_list.size() == start) {
        P.chunk_rng.push_back(first);
        P.chunk_rng.push_back((uint32_t)P.cls_list.size());
      }
      P.cls_chunk.push_back((uint32_t)(P.chunk_rng.size() / 2));
      P.max_chunks = std::max(P.max_chunks, P.cls_chunk.back() - P.cls_chunk[P.cls_chunk.size() - 2]);
    }
    P.row_class[row] = (uint8_t)it->second;
  }
  return P;
}

cudaError_t ed25519_lde_fill(const EdLdeFill& f, const uint64_t* d_trace, uint64_t height, uint64_t blowup,
                             uint64_t* d_lval, uint64_t* d_lde, cudaStream_t s) {
  unsigned log_n0 = 0;
  while ((1ull << log_n0) < height * blowup) ++log_n0;
  if ((1ull << log_n0) != height * blowup) return cudaErrorInvalidValue;
  SG_LAUNCH_SCOPE("ed25519_lde_fill", s);
  if (f.n_pairs) {
    const uint64_t t = (uint64_t)f.n_pairs * blowup;
    ed25519_lagrange_kernel<<<(unsigned)((t + 127) / 128), 128, 0, s>>>(f.ar, f.n_pairs, blowup, log_n0, height,
                                                                       d_lval);
  }
  if (f.n_tasks)
    ed25519_sparse_fill_kernel<<<f.n_tasks, (unsigned)std::min<uint64_t>(blowup, 128), 0, s>>>(
        f, d_trace, height, blowup, d_lval, d_lde);
  if (f.n_const) {
    const uint64_t total = (uint64_t)f.n_const * height * blowup;
    ed25519_const_fill_kernel<<<(unsigned)std::min<uint64_t>((total + 255) / 256, 148ull * 32), 256, 0, s>>>(
        f, d_trace, height, height * blowup, d_lde);
  }
  return cudaGetLastError();
}

cudaError_t ed25519_expand(const EdExpand& d, uint64_t* d_trace, cudaStream_t s) {
  const uint64_t total = (uint64_t)d.width * d.height;
  const unsigned blocks = (unsigned)std::min<uint64_t>((total + 255) / 256, 148ull * 32);
  SG_LAUNCH_SCOPE("ed25519_expand", s);
  ed25519_expand_kernel<<<blocks, 256, 0, s>>>(d, d_trace);
  return cudaGetLastError();
}

cudaError_t ed25519_phi_blocks(const EdPhi& a, uint64_t* d_part, cudaStream_t s) {
  if (a.blowup == 0 || a.n % (a.coset_len ? a.coset_len : a.blowup) || a.max_chunks == 0 || a.max_chunks > 65535)
    return cudaErrorInvalidValue;
  SG_LAUNCH_SCOPE("ed25519_phi", s);
  ed25519_phi_kernel<<<dim3((unsigned)((a.n + kPhiThreads - 1) / kPhiThreads), a.max_chunks), kPhiThreads, 0, s>>>(
      a, d_part);
  return cudaGetLastError();
}

cudaError_t ed25519_phi_add(const EdPhi& a, const uint64_t* d_part, uint64_t* d_phi, cudaStream_t s) {
  SG_LAUNCH_SCOPE("ed25519_phi_sum", s);
  ed25519_phi_sum<<<(unsigned)((a.n + 255) / 256), 256, 0, s>>>(a, d_part, d_phi);
  return cudaGetLastError();
}

cudaError_t ed25519_phi(const EdPhi& a, uint64_t* d_part, uint64_t* d_phi, cudaStream_t s) {
  const cudaError_t e = ed25519_phi_blocks(a, d_part, s);
  return e != cudaSuccess ? e : ed25519_phi_add(a, d_part, d_phi, s);
}

}  // namespace sg

// sha256_air.cu — SHA-256 AIR: host trace builder and the device constraint
// evaluation fused with the lambda-combination (deep_ali_merge_sha256,
// deep_ali/src/lib.rs:453-545).
//
// One thread per LDE point i reads row i and row (i + blowup) mod n straight
// from the column-major LDE (consecutive threads -> consecutive addresses in
// every column) and folds the 766 constraint values into Phi(w^i) as it goes;
// no constraint matrix is ever materialised. The emission order below is the
// reference's (sha256_air.rs:956-1294) because lambda_j multiplies the j-th value.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <thread>

#include "counters.hpp"
#include "gl.cuh"
#include "sha256_air.cuh"

namespace sg {
namespace {

static const uint32_t kK_host[64] = {
    0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
    0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
    0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
    0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
    0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
    0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
    0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
    0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};
__constant__ uint32_t kK[64];
static const uint32_t kIV[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                                0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};

// ------------------------------------------------------------------ trace
// Witness generation is split: the host runs the compressions (message schedule
// and the 65 working states of every block, sha::BlockWitness, 2368 bytes a
// block) and the 756 cells of each row are expanded from them by
// sha256_row_cells, the same code on the host (sg_sha256_trace) and on the
// device (sha256_expand_kernel), so a 2^20-row trace crosses PCIe as 19 MB of
// block witnesses instead of 6.3 GB of cells.
__host__ __device__ __forceinline__ uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }
__host__ __device__ __forceinline__ uint32_t Sig0(uint32_t x) { return rotr(x, 2) ^ rotr(x, 13) ^ rotr(x, 22); }
__host__ __device__ __forceinline__ uint32_t Sig1(uint32_t x) { return rotr(x, 6) ^ rotr(x, 11) ^ rotr(x, 25); }
__host__ __device__ __forceinline__ uint32_t sig0(uint32_t x) { return rotr(x, 7) ^ rotr(x, 18) ^ (x >> 3); }
__host__ __device__ __forceinline__ uint32_t sig1(uint32_t x) { return rotr(x, 17) ^ rotr(x, 19) ^ (x >> 10); }
__host__ __device__ __forceinline__ uint32_t chf(uint32_t x, uint32_t y, uint32_t z) { return (x & y) ^ (~x & z); }
__host__ __device__ __forceinline__ uint32_t majf(uint32_t x, uint32_t y, uint32_t z) {
  return (x & y) ^ (x & z) ^ (y & z);
}

void run_block(const uint8_t* blk, const uint32_t iv[8], sha::BlockWitness* b) {
  memcpy(b->iv, iv, 32);
  for (int i = 0; i < 16; ++i)
    b->w[i] = (uint32_t)blk[4 * i] << 24 | (uint32_t)blk[4 * i + 1] << 16 | (uint32_t)blk[4 * i + 2] << 8 |
              blk[4 * i + 3];
  for (int t = 16; t < 64; ++t) b->w[t] = sig1(b->w[t - 2]) + b->w[t - 7] + sig0(b->w[t - 15]) + b->w[t - 16];
  memcpy(b->st[0], iv, 32);
  for (int t = 0; t < 64; ++t) {
    const uint32_t* s = b->st[t];
    uint32_t t1 = s[7] + Sig1(s[4]) + chf(s[4], s[5], s[6]) + kK_host[t] + b->w[t];
    uint32_t t2 = Sig0(s[0]) + majf(s[0], s[1], s[2]);
    uint32_t* o = b->st[t + 1];
    o[0] = t1 + t2; o[1] = s[0]; o[2] = s[1]; o[3] = s[2];
    o[4] = s[3] + t1; o[5] = s[4]; o[6] = s[5]; o[7] = s[6];
  }
}

// fill_block (sha256_air.rs:648-937), one row: block row `br` of the block whose
// witness is B; kt = K[br] for compression rows, 0 otherwise. put(column, value).
template <class Put>
__host__ __device__ __forceinline__ void sha256_row_cells(const sha::BlockWitness& B, uint32_t br, uint32_t kt,
                                                          Put&& put) {
  using namespace sha;
  auto W = [&](int t) -> uint32_t { return (t >= 0 && t < 64) ? B.w[t] : 0u; };
  const uint32_t* s = B.st[br <= 64 ? br : 64];
  const uint32_t a = s[0], b = s[1], c = s[2], d = s[3], e = s[4], f = s[5], g = s[6], hh = s[7];
  for (int k = 0; k < 8; ++k) put(A_a + k, s[k]);
  for (int i = 0; i < 32; ++i) put(BIT_A + i, (a >> i) & 1);
  for (int i = 0; i < 32; ++i) put(BIT_B + i, (b >> i) & 1);
  for (int i = 0; i < 32; ++i) put(BIT_C + i, (c >> i) & 1);
  for (int i = 0; i < 32; ++i) put(BIT_E + i, (e >> i) & 1);
  for (int i = 0; i < 32; ++i) put(BIT_F + i, (f >> i) & 1);
  for (int i = 0; i < 32; ++i) put(BIT_G + i, (g >> i) & 1);
  const uint32_t s0a = rotr(a, 2) ^ rotr(a, 13), s1e = rotr(e, 6) ^ rotr(e, 11);
  for (int i = 0; i < 32; ++i) put(S0_T + i, (s0a >> i) & 1);
  for (int i = 0; i < 32; ++i) put(S0_BIT + i, (Sig0(a) >> i) & 1);
  put(S0_W, Sig0(a));
  for (int i = 0; i < 32; ++i) put(S1_T + i, (s1e >> i) & 1);
  for (int i = 0; i < 32; ++i) put(S1_BIT + i, (Sig1(e) >> i) & 1);
  put(S1_W, Sig1(e));
  const uint32_t chw = chf(e, f, g), mjw = majf(a, b, c), ab = a & b, ac = a & c, bc = b & c;
  for (int i = 0; i < 32; ++i) put(CH_BIT + i, (chw >> i) & 1);
  put(CH_W, chw);
  for (int i = 0; i < 32; ++i) put(MAJ_AB + i, (ab >> i) & 1);
  for (int i = 0; i < 32; ++i) put(MAJ_AC + i, (ac >> i) & 1);
  for (int i = 0; i < 32; ++i) put(MAJ_BC + i, (bc >> i) & 1);
  for (int i = 0; i < 32; ++i) put(MAJ_U + i, ((ab ^ ac) >> i) & 1);
  for (int i = 0; i < 32; ++i) put(MAJ_BIT + i, (mjw >> i) & 1);
  put(MAJ_W, mjw);
  const uint32_t wt = br < 64 ? B.w[br] : 0;
  put(W_, wt);
  const uint64_t t1 = (uint64_t)hh + Sig1(e) + chw + kt + wt, t2 = (uint64_t)Sig0(a) + mjw;
  const uint32_t t1c = (uint32_t)(t1 >> 32), t2c = (uint32_t)(t2 >> 32);
  put(T1_LO, t1 & 0xFFFFFFFFu);
  put(T1_C0, t1c & 1);
  put(T1_C1, (t1c >> 1) & 1);
  put(T1_C2, (t1c >> 2) & 1);
  put(T1_CW, t1c);
  put(T2_LO, t2 & 0xFFFFFFFFu);
  put(T2_C0, t2c & 1);
  put(T2_C1, (t2c >> 1) & 1);
  put(T2_CW, t2c);
  for (int k = 0; k < 8; ++k) put(H0 + k, br <= 64 ? B.iv[k] : B.iv[k] + B.st[64][k]);
  for (int k = 0; k < 15; ++k) put(WW0 + k, W((int)br - 15 + k));
  const uint32_t w14 = W((int)br - 1), w1 = W((int)br - 14);
  for (int i = 0; i < 32; ++i) put(BIT_WW14 + i, (w14 >> i) & 1);
  for (int i = 0; i < 32; ++i) put(BIT_WW1 + i, (w1 >> i) & 1);
  // sigma0 / sigma1: two rotations, then the shift (zero-filled above bit 31 - n)
  const uint32_t ss0t = rotr(w1, 7) ^ rotr(w1, 18), ss1t = rotr(w14, 17) ^ rotr(w14, 19);
  for (int i = 0; i < 32; ++i) put(SS0_T + i, (ss0t >> i) & 1);
  for (int i = 0; i < 32; ++i) put(SS0_BIT + i, (sig0(w1) >> i) & 1);
  put(SS0_W, sig0(w1));
  for (int i = 0; i < 32; ++i) put(SS1_T + i, (ss1t >> i) & 1);
  for (int i = 0; i < 32; ++i) put(SS1_BIT + i, (sig1(w14) >> i) & 1);
  put(SS1_W, sig1(w14));
  const uint64_t sum = (uint64_t)W((int)br - 15) + sig0(w1) + W((int)br - 6) + sig1(w14);
  const uint32_t sc = (uint32_t)(sum >> 32);
  put(WS_C0, sc & 1);
  put(WS_C1, (sc >> 1) & 1);
  put(WS_CW, sc);
  const uint64_t t1lo = t1 & 0xFFFFFFFFu, t2lo = t2 & 0xFFFFFFFFu;
  put(NA_C, br < 64 ? (t1lo + t2lo) >> 32 : 0);
  put(NE_C, br < 64 ? ((uint64_t)d + t1lo) >> 32 : 0);
}

// One thread per trace row; padding rows repeat the last useful row. Consecutive
// threads write consecutive addresses of every column.
__global__ void __launch_bounds__(256) sha256_expand_kernel(const sha::BlockWitness* __restrict__ wit,
                                                            uint64_t useful, uint64_t h, uint64_t* __restrict__ out) {
  const uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (r >= h) return;
  const uint64_t rr = r < useful ? r : useful - 1;
  const uint32_t br = (uint32_t)(rr % sha::ROWS_PER_BLOCK);
  sha256_row_cells(wit[rr / sha::ROWS_PER_BLOCK], br, br < 64 ? kK[br] : 0u,
                   [&](uint32_t c, uint64_t v) { out[(uint64_t)c * h + r] = v; });
}

// ------------------------------------------------------------------ device Phi
struct Acc {
  const uint64_t* lam;
  uint64_t phi;
  uint32_t k;
  __device__ __forceinline__ void push(uint64_t v) {
    phi = gl::add(phi, gl::mul(__ldg(lam + k), v));
    ++k;
  }
  __device__ __forceinline__ void zeros(uint32_t cnt) { k += cnt; }  // disabled slots contribute 0
};

__device__ __forceinline__ uint64_t xor_poly(uint64_t x, uint64_t y) {
  // x + y - 2xy
  return gl::sub(gl::add(x, y), gl::add(gl::mul(x, y), gl::mul(x, y)));
}

// Point i of a column-major evaluation buffer (n points per column): cur = point
// i, nxt = point (i + step) mod n, trace_row = i / row_div. The full LDE uses
// (step, row_div) = (blowup, blowup); one coset of it uses (1, 1).
// The 766 constraints are split into kPhiChunks chunks (grid.y): constraints
// 0-263 (bit booleanity, bit -> word packs), 264-523 (the four Sigma / sigma
// blocks) and 524-765 (Ch, Maj, carries, register shifts, H, W window,
// schedule). Chunk c writes its part of Phi at part[c n + i]; sha256_phi_sum adds
// them. Three shorter threads per point keep more warps in flight than one long
// one: a thread of the unsplit kernel spent most of its time waiting on loads.
constexpr int kPhiChunks = 3;
__global__ void __launch_bounds__(128, 4) sha256_phi_kernel(const uint64_t* __restrict__ lde, uint64_t n, uint64_t step,
                                                         uint64_t row_div, uint64_t n_blocks,
                                                         const uint64_t* __restrict__ lam, uint64_t* __restrict__ part) {
  using namespace sha;
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t chunk = blockIdx.y;
  const uint64_t j = (i + step) & (n - 1);
  auto C = [&](uint32_t col) { return __ldg(lde + (uint64_t)col * n + i); };
  auto X = [&](uint32_t col) { return __ldg(lde + (uint64_t)col * n + j); };
  const uint64_t row = i / row_div, blk = row / ROWS_PER_BLOCK, br = row % ROWS_PER_BLOCK;
  const bool past = blk >= n_blocks;
  const bool comp = !past && br < 64, fin = !past && br == 64, sched = !past && br >= 15 && br <= 62;
  Acc acc{lam, 0, chunk == 0 ? 0u : chunk == 1 ? 264u : 524u};
  // sum_b v_b 2^b over 32 columns: 96-bit terms summed exactly, one reduction
  auto pack = [&](uint32_t off) {
    gl::Acc128 a;
#pragma unroll
    for (int b = 0; b < 32; ++b) a.add_shl(C(off + b), b);
    return a.reduce();
  };
  if (chunk == 0) {
  // bit booleanity: A, B, C, E, F, G, W_win[14], W_win[1]
  const uint32_t bool_offs[8] = {BIT_A, BIT_B, BIT_C, BIT_E, BIT_F, BIT_G, BIT_WW14, BIT_WW1};
#pragma unroll 1
  for (int w = 0; w < 8; ++w)
#pragma unroll 4
    for (int b = 0; b < 32; ++b) {
      uint64_t v = C(bool_offs[w] + b);
      acc.push(gl::mul(v, gl::sub(1, v)));
    }
  // bit -> word decompositions
  acc.push(gl::sub(C(A_a), pack(BIT_A)));
  acc.push(gl::sub(C(A_b), pack(BIT_B)));
  acc.push(gl::sub(C(A_c), pack(BIT_C)));
  acc.push(gl::sub(C(A_e), pack(BIT_E)));
  acc.push(gl::sub(C(A_f), pack(BIT_F)));
  acc.push(gl::sub(C(A_g), pack(BIT_G)));
  acc.push(gl::sub(C(WW0 + 14), pack(BIT_WW14)));
  acc.push(gl::sub(C(WW0 + 1), pack(BIT_WW1)));
  part[i] = acc.phi;
  return;
  }
  if (chunk == 1) {
  // Sigma0(a), Sigma1(e) (rotations), sigma0(W[t-14]), sigma1(W[t-1]) (two rotations + a shift)
  struct Sg {
    uint32_t bits, t, bit, w;
    int r1, r2, r3;
    bool shift;
  };
  const Sg sgs[4] = {{BIT_A, S0_T, S0_BIT, S0_W, 2, 13, 22, false},
                     {BIT_E, S1_T, S1_BIT, S1_W, 6, 11, 25, false},
                     {BIT_WW1, SS0_T, SS0_BIT, SS0_W, 7, 18, 3, true},
                     {BIT_WW14, SS1_T, SS1_BIT, SS1_W, 17, 19, 10, true}};
#pragma unroll 1
  for (int q = 0; q < 4; ++q) {
    const Sg g = sgs[q];
#pragma unroll 4
    for (int b = 0; b < 32; ++b)
      acc.push(gl::sub(C(g.t + b), xor_poly(C(g.bits + ((b + g.r1) & 31)), C(g.bits + ((b + g.r2) & 31)))));
#pragma unroll 4
    for (int b = 0; b < 32; ++b) {
      uint64_t r = g.shift ? (b + g.r3 < 32 ? C(g.bits + b + g.r3) : 0) : C(g.bits + ((b + g.r3) & 31));
      acc.push(gl::sub(C(g.bit + b), xor_poly(C(g.t + b), r)));
    }
    acc.push(gl::sub(C(g.w), pack(g.bit)));
  }
  part[n + i] = acc.phi;
  return;
  }
  // Ch(e, f, g) = e f + g - e g
#pragma unroll 4
  for (int b = 0; b < 32; ++b) {
    uint64_t e = C(BIT_E + b), f = C(BIT_F + b), g = C(BIT_G + b);
    acc.push(gl::sub(C(CH_BIT + b), gl::sub(gl::add(gl::mul(e, f), g), gl::mul(e, g))));
  }
  acc.push(gl::sub(C(CH_W), pack(CH_BIT)));
  // Maj(a, b, c) with auxiliaries ab, ac, bc, u = ab^ac, maj = u^bc
#pragma unroll 4
  for (int b = 0; b < 32; ++b) {
    uint64_t a = C(BIT_A + b), bb = C(BIT_B + b), c = C(BIT_C + b);
    acc.push(gl::sub(C(MAJ_AB + b), gl::mul(a, bb)));
    acc.push(gl::sub(C(MAJ_AC + b), gl::mul(a, c)));
    acc.push(gl::sub(C(MAJ_BC + b), gl::mul(bb, c)));
  }
#pragma unroll 4
  for (int b = 0; b < 32; ++b) acc.push(gl::sub(C(MAJ_U + b), xor_poly(C(MAJ_AB + b), C(MAJ_AC + b))));
#pragma unroll 4
  for (int b = 0; b < 32; ++b) acc.push(gl::sub(C(MAJ_BIT + b), xor_poly(C(MAJ_U + b), C(MAJ_BC + b))));
  acc.push(gl::sub(C(MAJ_W), pack(MAJ_BIT)));
  // T1 = h + Sigma1 + Ch + K[t] + W[t] = T1_lo + 2^32 carry, 3 carry bits
  const uint64_t P32 = 1ull << 32;
  const uint64_t krow = comp ? kK[br] : 0;
  {
    uint64_t sum = gl::add(gl::add(gl::add(gl::add(C(A_h), C(S1_W)), C(CH_W)), krow), C(W_));
    acc.push(gl::sub(gl::add(C(T1_LO), gl::mul(P32, C(T1_CW))), sum));
  }
  {
    uint64_t c0 = C(T1_C0), c1 = C(T1_C1), c2 = C(T1_C2);
    acc.push(gl::mul(c0, gl::sub(1, c0)));
    acc.push(gl::mul(c1, gl::sub(1, c1)));
    acc.push(gl::mul(c2, gl::sub(1, c2)));
    acc.push(gl::sub(gl::sub(gl::sub(C(T1_CW), c0), gl::add(c1, c1)), gl::mul_pow2_lt64(c2, 2)));
  }
  // T2 = Sigma0 + Maj = T2_lo + 2^32 carry
  acc.push(gl::sub(gl::add(C(T2_LO), gl::mul(P32, C(T2_CW))), gl::add(C(S0_W), C(MAJ_W))));
  {
    uint64_t c0 = C(T2_C0), c1 = C(T2_C1);
    acc.push(gl::mul(c0, gl::sub(1, c0)));
    acc.push(gl::mul(c1, gl::sub(1, c1)));
    acc.push(gl::sub(gl::sub(C(T2_CW), c0), gl::add(c1, c1)));
  }
  // working-register shifts and new_a / new_e (compression rows only)
  if (comp) {
    acc.push(gl::sub(X(A_b), C(A_a)));
    acc.push(gl::sub(X(A_c), C(A_b)));
    acc.push(gl::sub(X(A_d), C(A_c)));
    acc.push(gl::sub(X(A_f), C(A_e)));
    acc.push(gl::sub(X(A_g), C(A_f)));
    acc.push(gl::sub(X(A_h), C(A_g)));
    const uint64_t na = C(NA_C), ne = C(NE_C);
    acc.push(gl::sub(gl::sub(gl::add(X(A_a), gl::mul(P32, na)), C(T1_LO)), C(T2_LO)));
    acc.push(gl::mul(na, gl::sub(1, na)));
    acc.push(gl::sub(gl::sub(gl::add(X(A_e), gl::mul(P32, ne)), C(A_d)), C(T1_LO)));
    acc.push(gl::mul(ne, gl::sub(1, ne)));
    acc.zeros(2);
  } else {
    acc.zeros(12);
  }
  // H-state: hold, or (finalisation row) delta (delta - 2^32) with delta = H + A - H'
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    if (fin) {
      uint64_t delta = gl::sub(gl::add(C(H0 + k), C(A_a + k)), X(H0 + k));
      acc.push(gl::mul(delta, gl::sub(delta, P32)));
    } else {
      acc.push(gl::sub(X(H0 + k), C(H0 + k)));
    }
  }
  // W window shifts
#pragma unroll
  for (int k = 0; k < 14; ++k) acc.push(gl::sub(X(WW0 + k), C(WW0 + k + 1)));
  acc.push(gl::sub(X(WW0 + 14), C(W_)));
  // message-schedule recurrence (rows 15..62)
  if (sched) {
    uint64_t sum = gl::add(gl::add(gl::add(C(WW0), C(SS0_W)), C(WW0 + 9)), C(SS1_W));
    acc.push(gl::sub(gl::add(X(W_), gl::mul(P32, C(WS_CW))), sum));
    const uint64_t c0 = C(WS_C0), c1 = C(WS_C1);
    acc.push(gl::mul(c0, gl::sub(1, c0)));
    acc.push(gl::mul(c1, gl::sub(1, c1)));
    acc.push(gl::sub(gl::sub(C(WS_CW), c0), gl::add(c1, c1)));
  } else {
    acc.zeros(4);
  }
  part[2 * n + i] = acc.phi;
}

__global__ void sha256_phi_sum(const uint64_t* __restrict__ part, uint64_t n, uint64_t* __restrict__ phi,
                               uint64_t out_stride, uint64_t out_off) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  phi[out_off + i * out_stride] = gl::add(gl::add(part[i], part[n + i]), part[2 * n + i]);
}

bool g_k_uploaded[64] = {false};
std::mutex g_k_mu;

// K lives in constant memory; it is copied once per device.
cudaError_t upload_k() {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> g(g_k_mu);
  if (!g_k_uploaded[dev]) {
    cudaError_t e = cudaMemcpyToSymbol(kK, kK_host, sizeof kK_host);
    if (e != cudaSuccess) return e;
    g_k_uploaded[dev] = true;
  }
  return cudaSuccess;
}

}  // namespace

uint64_t sha256_witness(const uint8_t* msg, uint64_t len, std::vector<sha::BlockWitness>* wit, uint8_t digest[32]) {
  using namespace sha;
  // FIPS 180-4 §5.1.1 padding
  std::vector<uint8_t> buf(msg, msg + len);
  buf.push_back(0x80);
  while (buf.size() % 64 != 56) buf.push_back(0);
  const uint64_t bits = len * 8;
  for (int i = 7; i >= 0; --i) buf.push_back((uint8_t)(bits >> (8 * i)));
  const uint64_t nb = buf.size() / 64;
  wit->resize(nb);
  uint32_t iv[8];
  memcpy(iv, kIV, sizeof iv);
  for (uint64_t b = 0; b < nb; ++b) {
    run_block(buf.data() + 64 * b, iv, &(*wit)[b]);
    for (int k = 0; k < 8; ++k) iv[k] += (*wit)[b].st[64][k];
  }
  for (int k = 0; k < 8; ++k)
    for (int q = 0; q < 4; ++q) digest[4 * k + q] = (uint8_t)(iv[k] >> (24 - 8 * q));
  return sha256_height(nb);
}

uint64_t sha256_height(uint64_t n_blocks) {
  uint64_t h = sha::ROWS_PER_BLOCK;
  while (h < sha::ROWS_PER_BLOCK * n_blocks) h <<= 1;
  return h;
}

void sha256_fill_host(const sha::BlockWitness* wit, uint64_t n_blocks, uint64_t h, uint64_t* out) {
  const uint64_t useful = sha::ROWS_PER_BLOCK * n_blocks;
  auto rows = [&](uint64_t lo, uint64_t hi) {
    for (uint64_t r = lo; r < hi; ++r) {
      const uint64_t rr = r < useful ? r : useful - 1;  // padding rows repeat the last useful row
      const uint32_t br = (uint32_t)(rr % sha::ROWS_PER_BLOCK);
      uint64_t* col0 = out + r;
      sha256_row_cells(wit[rr / sha::ROWS_PER_BLOCK], br, br < 64 ? kK_host[br] : 0u,
                       [&](uint32_t c, uint64_t v) { col0[(uint64_t)c * h] = v; });
    }
  };
  const uint64_t hw = std::max(1u, std::thread::hardware_concurrency());
  const uint64_t nt = std::min<uint64_t>({hw, 64, h / 1024});
  if (nt <= 1) return rows(0, h);
  std::vector<std::thread> th;
  const uint64_t chunk = (h + nt - 1) / nt;
  for (uint64_t t = 0; t < nt; ++t) th.emplace_back(rows, t * chunk, std::min(h, (t + 1) * chunk));
  for (auto& x : th) x.join();
}

uint64_t sha256_build_trace(const uint8_t* msg, uint64_t len, std::vector<uint64_t>* trace, uint64_t* n_blocks,
                            uint8_t digest[32]) {
  std::vector<sha::BlockWitness> wit;
  const uint64_t h = sha256_witness(msg, len, &wit, digest);
  *n_blocks = wit.size();
  trace->resize((uint64_t)sha::WIDTH * h);
  sha256_fill_host(wit.data(), wit.size(), h, trace->data());
  return h;
}

cudaError_t sha256_expand(const sha::BlockWitness* d_wit, uint64_t n_blocks, uint64_t h, uint64_t* d_trace,
                          cudaStream_t s) {
  cudaError_t e = upload_k();
  if (e != cudaSuccess) return e;
  SG_LAUNCH_SCOPE("sha256_expand", s);
  sha256_expand_kernel<<<(unsigned)((h + 255) / 256), 256, 0, s>>>(d_wit, sha::ROWS_PER_BLOCK * n_blocks, h, d_trace);
  return cudaGetLastError();
}

cudaError_t sha256_phi_points(const uint64_t* evals, uint64_t n, uint64_t step, uint64_t row_div, uint64_t n_blocks,
                              const uint64_t* lambdas, uint64_t* phi, uint64_t out_stride, uint64_t out_off,
                              cudaStream_t s) {
  cudaError_t e = upload_k();
  if (e != cudaSuccess) return e;
  const unsigned T = 128;
  uint64_t* part = nullptr;
  e = cudaMallocAsync((void**)&part, kPhiChunks * n * sizeof(uint64_t), s);
  if (e != cudaSuccess) return e;
  {
    SG_LAUNCH_SCOPE("merge_phi", s);
    sha256_phi_kernel<<<dim3((unsigned)((n + T - 1) / T), kPhiChunks), T, 0, s>>>(evals, n, step, row_div, n_blocks,
                                                                                   lambdas, part);
  }
  {
    SG_LAUNCH_SCOPE("merge_phi_sum", s);
    sha256_phi_sum<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(part, n, phi, out_stride, out_off);
  }
  e = cudaGetLastError();
  cudaFreeAsync(part, s);
  return e;
}

}  // namespace sg

#include "hash_air.hpp"
namespace sg {
namespace {
uint64_t sha256_witness_blob(const uint8_t* msg, uint64_t len, std::vector<uint8_t>* blob, uint64_t* n_blocks,
                             uint8_t* digest) {
  std::vector<sha::BlockWitness> wit;
  const uint64_t h = sha256_witness(msg, len, &wit, digest);
  *n_blocks = wit.size();
  blob->resize(wit.size() * sizeof(sha::BlockWitness));
  memcpy(blob->data(), wit.data(), blob->size());
  return h;
}
cudaError_t sha256_expand_blob(const void* d_wit, uint64_t n_blocks, uint64_t h, uint64_t* d_trace, cudaStream_t s) {
  return sha256_expand((const sha::BlockWitness*)d_wit, n_blocks, h, d_trace, s);
}
}  // namespace
const HashAir& sha256_hash_air() {
  static const HashAir a{"sha256", sha::WIDTH, sha::NUM_CONSTRAINTS, 32, sha256_witness_blob, sha256_expand_blob,
                         sha256_phi_points};
  return a;
}
}  // namespace sg

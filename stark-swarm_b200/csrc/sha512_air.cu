// sha512_air.cu — SHA-512 AIR (deep_ali/src/sha512_air.rs): host compressions,
// trace expansion (host threads or device), and the device constraint
// evaluation fused with the lambda-combination (deep_ali_merge_sha512,
// deep_ali/src/lib.rs:561-641).
//
// Same structure as the SHA-256 AIR. Every 64-bit word is two 32-bit limbs,
// because a u64 does not fit a Goldilocks cell with its integer meaning intact.
// Carries are decomposed per limb, and the H-state finalisation uses
// delta (delta - 2^32) = 0 on each limb, with the lo carry folded into the hi
// limb as delta_lo 2^-32. The emission order below is the reference's
// (sha512_air.rs:909-1270) because lambda_j multiplies the j-th value.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <thread>

#include "counters.hpp"
#include "gl.cuh"
#include "sha512_air.cuh"

namespace sg {
namespace {

// FIPS 180-4 §4.2.3 / §5.3.5: first 64 bits of the fractional parts of the cube
// roots of the first 80 primes, and of the square roots of the first 8.
static const uint64_t kK512_host[80] = {
0x428a2f98d728ae22ull, 0x7137449123ef65cdull, 0xb5c0fbcfec4d3b2full, 0xe9b5dba58189dbbcull,
0x3956c25bf348b538ull, 0x59f111f1b605d019ull, 0x923f82a4af194f9bull, 0xab1c5ed5da6d8118ull,
0xd807aa98a3030242ull, 0x12835b0145706fbeull, 0x243185be4ee4b28cull, 0x550c7dc3d5ffb4e2ull,
0x72be5d74f27b896full, 0x80deb1fe3b1696b1ull, 0x9bdc06a725c71235ull, 0xc19bf174cf692694ull,
0xe49b69c19ef14ad2ull, 0xefbe4786384f25e3ull, 0x0fc19dc68b8cd5b5ull, 0x240ca1cc77ac9c65ull,
0x2de92c6f592b0275ull, 0x4a7484aa6ea6e483ull, 0x5cb0a9dcbd41fbd4ull, 0x76f988da831153b5ull,
0x983e5152ee66dfabull, 0xa831c66d2db43210ull, 0xb00327c898fb213full, 0xbf597fc7beef0ee4ull,
0xc6e00bf33da88fc2ull, 0xd5a79147930aa725ull, 0x06ca6351e003826full, 0x142929670a0e6e70ull,
0x27b70a8546d22ffcull, 0x2e1b21385c26c926ull, 0x4d2c6dfc5ac42aedull, 0x53380d139d95b3dfull,
0x650a73548baf63deull, 0x766a0abb3c77b2a8ull, 0x81c2c92e47edaee6ull, 0x92722c851482353bull,
0xa2bfe8a14cf10364ull, 0xa81a664bbc423001ull, 0xc24b8b70d0f89791ull, 0xc76c51a30654be30ull,
0xd192e819d6ef5218ull, 0xd69906245565a910ull, 0xf40e35855771202aull, 0x106aa07032bbd1b8ull,
0x19a4c116b8d2d0c8ull, 0x1e376c085141ab53ull, 0x2748774cdf8eeb99ull, 0x34b0bcb5e19b48a8ull,
0x391c0cb3c5c95a63ull, 0x4ed8aa4ae3418acbull, 0x5b9cca4f7763e373ull, 0x682e6ff3d6b2b8a3ull,
0x748f82ee5defb2fcull, 0x78a5636f43172f60ull, 0x84c87814a1f0ab72ull, 0x8cc702081a6439ecull,
0x90befffa23631e28ull, 0xa4506cebde82bde9ull, 0xbef9a3f7b2c67915ull, 0xc67178f2e372532bull,
0xca273eceea26619cull, 0xd186b8c721c0c207ull, 0xeada7dd6cde0eb1eull, 0xf57d4f7fee6ed178ull,
0x06f067aa72176fbaull, 0x0a637dc5a2c898a6ull, 0x113f9804bef90daeull, 0x1b710b35131c471bull,
0x28db77f523047d84ull, 0x32caab7b40c72493ull, 0x3c9ebe0a15c9bebcull, 0x431d67c49c100d4cull,
0x4cc5d4becb3e42b6ull, 0x597f299cfc657e2aull, 0x5fcb6fab3ad6faecull, 0x6c44198c4a475817ull};
__constant__ uint64_t kK512[80];
static const uint64_t kIV512[8] = {
0x6a09e667f3bcc908ull, 0xbb67ae8584caa73bull, 0x3c6ef372fe94f82bull, 0xa54ff53a5f1d36f1ull,
0x510e527fade682d1ull, 0x9b05688c2b3e6c1full, 0x1f83d9abfb41bd6bull, 0x5be0cd19137e2179ull};

__host__ __device__ __forceinline__ uint64_t rotr64(uint64_t x, int n) { return (x >> n) | (x << (64 - n)); }
__host__ __device__ __forceinline__ uint64_t Sig0(uint64_t x) { return rotr64(x, 28) ^ rotr64(x, 34) ^ rotr64(x, 39); }
__host__ __device__ __forceinline__ uint64_t Sig1(uint64_t x) { return rotr64(x, 14) ^ rotr64(x, 18) ^ rotr64(x, 41); }
__host__ __device__ __forceinline__ uint64_t sig0(uint64_t x) { return rotr64(x, 1) ^ rotr64(x, 8) ^ (x >> 7); }
__host__ __device__ __forceinline__ uint64_t sig1(uint64_t x) { return rotr64(x, 19) ^ rotr64(x, 61) ^ (x >> 6); }
__host__ __device__ __forceinline__ uint64_t chf(uint64_t x, uint64_t y, uint64_t z) { return (x & y) ^ (~x & z); }
__host__ __device__ __forceinline__ uint64_t majf(uint64_t x, uint64_t y, uint64_t z) {
  return (x & y) ^ (x & z) ^ (y & z);
}
__host__ __device__ __forceinline__ uint64_t lo32(uint64_t x) { return x & 0xFFFFFFFFull; }
__host__ __device__ __forceinline__ uint64_t hi32(uint64_t x) { return x >> 32; }

void run_block(const uint8_t* blk, const uint64_t iv[8], sha512::BlockWitness* b) {
  memcpy(b->iv, iv, 64);
  for (int i = 0; i < 16; ++i) {
    uint64_t v = 0;
    for (int k = 0; k < 8; ++k) v = v << 8 | blk[8 * i + k];
    b->w[i] = v;
  }
  for (int t = 16; t < 80; ++t) b->w[t] = sig1(b->w[t - 2]) + b->w[t - 7] + sig0(b->w[t - 15]) + b->w[t - 16];
  memcpy(b->st[0], iv, 64);
  for (int t = 0; t < 80; ++t) {
    const uint64_t* s = b->st[t];
    const uint64_t t1 = s[7] + Sig1(s[4]) + chf(s[4], s[5], s[6]) + kK512_host[t] + b->w[t];
    const uint64_t t2 = Sig0(s[0]) + majf(s[0], s[1], s[2]);
    uint64_t* o = b->st[t + 1];
    o[0] = t1 + t2; o[1] = s[0]; o[2] = s[1]; o[3] = s[2];
    o[4] = s[3] + t1; o[5] = s[4]; o[6] = s[5]; o[7] = s[6];
  }
}

// fill_block (sha512_air.rs:585-896), one row: block row `br` of the block whose
// witness is B; kt = K[br] on compression rows, 0 otherwise. put(column, value).
template <class Put>
__host__ __device__ __forceinline__ void sha512_row_cells(const sha512::BlockWitness& B, uint32_t br, uint64_t kt,
                                                          Put&& put) {
  using namespace sha512;
  auto W = [&](int t) -> uint64_t { return (t >= 0 && t < 80) ? B.w[t] : 0ull; };
  const uint64_t* s = B.st[br <= 80 ? br : 80];
  const uint64_t a = s[0], b = s[1], c = s[2], d = s[3], e = s[4], f = s[5], g = s[6], h = s[7];
  for (int k = 0; k < 8; ++k) {
    put(A_LO + 2 * k, lo32(s[k]));
    put(A_LO + 2 * k + 1, hi32(s[k]));
  }
  for (int i = 0; i < 64; ++i) put(BIT_A + i, (a >> i) & 1);
  for (int i = 0; i < 64; ++i) put(BIT_B + i, (b >> i) & 1);
  for (int i = 0; i < 64; ++i) put(BIT_C + i, (c >> i) & 1);
  for (int i = 0; i < 64; ++i) put(BIT_E + i, (e >> i) & 1);
  for (int i = 0; i < 64; ++i) put(BIT_F + i, (f >> i) & 1);
  for (int i = 0; i < 64; ++i) put(BIT_G + i, (g >> i) & 1);
  const uint64_t s0 = Sig0(a), s1 = Sig1(e), s0t = rotr64(a, 28) ^ rotr64(a, 34), s1t = rotr64(e, 14) ^ rotr64(e, 18);
  for (int i = 0; i < 64; ++i) put(S0_T + i, (s0t >> i) & 1);
  for (int i = 0; i < 64; ++i) put(S0_BIT + i, (s0 >> i) & 1);
  put(S0_LO, lo32(s0));
  put(S0_HI, hi32(s0));
  for (int i = 0; i < 64; ++i) put(S1_T + i, (s1t >> i) & 1);
  for (int i = 0; i < 64; ++i) put(S1_BIT + i, (s1 >> i) & 1);
  put(S1_LO, lo32(s1));
  put(S1_HI, hi32(s1));
  const uint64_t chw = chf(e, f, g), mjw = majf(a, b, c), ab = a & b, ac = a & c, bc = b & c;
  for (int i = 0; i < 64; ++i) put(CH_BIT + i, (chw >> i) & 1);
  put(CH_LO, lo32(chw));
  put(CH_HI, hi32(chw));
  for (int i = 0; i < 64; ++i) put(MAJ_AB + i, (ab >> i) & 1);
  for (int i = 0; i < 64; ++i) put(MAJ_AC + i, (ac >> i) & 1);
  for (int i = 0; i < 64; ++i) put(MAJ_BC + i, (bc >> i) & 1);
  for (int i = 0; i < 64; ++i) put(MAJ_U + i, ((ab ^ ac) >> i) & 1);
  for (int i = 0; i < 64; ++i) put(MAJ_BIT + i, (mjw >> i) & 1);
  put(MAJ_LO, lo32(mjw));
  put(MAJ_HI, hi32(mjw));
  const uint64_t wt = br < 80 ? B.w[br] : 0;
  put(W_LO, lo32(wt));
  put(W_HI, hi32(wt));
  const uint64_t t1l = lo32(h) + lo32(s1) + lo32(chw) + lo32(kt) + lo32(wt), t1lc = t1l >> 32;
  const uint64_t t1h = hi32(h) + hi32(s1) + hi32(chw) + hi32(kt) + hi32(wt) + t1lc, t1hc = t1h >> 32;
  put(T1_LO_LO, lo32(t1l));
  put(T1_LO_C0, t1lc & 1);
  put(T1_LO_C1, (t1lc >> 1) & 1);
  put(T1_LO_C2, (t1lc >> 2) & 1);
  put(T1_LO_CW, t1lc);
  put(T1_HI_LO, lo32(t1h));
  put(T1_HI_C0, t1hc & 1);
  put(T1_HI_C1, (t1hc >> 1) & 1);
  put(T1_HI_C2, (t1hc >> 2) & 1);
  put(T1_HI_CW, t1hc);
  const uint64_t t2l = lo32(s0) + lo32(mjw), t2lc = t2l >> 32;
  const uint64_t t2h = hi32(s0) + hi32(mjw) + t2lc, t2hc = t2h >> 32;
  put(T2_LO_LO, lo32(t2l));
  put(T2_LO_C0, t2lc & 1);
  put(T2_LO_CW, t2lc);
  put(T2_HI_LO, lo32(t2h));
  put(T2_HI_C0, t2hc & 1);
  put(T2_HI_CW, t2hc);
  for (int k = 0; k < 8; ++k) {
    const uint64_t hv = br <= 80 ? B.iv[k] : B.iv[k] + B.st[80][k];
    put(H0_LO + 2 * k, lo32(hv));
    put(H0_LO + 2 * k + 1, hi32(hv));
  }
  for (int k = 0; k < 15; ++k) {
    const uint64_t v = W((int)br - 15 + k);
    put(WW0_LO + 2 * k, lo32(v));
    put(WW0_LO + 2 * k + 1, hi32(v));
  }
  const uint64_t w14 = W((int)br - 1), w1 = W((int)br - 14);
  for (int i = 0; i < 64; ++i) put(BIT_WW14 + i, (w14 >> i) & 1);
  for (int i = 0; i < 64; ++i) put(BIT_WW1 + i, (w1 >> i) & 1);
  // sigma0 / sigma1: two rotations, then the shift (zero-filled at the top)
  const uint64_t ss0 = sig0(w1), ss1 = sig1(w14), ss0t = rotr64(w1, 1) ^ rotr64(w1, 8),
                 ss1t = rotr64(w14, 19) ^ rotr64(w14, 61);
  for (int i = 0; i < 64; ++i) put(SS0_T + i, (ss0t >> i) & 1);
  for (int i = 0; i < 64; ++i) put(SS0_BIT + i, (ss0 >> i) & 1);
  put(SS0_LO, lo32(ss0));
  put(SS0_HI, hi32(ss0));
  for (int i = 0; i < 64; ++i) put(SS1_T + i, (ss1t >> i) & 1);
  for (int i = 0; i < 64; ++i) put(SS1_BIT + i, (ss1 >> i) & 1);
  put(SS1_LO, lo32(ss1));
  put(SS1_HI, hi32(ss1));
  const uint64_t w0 = W((int)br - 15), w9 = W((int)br - 6);
  const uint64_t wsl = lo32(w0) + lo32(ss0) + lo32(w9) + lo32(ss1), wslc = wsl >> 32;
  const uint64_t wsh = hi32(w0) + hi32(ss0) + hi32(w9) + hi32(ss1) + wslc, wshc = wsh >> 32;
  put(WS_LO_C0, wslc & 1);
  put(WS_LO_C1, (wslc >> 1) & 1);
  put(WS_LO_CW, wslc);
  put(WS_HI_C0, wshc & 1);
  put(WS_HI_C1, (wshc >> 1) & 1);
  put(WS_HI_CW, wshc);
  const bool comp = br < 80;
  const uint64_t nal = lo32(t1l) + lo32(t2l), nalc = nal >> 32;
  const uint64_t nel = lo32(d) + lo32(t1l), nelc = nel >> 32;
  put(NA_LO_C, comp ? nalc : 0);
  put(NA_HI_C, comp ? (lo32(t1h) + lo32(t2h) + nalc) >> 32 : 0);
  put(NE_LO_C, comp ? nelc : 0);
  put(NE_HI_C, comp ? (hi32(d) + lo32(t1h) + nelc) >> 32 : 0);
}

__global__ void __launch_bounds__(256) sha512_expand_kernel(const sha512::BlockWitness* __restrict__ wit,
                                                            uint64_t useful, uint64_t h, uint64_t stride,
                                                            uint64_t* __restrict__ out) {
  const uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (r >= h) return;
  const uint64_t rr = r < useful ? r : useful - 1;
  const uint32_t br = (uint32_t)(rr % sha512::ROWS_PER_BLOCK);
  sha512_row_cells(wit[rr / sha512::ROWS_PER_BLOCK], br, br < 80 ? kK512[br] : 0ull,
                   [&](uint32_t c, uint64_t v) { out[(uint64_t)c * stride + r] = v; });
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
  const uint64_t m = gl::mul(x, y);
  return gl::sub(gl::add(x, y), gl::add(m, m));
}

// The 1526 constraints in kPhiChunks chunks (grid.y), as in the SHA-256 kernel:
// 0-527 (bit booleanity, limb packs), 528-1047 (the four Sigma / sigma blocks),
// 1048-1525 (the rest); chunk c writes its part of Phi at part[c n + i].
constexpr int kPhiChunks = 3;
// Work item i < count. Without cosets (coset_len = 0) it is point i of n (a power of
// two), cell col at lde[col * stride + i], its next row at point (i + step) mod n,
// trace row i / row_div. With cosets it is row a = i mod rows_pc of coset c = i / rows_pc:
// point c coset_len + a, next row c coset_len + (a + 1) mod coset_len. Chunk ch writes
// part[ch * count + i].
__global__ void __launch_bounds__(128, 4) sha512_phi_kernel(const uint64_t* __restrict__ lde, uint64_t n,
                                                            uint64_t stride, uint64_t count, uint64_t step,
                                                            uint64_t row_div, uint64_t n_blocks,
                                                            const uint64_t* __restrict__ lam,
                                                            uint64_t* __restrict__ part, uint64_t coset_len,
                                                            uint64_t rows_pc) {
  using namespace sha512;
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= count) return;
  const uint32_t chunk = blockIdx.y;
  uint64_t pt, j, row;
  if (coset_len == 0) {
    pt = i;
    j = (i + step) & (n - 1);
    row = i / row_div;
  } else {
    const uint64_t c = i / rows_pc;
    row = i - c * rows_pc;
    pt = c * coset_len + row;
    j = c * coset_len + (row + 1 == coset_len ? 0 : row + 1);
  }
  auto C = [&](uint32_t col) { return __ldg(lde + (uint64_t)col * stride + pt); };
  auto X = [&](uint32_t col) { return __ldg(lde + (uint64_t)col * stride + j); };
  const uint64_t blk = row / ROWS_PER_BLOCK, br = row % ROWS_PER_BLOCK;
  const bool past = blk >= n_blocks;
  const bool comp = !past && br < ROUNDS, fin = !past && br == ROUNDS, sched = !past && br >= 15 && br <= 78;
  Acc acc{lam, 0, chunk == 0 ? 0u : chunk == 1 ? 528u : 1048u};
  // sum_{b<32} v_b 2^b over 32 columns: 96-bit terms summed exactly, one reduction
  auto pack = [&](uint32_t off) {
    gl::Acc128 a;
#pragma unroll
    for (int b = 0; b < 32; ++b) a.add_shl(C(off + b), b);
    return a.reduce();
  };
  const uint64_t P32 = 1ull << 32;
  if (chunk == 0) {
  // bit booleanity: A, B, C, E, F, G, W_win[14], W_win[1]
  const uint32_t bool_offs[8] = {BIT_A, BIT_B, BIT_C, BIT_E, BIT_F, BIT_G, BIT_WW14, BIT_WW1};
#pragma unroll 1
  for (int w = 0; w < 8; ++w)
#pragma unroll 4
    for (int b = 0; b < 64; ++b) {
      const uint64_t v = C(bool_offs[w] + b);
      acc.push(gl::mul(v, gl::sub(1, v)));
    }
  // bit -> limb decompositions: a, b, c, e, f, g, then W_win[14], W_win[1]
  const uint32_t limb_words[8][2] = {{A_LO + 0, BIT_A}, {A_LO + 2, BIT_B}, {A_LO + 4, BIT_C}, {A_LO + 8, BIT_E},
                                     {A_LO + 10, BIT_F}, {A_LO + 12, BIT_G}, {WW0_LO + 28, BIT_WW14},
                                     {WW0_LO + 2, BIT_WW1}};
#pragma unroll 1
  for (int q = 0; q < 8; ++q) {
    acc.push(gl::sub(C(limb_words[q][0]), pack(limb_words[q][1])));
    acc.push(gl::sub(C(limb_words[q][0] + 1), pack(limb_words[q][1] + 32)));
  }
  part[i] = acc.phi;
  return;
  }
  if (chunk == 1) {
  // Sigma0(a), Sigma1(e) (rotations), sigma0(W_win[1]), sigma1(W_win[14]) (two rotations + a shift)
  struct Sg {
    uint32_t bits, t, bit, lo;
    int r1, r2, r3;
    bool shift;
  };
  const Sg sgs[4] = {{BIT_A, S0_T, S0_BIT, S0_LO, 28, 34, 39, false},
                     {BIT_E, S1_T, S1_BIT, S1_LO, 14, 18, 41, false},
                     {BIT_WW1, SS0_T, SS0_BIT, SS0_LO, 1, 8, 7, true},
                     {BIT_WW14, SS1_T, SS1_BIT, SS1_LO, 19, 61, 6, true}};
#pragma unroll 1
  for (int q = 0; q < 4; ++q) {
    const Sg g = sgs[q];
#pragma unroll 4
    for (int b = 0; b < 64; ++b)
      acc.push(gl::sub(C(g.t + b), xor_poly(C(g.bits + ((b + g.r1) & 63)), C(g.bits + ((b + g.r2) & 63)))));
#pragma unroll 4
    for (int b = 0; b < 64; ++b) {
      const uint64_t r = g.shift ? (b + g.r3 < 64 ? C(g.bits + b + g.r3) : 0) : C(g.bits + ((b + g.r3) & 63));
      acc.push(gl::sub(C(g.bit + b), xor_poly(C(g.t + b), r)));
    }
    acc.push(gl::sub(C(g.lo), pack(g.bit)));
    acc.push(gl::sub(C(g.lo + 1), pack(g.bit + 32)));
  }
  part[count + i] = acc.phi;
  return;
  }
  // Ch(e, f, g) = e f + g - e g
#pragma unroll 4
  for (int b = 0; b < 64; ++b) {
    const uint64_t e = C(BIT_E + b), f = C(BIT_F + b), g = C(BIT_G + b);
    acc.push(gl::sub(C(CH_BIT + b), gl::sub(gl::add(gl::mul(e, f), g), gl::mul(e, g))));
  }
  acc.push(gl::sub(C(CH_LO), pack(CH_BIT)));
  acc.push(gl::sub(C(CH_HI), pack(CH_BIT + 32)));
  // Maj(a, b, c) with auxiliaries ab, ac, bc, u = ab^ac, maj = u^bc
#pragma unroll 4
  for (int b = 0; b < 64; ++b) {
    const uint64_t a = C(BIT_A + b), bb = C(BIT_B + b), c = C(BIT_C + b);
    acc.push(gl::sub(C(MAJ_AB + b), gl::mul(a, bb)));
    acc.push(gl::sub(C(MAJ_AC + b), gl::mul(a, c)));
    acc.push(gl::sub(C(MAJ_BC + b), gl::mul(bb, c)));
  }
#pragma unroll 4
  for (int b = 0; b < 64; ++b) acc.push(gl::sub(C(MAJ_U + b), xor_poly(C(MAJ_AB + b), C(MAJ_AC + b))));
#pragma unroll 4
  for (int b = 0; b < 64; ++b) acc.push(gl::sub(C(MAJ_BIT + b), xor_poly(C(MAJ_U + b), C(MAJ_BC + b))));
  acc.push(gl::sub(C(MAJ_LO), pack(MAJ_BIT)));
  acc.push(gl::sub(C(MAJ_HI), pack(MAJ_BIT + 32)));
  // T1 / T2 per-limb carry decompositions
  const uint64_t kt = comp ? kK512[br] : 0;
  {
    const uint64_t sum = gl::add(gl::add(gl::add(gl::add(C(A_LO + 14), C(S1_LO)), C(CH_LO)), lo32(kt)), C(W_LO));
    acc.push(gl::sub(gl::add(C(T1_LO_LO), gl::mul(P32, C(T1_LO_CW))), sum));
    const uint64_t c0 = C(T1_LO_C0), c1 = C(T1_LO_C1), c2 = C(T1_LO_C2);
    acc.push(gl::mul(c0, gl::sub(1, c0)));
    acc.push(gl::mul(c1, gl::sub(1, c1)));
    acc.push(gl::mul(c2, gl::sub(1, c2)));
    acc.push(gl::sub(gl::sub(gl::sub(C(T1_LO_CW), c0), gl::add(c1, c1)), gl::mul_pow2_lt64(c2, 2)));
  }
  {
    const uint64_t sum = gl::add(gl::add(gl::add(gl::add(gl::add(C(A_LO + 15), C(S1_HI)), C(CH_HI)), hi32(kt)),
                                         C(W_HI)),
                                 C(T1_LO_CW));
    acc.push(gl::sub(gl::add(C(T1_HI_LO), gl::mul(P32, C(T1_HI_CW))), sum));
    const uint64_t c0 = C(T1_HI_C0), c1 = C(T1_HI_C1), c2 = C(T1_HI_C2);
    acc.push(gl::mul(c0, gl::sub(1, c0)));
    acc.push(gl::mul(c1, gl::sub(1, c1)));
    acc.push(gl::mul(c2, gl::sub(1, c2)));
    acc.push(gl::sub(gl::sub(gl::sub(C(T1_HI_CW), c0), gl::add(c1, c1)), gl::mul_pow2_lt64(c2, 2)));
  }
  {
    acc.push(gl::sub(gl::add(C(T2_LO_LO), gl::mul(P32, C(T2_LO_CW))), gl::add(C(S0_LO), C(MAJ_LO))));
    const uint64_t c0 = C(T2_LO_C0);
    acc.push(gl::mul(c0, gl::sub(1, c0)));
    acc.push(gl::sub(C(T2_LO_CW), c0));
    acc.push(gl::sub(gl::add(C(T2_HI_LO), gl::mul(P32, C(T2_HI_CW))),
                     gl::add(gl::add(C(S0_HI), C(MAJ_HI)), C(T2_LO_CW))));
    const uint64_t c1 = C(T2_HI_C0);
    acc.push(gl::mul(c1, gl::sub(1, c1)));
    acc.push(gl::sub(C(T2_HI_CW), c1));
  }
  // working-register shifts b<-a, c<-b, d<-c, f<-e, g<-f, h<-g (lo, hi), then new_a / new_e
  if (comp) {
    const uint32_t sh[6][2] = {{2, 0}, {4, 2}, {6, 4}, {10, 8}, {12, 10}, {14, 12}};
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      acc.push(gl::sub(X(A_LO + sh[q][0]), C(A_LO + sh[q][1])));
      acc.push(gl::sub(X(A_LO + sh[q][0] + 1), C(A_LO + sh[q][1] + 1)));
    }
    const uint64_t nal = C(NA_LO_C), nah = C(NA_HI_C), nel = C(NE_LO_C), neh = C(NE_HI_C);
    acc.push(gl::sub(gl::sub(gl::add(X(A_LO), gl::mul(P32, nal)), C(T1_LO_LO)), C(T2_LO_LO)));
    acc.push(gl::mul(nal, gl::sub(1, nal)));
    acc.push(gl::sub(gl::sub(gl::sub(gl::add(X(A_LO + 1), gl::mul(P32, nah)), C(T1_HI_LO)), C(T2_HI_LO)), nal));
    acc.push(gl::mul(nah, gl::sub(1, nah)));
    acc.push(gl::sub(gl::sub(gl::add(X(A_LO + 8), gl::mul(P32, nel)), C(A_LO + 6)), C(T1_LO_LO)));
    acc.push(gl::mul(nel, gl::sub(1, nel)));
    acc.push(gl::sub(gl::sub(gl::sub(gl::add(X(A_LO + 9), gl::mul(P32, neh)), C(A_LO + 7)), C(T1_HI_LO)), nel));
    acc.push(gl::mul(neh, gl::sub(1, neh)));
  } else {
    acc.zeros(20);
  }
  // H-state: hold, or (finalisation row) delta (delta - 2^32) per limb with the lo
  // carry delta_lo 2^-32 folded into the hi limb (2^-32 = p + 1 - 2^32)
  const uint64_t INV32 = 0xFFFFFFFE00000002ull;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t hl = H0_LO + 2 * k, al = A_LO + 2 * k;
    if (fin) {
      const uint64_t dlo = gl::sub(gl::add(C(hl), C(al)), X(hl));
      const uint64_t dhi = gl::sub(gl::add(gl::add(C(hl + 1), C(al + 1)), gl::mul(dlo, INV32)), X(hl + 1));
      acc.push(gl::mul(dlo, gl::sub(dlo, P32)));
      acc.push(gl::mul(dhi, gl::sub(dhi, P32)));
    } else {
      acc.push(gl::sub(X(hl), C(hl)));
      acc.push(gl::sub(X(hl + 1), C(hl + 1)));
    }
  }
  // W window shifts
#pragma unroll
  for (int k = 0; k < 14; ++k) {
    acc.push(gl::sub(X(WW0_LO + 2 * k), C(WW0_LO + 2 * k + 2)));
    acc.push(gl::sub(X(WW0_LO + 2 * k + 1), C(WW0_LO + 2 * k + 3)));
  }
  acc.push(gl::sub(X(WW0_LO + 28), C(W_LO)));
  acc.push(gl::sub(X(WW0_LO + 29), C(W_HI)));
  // message-schedule recurrence (rows 15..78), lo then hi with the carry in
  if (sched) {
    const uint64_t sl = gl::add(gl::add(gl::add(C(WW0_LO), C(SS0_LO)), C(WW0_LO + 18)), C(SS1_LO));
    acc.push(gl::sub(gl::add(X(W_LO), gl::mul(P32, C(WS_LO_CW))), sl));
    const uint64_t c0 = C(WS_LO_C0), c1 = C(WS_LO_C1);
    acc.push(gl::mul(c0, gl::sub(1, c0)));
    acc.push(gl::mul(c1, gl::sub(1, c1)));
    acc.push(gl::sub(gl::sub(C(WS_LO_CW), c0), gl::add(c1, c1)));
    const uint64_t sh =
        gl::add(gl::add(gl::add(gl::add(C(WW0_LO + 1), C(SS0_HI)), C(WW0_LO + 19)), C(SS1_HI)), C(WS_LO_CW));
    acc.push(gl::sub(gl::add(X(W_HI), gl::mul(P32, C(WS_HI_CW))), sh));
    const uint64_t d0 = C(WS_HI_C0), d1 = C(WS_HI_C1);
    acc.push(gl::mul(d0, gl::sub(1, d0)));
    acc.push(gl::mul(d1, gl::sub(1, d1)));
    acc.push(gl::sub(gl::sub(C(WS_HI_CW), d0), gl::add(d1, d1)));
  } else {
    acc.zeros(8);
  }
  part[2 * count + i] = acc.phi;
}

__global__ void sha512_phi_sum(const uint64_t* __restrict__ part, uint64_t n, uint64_t* __restrict__ phi,
                               uint64_t out_stride, uint64_t out_off, uint64_t coset_len, uint64_t rows_pc) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t o = coset_len ? (i / rows_pc) * coset_len + i % rows_pc : out_off + i * out_stride;
  phi[o] = gl::add(gl::add(part[i], part[n + i]), part[2 * n + i]);
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
    cudaError_t e = cudaMemcpyToSymbol(kK512, kK512_host, sizeof kK512_host);
    if (e != cudaSuccess) return e;
    g_k_uploaded[dev] = true;
  }
  return cudaSuccess;
}

}  // namespace

uint64_t sha512_witness(const uint8_t* msg, uint64_t len, std::vector<sha512::BlockWitness>* wit,
                        uint8_t digest[64]) {
  // FIPS 180-4 §5.1.2 padding: 0x80, zeros to 112 mod 128, 128-bit big-endian length
  std::vector<uint8_t> buf(msg, msg + len);
  buf.push_back(0x80);
  while (buf.size() % 128 != 112) buf.push_back(0);
  for (int i = 0; i < 8; ++i) buf.push_back(0);
  const uint64_t bits = len * 8;
  for (int i = 7; i >= 0; --i) buf.push_back((uint8_t)(bits >> (8 * i)));
  const uint64_t nb = buf.size() / 128;
  wit->resize(nb);
  uint64_t iv[8];
  memcpy(iv, kIV512, sizeof iv);
  for (uint64_t b = 0; b < nb; ++b) {
    run_block(buf.data() + 128 * b, iv, &(*wit)[b]);
    for (int k = 0; k < 8; ++k) iv[k] += (*wit)[b].st[80][k];
  }
  for (int k = 0; k < 8; ++k)
    for (int q = 0; q < 8; ++q) digest[8 * k + q] = (uint8_t)(iv[k] >> (56 - 8 * q));
  uint64_t h = sha512::ROWS_PER_BLOCK;
  while (h < sha512::ROWS_PER_BLOCK * nb) h <<= 1;
  return h;
}

void sha512_fill_host(const sha512::BlockWitness* wit, uint64_t n_blocks, uint64_t h, uint64_t* out) {
  const uint64_t useful = sha512::ROWS_PER_BLOCK * n_blocks;
  auto rows = [&](uint64_t lo, uint64_t hi) {
    for (uint64_t r = lo; r < hi; ++r) {
      const uint64_t rr = r < useful ? r : useful - 1;  // padding rows repeat the last useful row
      const uint32_t br = (uint32_t)(rr % sha512::ROWS_PER_BLOCK);
      uint64_t* col0 = out + r;
      sha512_row_cells(wit[rr / sha512::ROWS_PER_BLOCK], br, br < 80 ? kK512_host[br] : 0ull,
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

cudaError_t sha512_expand(const sha512::BlockWitness* d_wit, uint64_t n_blocks, uint64_t h, uint64_t* d_trace,
                          cudaStream_t s) {
  return sha512_expand_strided(d_wit, n_blocks, h, h, d_trace, s);
}

cudaError_t sha512_expand_strided(const sha512::BlockWitness* d_wit, uint64_t n_blocks, uint64_t h, uint64_t stride,
                                  uint64_t* d_trace, cudaStream_t s) {
  if (stride < h) return cudaErrorInvalidValue;
  cudaError_t e = upload_k();
  if (e != cudaSuccess) return e;
  SG_LAUNCH_SCOPE("sha512_expand", s);
  sha512_expand_kernel<<<(unsigned)((h + 255) / 256), 256, 0, s>>>(d_wit, sha512::ROWS_PER_BLOCK * n_blocks, h,
                                                                     stride, d_trace);
  return cudaGetLastError();
}

cudaError_t sha512_phi_points(const uint64_t* evals, uint64_t n, uint64_t step, uint64_t row_div, uint64_t n_blocks,
                              const uint64_t* lambdas, uint64_t* phi, uint64_t out_stride, uint64_t out_off,
                              cudaStream_t s) {
  return sha512_phi_points_ex(evals, n, n, n, step, row_div, n_blocks, lambdas, phi, out_stride, out_off, s);
}

cudaError_t sha512_phi_points_ex(const uint64_t* evals, uint64_t n, uint64_t stride, uint64_t count, uint64_t step,
                                 uint64_t row_div, uint64_t n_blocks, const uint64_t* lambdas, uint64_t* phi,
                                 uint64_t out_stride, uint64_t out_off, cudaStream_t s) {
  if (count == 0) return cudaSuccess;
  if (count > n || stride < count || (n & (n - 1))) return cudaErrorInvalidValue;
  cudaError_t e = upload_k();
  if (e != cudaSuccess) return e;
  const unsigned T = 128;
  uint64_t* part = nullptr;
  e = cudaMallocAsync((void**)&part, kPhiChunks * count * sizeof(uint64_t), s);
  if (e != cudaSuccess) return e;
  {
    SG_LAUNCH_SCOPE("merge_phi", s);
    sha512_phi_kernel<<<dim3((unsigned)((count + T - 1) / T), kPhiChunks), T, 0, s>>>(
        evals, n, stride, count, step, row_div, n_blocks, lambdas, part, 0, 0);
  }
  {
    SG_LAUNCH_SCOPE("merge_phi_sum", s);
    sha512_phi_sum<<<(unsigned)((count + 255) / 256), 256, 0, s>>>(part, count, phi, out_stride, out_off, 0, 0);
  }
  e = cudaGetLastError();
  cudaFreeAsync(part, s);
  return e;
}

cudaError_t sha512_phi_cosets(const uint64_t* evals, uint64_t n_cosets, uint64_t coset_len, uint64_t rows,
                              uint64_t n_blocks, const uint64_t* lambdas, uint64_t* phi, cudaStream_t s) {
  const uint64_t count = n_cosets * rows;
  if (count == 0) return cudaSuccess;
  if (rows > coset_len) return cudaErrorInvalidValue;
  cudaError_t e = upload_k();
  if (e != cudaSuccess) return e;
  const unsigned T = 128;
  uint64_t* part = nullptr;
  e = cudaMallocAsync((void**)&part, kPhiChunks * count * sizeof(uint64_t), s);
  if (e != cudaSuccess) return e;
  {
    SG_LAUNCH_SCOPE("merge_phi", s);
    sha512_phi_kernel<<<dim3((unsigned)((count + T - 1) / T), kPhiChunks), T, 0, s>>>(
        evals, coset_len, n_cosets * coset_len, count, 1, 1, n_blocks, lambdas, part, coset_len, rows);
  }
  {
    SG_LAUNCH_SCOPE("merge_phi_sum", s);
    sha512_phi_sum<<<(unsigned)((count + 255) / 256), 256, 0, s>>>(part, count, phi, 0, 0, coset_len, rows);
  }
  e = cudaGetLastError();
  cudaFreeAsync(part, s);
  return e;
}

}  // namespace sg

#include "hash_air.hpp"
namespace sg {
namespace {
uint64_t sha512_witness_blob(const uint8_t* msg, uint64_t len, std::vector<uint8_t>* blob, uint64_t* n_blocks,
                             uint8_t* digest) {
  std::vector<sha512::BlockWitness> wit;
  const uint64_t h = sha512_witness(msg, len, &wit, digest);
  *n_blocks = wit.size();
  blob->resize(wit.size() * sizeof(sha512::BlockWitness));
  memcpy(blob->data(), wit.data(), blob->size());
  return h;
}
cudaError_t sha512_expand_blob(const void* d_wit, uint64_t n_blocks, uint64_t h, uint64_t* d_trace, cudaStream_t s) {
  return sha512_expand((const sha512::BlockWitness*)d_wit, n_blocks, h, d_trace, s);
}
}  // namespace
const HashAir& sha512_hash_air() {
  static const HashAir a{"sha512", sha512::WIDTH, sha512::NUM_CONSTRAINTS, 64, sha512_witness_blob,
                         sha512_expand_blob, sha512_phi_points};
  return a;
}
}  // namespace sg

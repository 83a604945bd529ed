// dft.cuh — in-register small DFTs over Goldilocks with shift-only twiddles.
//
// For ark-poly's root chain the small roots are powers of two:
// w_2 = 2^96, w_4 = 2^48, w_8 = 2^120, w_16 = 2^156 (and w_16^-1 = 2^36),
// because 2 has order 192 in this field. A radix-R DFT (R <= 16) therefore
// needs no multiplications, only shifts and 128-bit reductions.
#pragma once
#include "gl.cuh"

namespace sg {

__host__ __device__ constexpr unsigned exp16(bool inv) { return inv ? 36u : 156u; }  // w_16^{+-1} = 2^e

template <int R>
struct BitRev {
  static constexpr int v(int i) {
    int r = 0;
    for (int b = 1, c = R >> 1; b < R; b <<= 1, c >>= 1)
      if (i & b) r |= c;
    return r;
  }
};

// X[k] = sum_j v[j] w_R^{jk} (INV: w_R^{-jk}), natural order in and out, no scaling.
template <int R, bool INV>
__device__ __forceinline__ void dft_reg(uint64_t* v) {
  if constexpr (R == 1) {
    return;
  } else {
    constexpr unsigned ER = (exp16(INV) * (16 / R)) % 192;  // w_R = 2^ER
#pragma unroll
    for (int h = R / 2; h >= 1; h >>= 1) {
#pragma unroll
      for (int s = 0; s < R; s += 2 * h) {
#pragma unroll
        for (int j = 0; j < h; ++j) {
          uint64_t u = v[s + j], w = v[s + j + h];
          v[s + j] = gl::add(u, w);
          // (u - w) w_R^t = (u - w) 2^e; for e >= 96 the sign of 2^96 = -1 is
          // taken by swapping the subtraction
          const unsigned e = (ER * (unsigned)j * (unsigned)(R / (2 * h))) % 192u;
          v[s + j + h] = e >= 96 ? gl::mul2e(gl::sub(w, u), e - 96) : gl::mul2e(gl::sub(u, w), e);
        }
      }
    }
    uint64_t tmp[R];
#pragma unroll
    for (int i = 0; i < R; ++i) tmp[BitRev<R>::v(i)] = v[i];
#pragma unroll
    for (int i = 0; i < R; ++i) v[i] = tmp[i];
  }
}

}  // namespace sg

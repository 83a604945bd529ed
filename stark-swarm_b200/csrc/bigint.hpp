// bigint.hpp — small unsigned big-integer helpers for the host witness builders
// (RSA-2048, P-256): little-endian arrays of 32-bit words.
//
// The product is schoolbook. Division is Knuth's Algorithm D (TAOCP vol. 2,
// 4.3.1): normalise so the divisor's top word has its high bit set, estimate each
// quotient word from the top two dividend words and the top divisor word, correct
// the estimate with the second divisor word, multiply and subtract, and add back
// in the rare case the estimate was still one too large.
#pragma once
#include <cstdint>
#include <cstring>
#include <vector>

namespace sg {
namespace bn {

// index of the highest non-zero word, -1 for zero
inline int top_word(const uint32_t* w, int n) {
  for (int i = n - 1; i >= 0; --i)
    if (w[i]) return i;
  return -1;
}

inline int cmp(const uint32_t* a, const uint32_t* b, int n) {
  for (int i = n - 1; i >= 0; --i)
    if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
  return 0;
}

// out (na + nb words) = a (na words) * b (nb words)
inline void mul(const uint32_t* a, int na, const uint32_t* b, int nb, uint32_t* out) {
  memset(out, 0, 4 * (na + nb));
  for (int i = 0; i < na; ++i) {
    uint64_t carry = 0;
    for (int j = 0; j < nb; ++j) {
      const uint64_t t = (uint64_t)a[i] * b[j] + out[i + j] + carry;
      out[i + j] = (uint32_t)t;
      carry = t >> 32;
    }
    out[i + nb] = (uint32_t)carry;
  }
}

// u (m words) = q * v + r with v of n significant words (m >= n >= 1, v[n-1] != 0);
// q gets m - n + 1 words, r gets n words.
inline void divmod(const uint32_t* u, int m, const uint32_t* v, int n, uint32_t* q, uint32_t* r) {
  if (n == 1) {
    uint64_t rem = 0;
    for (int i = m - 1; i >= 0; --i) {
      const uint64_t cur = rem << 32 | u[i];
      q[i] = (uint32_t)(cur / v[0]);
      rem = cur % v[0];
    }
    r[0] = (uint32_t)rem;
    return;
  }
  const int s = __builtin_clz(v[n - 1]);
  // normalised copies on the stack for the sizes the witness builders use
  // (up to 4096-bit dividends), on the heap beyond
  uint32_t vn_small[64], un_small[129];
  std::vector<uint32_t> vn_big, un_big;
  uint32_t* vn = vn_small;
  uint32_t* un = un_small;
  if (n > 64 || m + 1 > 129) {
    vn_big.resize(n);
    un_big.resize(m + 1);
    vn = vn_big.data();
    un = un_big.data();
  }
  for (int i = n - 1; i > 0; --i) vn[i] = s ? (v[i] << s | v[i - 1] >> (32 - s)) : v[i];
  vn[0] = v[0] << s;
  un[m] = s ? u[m - 1] >> (32 - s) : 0;
  for (int i = m - 1; i > 0; --i) un[i] = s ? (u[i] << s | u[i - 1] >> (32 - s)) : u[i];
  un[0] = u[0] << s;
  const uint64_t B = 1ull << 32;
  for (int j = m - n; j >= 0; --j) {
    const uint64_t top = (uint64_t)un[j + n] << 32 | un[j + n - 1];
    uint64_t qh = top / vn[n - 1], rh = top % vn[n - 1];
    while (qh >= B || qh * vn[n - 2] > (rh << 32 | un[j + n - 2])) {
      --qh;
      rh += vn[n - 1];
      if (rh >= B) break;
    }
    int64_t borrow = 0;
    uint64_t carry = 0;
    for (int i = 0; i < n; ++i) {
      const uint64_t p = qh * vn[i] + carry;
      carry = p >> 32;
      const int64_t t = (int64_t)un[i + j] - (int64_t)(uint32_t)p + borrow;
      un[i + j] = (uint32_t)t;
      borrow = t >> 32;  // 0 or -1
    }
    const int64_t t = (int64_t)un[j + n] - (int64_t)carry + borrow;
    un[j + n] = (uint32_t)t;
    if (t < 0) {
      --qh;
      uint64_t c = 0;
      for (int i = 0; i < n; ++i) {
        const uint64_t s2 = (uint64_t)un[i + j] + vn[i] + c;
        un[i + j] = (uint32_t)s2;
        c = s2 >> 32;
      }
      un[j + n] += (uint32_t)c;
    }
    q[j] = (uint32_t)qh;
  }
  for (int i = 0; i < n; ++i) r[i] = s ? (un[i] >> s | un[i + 1] << (32 - s)) : un[i];
}

}  // namespace bn
}  // namespace sg

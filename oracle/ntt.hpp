// oracle/ntt.hpp — CPU radix-2 NTT with ark-poly Radix2EvaluationDomain semantics.
//
// TEST INFRASTRUCTURE ONLY (part of the oracle; never linked into the product).
//
// ark-poly 0.4.2 (a dependency pinned in stark-stir-swarm/Cargo.lock, not vendored):
//   Radix2EvaluationDomain::new(n).fft(c)  -> [c(w^0), ..., c(w^{n-1})], natural order,
//       w = group_gen = root_of_unity(log2 n)          (fri.rs:165-168 FriDomain)
//   ifft(e) -> coefficients, including the 1/n factor.
// Call sites: trace_import.rs:272-280, lib.rs:400-410, fri.rs:273-282,357-367.
// Both are plain DFTs, so this textbook iterative Cooley-Tukey gives identical values.
#pragma once
#include <vector>
#include "gl.hpp"

namespace orc {

inline unsigned log2_exact(size_t n) {
  unsigned l = 0;
  while ((size_t(1) << l) < n) ++l;
  return l;
}

inline void bit_reverse_permute(Fp* a, size_t n) {
  unsigned lg = log2_exact(n);
  for (size_t i = 0; i < n; ++i) {
    size_t j = 0;
    for (unsigned b = 0; b < lg; ++b)
      if (i >> b & 1) j |= size_t(1) << (lg - 1 - b);
    if (i < j) { Fp t = a[i]; a[i] = a[j]; a[j] = t; }
  }
}

// In-place DFT with an arbitrary primitive n-th root `w` (n a power of two).
inline void dft_with_root(Fp* a, size_t n, Fp w) {
  if (n <= 1) return;
  bit_reverse_permute(a, n);
  std::vector<Fp> tw(n / 2);
  tw[0] = Fp::raw(1);
  for (size_t i = 1; i < n / 2; ++i) tw[i] = tw[i - 1] * w;
  for (size_t len = 2; len <= n; len <<= 1) {
    size_t half = len >> 1, step = n / len;
    for (size_t s = 0; s < n; s += len)
      for (size_t j = 0; j < half; ++j) {
        Fp u = a[s + j], t = a[s + j + half] * tw[j * step];
        a[s + j] = u + t;
        a[s + j + half] = u - t;
      }
  }
}

inline void fft(Fp* a, size_t n) {
  if (n <= 1) return;
  dft_with_root(a, n, root_of_unity(log2_exact(n)));
}

inline void ifft(Fp* a, size_t n) {
  if (n <= 1) return;
  dft_with_root(a, n, inv(root_of_unity(log2_exact(n))));
  Fp ninv = inv(Fp::raw(n));
  for (size_t i = 0; i < n; ++i) a[i] = a[i] * ninv;
}

}  // namespace orc

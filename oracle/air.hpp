// oracle/air.hpp — CPU restatement of the AIR trace builders and constraint evaluators.
//
// TEST INFRASTRUCTURE ONLY (part of the oracle; never linked into the product).
//
// HashRollup (w = 4, 3 constraints), deep_ali/src/air_workloads.rs:
//   :64-84    column meaning [idx, leaf_val, state, state_sq]
//   :571-589  build_hash_rollup_trace: state_{i+1} = state_i^2 + leaf_i
//   :591-599  eval_hash_rollup_constraints
//   :237-260  evaluate_constraints registry ids (HashRollup = variant 4)
#pragma once
#include <cstddef>
#include "gl.hpp"
#include "sha256_air.hpp"
#include "sha512_air.hpp"

namespace orc {

// AIR_SHA512 has no registry variant in the reference (it is reached through
// deep_ali_merge_sha512, lib.rs:561-641); its id here is internal to the oracle.
enum { AIR_HASH_ROLLUP = 4, AIR_SHA256 = 6, AIR_SHA512 = 100 };

inline size_t air_width(int air) {
  switch (air) {
    case AIR_HASH_ROLLUP: return 4;
    case AIR_SHA256: return sha::WIDTH;
    case AIR_SHA512: return sha512::WIDTH;
    default: return 0;
  }
}
inline size_t air_num_constraints(int air) {
  switch (air) {
    case AIR_HASH_ROLLUP: return 3;
    case AIR_SHA256: return sha::NUM_CONSTRAINTS;
    case AIR_SHA512: return sha512::NUM_CONSTRAINTS;
    default: return 0;
  }
}

// Column-major 4 x n_trace trace. Leaves past n_leaves are zero. A leaf value
// >= p is reduced mod p (the reference's F::from(u64) with 2-limb Montgomery
// would reject it; such a value occurs with probability ~2^-32 per leaf).
inline void build_hash_rollup_trace(const uint64_t* leaves, size_t n_leaves, size_t n_trace, Fp* tr) {
  Fp s;
  for (size_t i = 0; i < n_trace; ++i) {
    Fp leaf = i < n_leaves ? Fp(leaves[i]) : Fp();
    tr[0 * n_trace + i] = Fp(i);
    tr[1 * n_trace + i] = leaf;
    tr[2 * n_trace + i] = s;
    tr[3 * n_trace + i] = s * s;
    s = tr[3 * n_trace + i] + leaf;
  }
}

inline void eval_constraints(int air, const Fp* cur, const Fp* nxt, size_t row, size_t n_blocks, Fp* out) {
  switch (air) {
    case AIR_HASH_ROLLUP:
      out[0] = nxt[0] - cur[0] - Fp::raw(1);
      out[1] = cur[3] - cur[2] * cur[2];
      out[2] = nxt[2] - cur[3] - cur[1];
      break;
    case AIR_SHA256: sha::eval(cur, nxt, row, n_blocks, out); break;
    case AIR_SHA512: sha512::eval(cur, nxt, row, n_blocks, out); break;
    default: break;
  }
}

}  // namespace orc

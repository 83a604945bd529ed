// merkle.cuh — device SHA3 Merkle trees (the build's hash profile) with the
// reference's DsLabel framing.
//
// merkle/src/lib.rs:95-113 DsLabel = le64(arity) || le64(level) || le64(pos) || le64(label)
//   leaf  = SHA3(DsLabel{arities[0], u32::MAX, i, label} || le64 values)      (:185-217)
//   node  = SHA3(DsLabel{arity, parent_level, parent_pos, label} || children) (:219-238)
//   a level whose length is not a multiple of its arity is padded with copies
//   of its last node (:423-476); openings read padding as the last node (:478-512).
// Every leaf here is "row i of a column-major matrix": the packed f0 fibres
// (column stride n0/m0), STIR layer values (6 planes), coefficient tuples
// (6m planes) and LDE rows (w columns) all fit that one form.
#pragma once
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

#include "keccak.cuh"

namespace sg {

struct DevTree {
  uint64_t label = 0;
  uint32_t arity0 = 2;               // arities[0]: the arity field of every leaf label
  std::vector<uint32_t> arity;       // arity[l]: children per parent from level l to l+1
  std::vector<uint64_t> len;         // logical length of each level (len.back() == 1)
  std::vector<uint64_t> off;         // digest offset of each level inside `d`
  uint64_t* d = nullptr;             // all levels, kc::kDigestLanes lanes per digest
  uint64_t total_digests = 0;
  bool owns = false;
};

// Plan the level shapes of a tree with `n_leaves` leaves and per-level arities
// (the reference indexes arities by level; a tree stops at the first level of length 1).
// Returns false when the arities run out before the root.
bool tree_plan(DevTree* t, uint64_t n_leaves, const std::vector<uint32_t>& arities, uint64_t label);

// Hash level 0: leaf i = row i of the column-major matrix cols (width w, column
// stride cs) followed by `zeros` zero lanes.
cudaError_t tree_hash_leaves(const DevTree& t, const uint64_t* cols, uint32_t w, uint64_t cs, uint32_t zeros,
                             cudaStream_t s);
// Hash levels 1..depth from level 0.
cudaError_t tree_hash_levels(const DevTree& t, cudaStream_t s);
// The same for n_trees trees of t's shape side by side: tree g's digests at
// t.d + g * g_tree (u64) and, for the leaves, its rows at cols + g * g_cols.
cudaError_t tree_hash_leaves_group(const DevTree& t, const uint64_t* cols, uint32_t w, uint64_t cs, uint32_t zeros,
                                   uint64_t g_cols, uint64_t g_tree, uint32_t n_trees, cudaStream_t s);
cudaError_t tree_hash_levels_group(const DevTree& t, uint64_t g_tree, uint32_t n_trees, cudaStream_t s);
// Copy digests at the given global digest indices into out (kc::kDigestLanes lanes each).
cudaError_t gather_digests(const uint64_t* d, const uint64_t* idx, uint64_t n, uint64_t* out, cudaStream_t s);
// Gather u64 values src[idx[i]] into out.
cudaError_t gather_u64(const uint64_t* src, const uint64_t* idx, uint64_t n, uint64_t* out, cudaStream_t s);

// Device-side leaf hash used by fused kernels (fold writes the next layer's leaves).
#if defined(__CUDACC__)
__device__ void leaf_digest_row(const uint64_t* cols, uint32_t w, uint64_t cs, uint32_t zeros, uint64_t i,
                                uint64_t arity0, uint64_t label, uint64_t out[kc::kDigestLanes]);
#endif

// Host-side list of the global digest indices that make up opening `index`:
// [leaf, then for each level the (arity-1) siblings in group order].
void opening_indices(const DevTree& t, uint64_t index, std::vector<uint64_t>* out);

}  // namespace sg

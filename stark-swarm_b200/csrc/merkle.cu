// merkle.cu — leaf and node hashing kernels for the SHA3 Merkle channel.
#include "keccak.cuh"
#include "merkle.cuh"
#include "counters.hpp"

namespace sg {

bool tree_plan(DevTree* t, uint64_t n_leaves, const std::vector<uint32_t>& arities, uint64_t label) {
  t->label = label;
  if (arities.empty()) return false;
  t->arity0 = arities[0];
  t->arity.clear();
  t->len.assign(1, n_leaves);
  t->off.assign(1, 0);
  uint64_t total = n_leaves;
  size_t l = 0;
  while (t->len.back() > 1) {
    if (l >= arities.size() || arities[l] < 2) return false;
    uint64_t a = arities[l];
    uint64_t np = (t->len.back() + a - 1) / a;
    t->arity.push_back((uint32_t)a);
    t->off.push_back(total);
    t->len.push_back(np);
    total += np;
    ++l;
  }
  t->total_digests = total;
  return n_leaves > 0;
}

__device__ void leaf_digest_row(const uint64_t* cols, uint32_t w, uint64_t cs, uint32_t zeros, uint64_t i,
                                uint64_t arity0, uint64_t label, uint64_t out[kc::kDigestLanes]) {
  kc::LaneSponge sp;
  sp.init();
  sp.lane(arity0);
  sp.lane(0xFFFFFFFFull);
  sp.lane(i);
  sp.lane(label);
  for (uint32_t c = 0; c < w; ++c) sp.lane(__ldg(cols + (uint64_t)c * cs + i));
  for (uint32_t c = 0; c < zeros; ++c) sp.lane(0);
  sp.finish(out);
}

namespace {

constexpr int DL = kc::kDigestLanes;

__device__ __forceinline__ void put_digest(uint64_t* o, const uint64_t* d) {
#pragma unroll
  for (int q = 0; q < DL; ++q) o[q] = d[q];
}

// Generic width: runtime loop (positions resolved by the sponge's switch).
// Trees of one shape side by side (grid.y = tree g): tree g's rows start g_cols
// elements and its digests g_out elements further on.
__global__ void leaf_kernel(const uint64_t* cols, uint32_t w, uint64_t cs, uint32_t zeros, uint64_t n,
                            uint64_t arity0, uint64_t label, uint64_t* out, uint64_t g_cols, uint64_t g_out) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  cols += blockIdx.y * g_cols;
  out += blockIdx.y * g_out;
  uint64_t d[DL];
  leaf_digest_row(cols, w, cs, zeros, i, arity0, label, d);
  put_digest(out + DL * i, d);
}

// Fixed width: fully unrolled, every lane position is a compile-time constant.
template <int W, int Z>
__global__ void leaf_kernel_t(const uint64_t* __restrict__ cols, uint64_t cs, uint64_t n, uint64_t arity0,
                              uint64_t label, uint64_t* __restrict__ out, uint64_t g_cols, uint64_t g_out) {
  uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  cols += blockIdx.y * g_cols;
  out += blockIdx.y * g_out;
  kc::LaneSponge sp;
  sp.init();
  sp.lane(arity0);
  sp.lane(0xFFFFFFFFull);
  sp.lane(i);
  sp.lane(label);
#pragma unroll
  for (int c = 0; c < W; ++c) sp.lane(__ldg(cols + (uint64_t)c * cs + i));
#pragma unroll
  for (int c = 0; c < Z; ++c) sp.lane(0);
  uint64_t d[DL];
  sp.finish(d);
  put_digest(out + DL * i, d);
}

template <int A>
__device__ __forceinline__ void node_hash(const uint64_t* child, uint64_t n_child, uint64_t* parent, uint64_t p,
                                          uint64_t level, uint64_t label) {
  kc::LaneSponge sp;
  sp.init();
  sp.lane(A);
  sp.lane(level);
  sp.lane(p);
  sp.lane(label);
#pragma unroll
  for (int k = 0; k < A; ++k) {
    uint64_t c = p * A + k;
    if (c >= n_child) c = n_child - 1;  // padding = copies of the last node
    const uint64_t* cd = child + DL * c;
#pragma unroll
    for (int q = 0; q < DL; ++q) sp.lane(cd[q]);
  }
  uint64_t d[DL];
  sp.finish(d);
  put_digest(parent + DL * p, d);
}

template <int A>
__global__ void node_kernel_t(const uint64_t* __restrict__ child, uint64_t n_child, uint64_t* __restrict__ parent,
                              uint64_t n_parent, uint64_t level, uint64_t label, uint64_t g_tree) {
  uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (p < n_parent) node_hash<A>(child + blockIdx.y * g_tree, n_child, parent + blockIdx.y * g_tree, p, level, label);
}

__device__ void node_hash_any(const uint64_t* child, uint64_t n_child, uint64_t* parent, uint64_t p, uint32_t arity,
                              uint64_t level, uint64_t label) {
  kc::LaneSponge sp;
  sp.init();
  sp.lane(arity);
  sp.lane(level);
  sp.lane(p);
  sp.lane(label);
  for (uint32_t k = 0; k < arity; ++k) {
    uint64_t c = p * arity + k;
    if (c >= n_child) c = n_child - 1;  // padding = copies of the last node
    const uint64_t* cd = child + DL * c;
#pragma unroll
    for (int q = 0; q < DL; ++q) sp.lane(cd[q]);
  }
  uint64_t d[DL];
  sp.finish(d);
  put_digest(parent + DL * p, d);
}

__global__ void node_kernel(const uint64_t* child, uint64_t n_child, uint64_t* parent, uint64_t n_parent,
                            uint32_t arity, uint64_t level, uint64_t label, uint64_t g_tree) {
  uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (p < n_parent)
    node_hash_any(child + blockIdx.y * g_tree, n_child, parent + blockIdx.y * g_tree, p, arity, level, label);
}

// Keccak-f[1600] by one warp: thread t < 25 holds state lane A[t] (t = x + 5y) and
// the others follow along with lanes they never hand out. Per round, theta's column
// parities and D, pi's lane move and chi's two neighbours are warp shuffles, rho is
// the thread's own rotation. About 33 instructions a round for the warp against
// some 260 for one thread holding the whole state, so a lone permutation (the
// narrow top levels of a tree) finishes about three times sooner. The rotation
// offsets and round constants are Keccak's (FIPS 202, section 3.2).
__constant__ uint8_t kRhoOff[25] = {0, 1, 62, 28, 27, 36, 44, 6, 55, 20, 3, 10, 43, 25, 39,
                                    41, 45, 15, 21, 8, 18, 2, 61, 56, 14};

__device__ __forceinline__ uint64_t shfl64(uint64_t v, int src) {
  const uint32_t lo = __shfl_sync(0xffffffffu, (uint32_t)v, src);
  const uint32_t hi = __shfl_sync(0xffffffffu, (uint32_t)(v >> 32), src);
  return (uint64_t)hi << 32 | lo;
}

__device__ __forceinline__ uint64_t rotl_var(uint64_t v, uint32_t n) { return n ? (v << n) | (v >> (64 - n)) : v; }

__device__ void keccak_f_warp(uint64_t& a, int t) {
  const int x = t % 5, y = (t / 5) % 5;
  const int s1 = x + 5 * ((y + 1) % 5), s2 = x + 5 * ((y + 2) % 5), s3 = x + 5 * ((y + 3) % 5),
            s4 = x + 5 * ((y + 4) % 5);
  const int cm = (x + 4) % 5, cp = (x + 1) % 5;
  // pi: the lane landing at (x, y) comes from (x', y') = (3 (y - 3x) mod 5, x)
  const int pi = (3 * (y - 3 * x) % 5 + 5) % 5 + 5 * x;
  const int n1 = (x + 1) % 5 + 5 * y, n2 = (x + 2) % 5 + 5 * y;
  const uint32_t rho = t < 25 ? kRhoOff[t] : 0;
#pragma unroll 1
  for (int r = 0; r < 24; ++r) {
    const uint64_t c = kc::xor3(kc::xor3(a, shfl64(a, s1), shfl64(a, s2)), shfl64(a, s3), shfl64(a, s4));
    a = kc::xor3(a, shfl64(c, cm), kc::rotl(shfl64(c, cp), 1));
    const uint64_t b = shfl64(rotl_var(a, rho), pi);
    a = kc::chi(b, shfl64(b, n1), shfl64(b, n2));
    if (t == 0) a ^= kc::kRC_dev[r];
  }
}

// node_hash by one warp: lane j of the message (arity, level, p, label, then the
// children's digests) goes into rate position j mod kRateLanes of block j / kRateLanes,
// padded as LaneSponge::finish does.
__device__ void node_hash_warp(const uint64_t* child, uint64_t n_child, uint64_t* parent, uint64_t p,
                               uint32_t arity, uint64_t level, uint64_t label, int t) {
  const uint32_t total = 4 + arity * DL;
  uint64_t a = 0;
  for (uint32_t b0 = 0;; b0 += kc::kRateLanes) {
    if (t < kc::kRateLanes) {
      const uint32_t j = b0 + t;
      uint64_t w = 0;
      if (j < total) {
        if (j < 4) {
          w = j == 0 ? arity : j == 1 ? level : j == 2 ? p : label;
        } else {
          uint64_t c = p * arity + (j - 4) / DL;
          if (c >= n_child) c = n_child - 1;  // padding = copies of the last node
          w = child[DL * c + (j - 4) % DL];
        }
      } else if (j == total) {
        w = 0x06ull;
      }
      if (t == kc::kRateLanes - 1 && b0 + kc::kRateLanes > total) w ^= 0x8000000000000000ull;
      a ^= w;
    }
    keccak_f_warp(a, t);
    if (b0 + kc::kRateLanes > total) break;
  }
  if (t < DL) parent[DL * p + t] = a;
}

// The levels from the first one of at most kTopWork Keccak-f (parents x
// permutations per node: two per thread of the CTA) upward, in one CTA: each level
// is a block-wide loop over its parents, then a barrier (which makes the level's
// global writes visible to the whole block) before the next. Larger levels go to
// the whole GPU: on one SM a level of 1024 arity-16 parents (4096 Keccak-f) took
// about 0.2 ms, against a few microseconds spread over 148 SMs. Levels of at most
// 48 parents hash each node with a warp (node_hash_warp): the tree tops of a
// 64-byte SHA-256 proof went from 0.42 to 0.33 ms.
constexpr int kTopThreads = 512;
constexpr uint64_t kTopWork = 2 * kTopThreads;
// Keccak-f per node hash: the 4-lane label and `arity` digests, padded
inline uint64_t node_perms(uint64_t arity) { return (4 + arity * DL) / kc::kRateLanes + 1; }
constexpr int kMaxTopLevels = 24;
struct TopLevels {
  int n;
  uint32_t arity[kMaxTopLevels];
  uint64_t n_child[kMaxTopLevels], child_off[kMaxTopLevels], parent_off[kMaxTopLevels], n_parent[kMaxTopLevels];
  uint64_t level[kMaxTopLevels];
};

// one CTA per tree of a group (tree g's digests at d + g g_tree)
__global__ void __launch_bounds__(kTopThreads) tree_top_kernel(uint64_t* d, TopLevels tl, uint64_t label,
                                                               uint64_t g_tree) {
  d += blockIdx.x * g_tree;
  constexpr int kWarps = kTopThreads / 32;
  for (int k = 0; k < tl.n; ++k) {
    const uint64_t* ch = d + DL * tl.child_off[k];
    uint64_t* par = d + DL * tl.parent_off[k];
    // a narrow level (at most three nodes a warp): a warp per node, whose permutations
    // take about a third of one thread's
    if (tl.n_parent[k] <= 3 * kWarps) {
      const int w = threadIdx.x >> 5, t = threadIdx.x & 31;
      for (uint64_t p = w; p < tl.n_parent[k]; p += kWarps)
        node_hash_warp(ch, tl.n_child[k], par, p, tl.arity[k], tl.level[k], label, t);
      __syncthreads();
      continue;
    }
    for (uint64_t p = threadIdx.x; p < tl.n_parent[k]; p += kTopThreads) {
      switch (tl.arity[k]) {
        case 2: node_hash<2>(ch, tl.n_child[k], par, p, tl.level[k], label); break;
        case 4: node_hash<4>(ch, tl.n_child[k], par, p, tl.level[k], label); break;
        case 8: node_hash<8>(ch, tl.n_child[k], par, p, tl.level[k], label); break;
        case 16: node_hash<16>(ch, tl.n_child[k], par, p, tl.level[k], label); break;
        default: node_hash_any(ch, tl.n_child[k], par, p, tl.arity[k], tl.level[k], label); break;
      }
    }
    __syncthreads();
  }
}

__global__ void gather_digests_kernel(const uint64_t* d, const uint64_t* idx, uint64_t n, uint64_t* out) {
  uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (e >= DL * n) return;
  out[e] = d[DL * idx[e / DL] + e % DL];
}

__global__ void gather_u64_kernel(const uint64_t* src, const uint64_t* idx, uint64_t n, uint64_t* out) {
  uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (e < n) out[e] = src[idx[e]];
}

inline unsigned blocks_for(uint64_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

cudaError_t tree_hash_leaves(const DevTree& t, const uint64_t* cols, uint32_t w, uint64_t cs, uint32_t zeros,
                             cudaStream_t s) {
  return tree_hash_leaves_group(t, cols, w, cs, zeros, 0, 0, 1, s);
}

cudaError_t tree_hash_leaves_group(const DevTree& t, const uint64_t* cols, uint32_t w, uint64_t cs, uint32_t zeros,
                                   uint64_t g_cols, uint64_t g_tree, uint32_t n_trees, cudaStream_t s) {
  if (n_trees == 0 || n_trees > 65535) return cudaErrorInvalidValue;
  const uint64_t n = t.len[0];
  const unsigned T = 128;
  const dim3 B(blocks_for(n, T), n_trees);
#define SG_LEAF_CASE(WW, ZZ)                                                                   \
  if (w == WW && zeros == ZZ) {                                                                \
    SG_LAUNCH_SCOPE("merkle_leaves", s);                                                       \
    leaf_kernel_t<WW, ZZ><<<B, T, 0, s>>>(cols, cs, n, t.arity0, t.label, t.d, g_cols, g_tree); \
    return cudaGetLastError();                                                                 \
  }
  SG_LEAF_CASE(1, 5)
  SG_LEAF_CASE(2, 0)
  SG_LEAF_CASE(4, 0)
  SG_LEAF_CASE(6, 0)
  SG_LEAF_CASE(8, 0)
  SG_LEAF_CASE(16, 0)
  SG_LEAF_CASE(64, 0)
#undef SG_LEAF_CASE
  SG_LAUNCH_SCOPE("merkle_leaves", s);
  leaf_kernel<<<B, T, 0, s>>>(cols, w, cs, zeros, n, t.arity0, t.label, t.d, g_cols, g_tree);
  return cudaGetLastError();
}

cudaError_t tree_hash_levels(const DevTree& t, cudaStream_t s) { return tree_hash_levels_group(t, 0, 1, s); }

cudaError_t tree_hash_levels_group(const DevTree& t, uint64_t g_tree, uint32_t n_trees, cudaStream_t s) {
  if (n_trees == 0 || n_trees > 65535) return cudaErrorInvalidValue;
  for (size_t l = 0; l + 1 < t.len.size(); ++l) {
    const uint64_t np = t.len[l + 1];
    if (np * node_perms(t.arity[l]) <= kTopWork && t.len.size() - 1 - l <= (size_t)kMaxTopLevels) {
      TopLevels tl{};
      for (size_t k = l; k + 1 < t.len.size(); ++k, ++tl.n) {
        tl.arity[tl.n] = t.arity[k];
        tl.n_child[tl.n] = t.len[k];
        tl.child_off[tl.n] = t.off[k];
        tl.parent_off[tl.n] = t.off[k + 1];
        tl.n_parent[tl.n] = t.len[k + 1];
        tl.level[tl.n] = k + 1;
      }
      SG_LAUNCH_SCOPE("merkle_nodes", s);
      tree_top_kernel<<<n_trees, kTopThreads, 0, s>>>(t.d, tl, t.label, g_tree);
      return cudaGetLastError();
    }
    const uint64_t* ch = t.d + DL * t.off[l];
    uint64_t* par = t.d + DL * t.off[l + 1];
    const dim3 B(blocks_for(np, 128), n_trees);
    SG_LAUNCH_SCOPE("merkle_nodes", s);
    switch (t.arity[l]) {
      case 2: node_kernel_t<2><<<B, 128, 0, s>>>(ch, t.len[l], par, np, l + 1, t.label, g_tree); break;
      case 4: node_kernel_t<4><<<B, 128, 0, s>>>(ch, t.len[l], par, np, l + 1, t.label, g_tree); break;
      case 8: node_kernel_t<8><<<B, 128, 0, s>>>(ch, t.len[l], par, np, l + 1, t.label, g_tree); break;
      case 16: node_kernel_t<16><<<B, 128, 0, s>>>(ch, t.len[l], par, np, l + 1, t.label, g_tree); break;
      default: node_kernel<<<B, 128, 0, s>>>(ch, t.len[l], par, np, t.arity[l], l + 1, t.label, g_tree); break;
    }
  }
  return cudaGetLastError();
}

cudaError_t gather_digests(const uint64_t* d, const uint64_t* idx, uint64_t n, uint64_t* out, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  SG_LAUNCH_SCOPE("gather", s);
  gather_digests_kernel<<<blocks_for(DL * n, 256), 256, 0, s>>>(d, idx, n, out);
  return cudaGetLastError();
}

cudaError_t gather_u64(const uint64_t* src, const uint64_t* idx, uint64_t n, uint64_t* out, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  SG_LAUNCH_SCOPE("gather", s);
  gather_u64_kernel<<<blocks_for(n, 256), 256, 0, s>>>(src, idx, n, out);
  return cudaGetLastError();
}

void opening_indices(const DevTree& t, uint64_t index, std::vector<uint64_t>* out) {
  out->push_back(t.off[0] + index);
  uint64_t idx = index;
  for (size_t l = 0; l + 1 < t.len.size(); ++l) {
    uint64_t a = t.arity[l], g = (idx / a) * a;
    for (uint64_t k = 0; k < a; ++k) {
      uint64_t pos = g + k;
      if (pos == idx) continue;
      if (pos >= t.len[l]) pos = t.len[l] - 1;
      out->push_back(t.off[l] + pos);
    }
    idx /= a;
  }
}

}  // namespace sg

// oracle/merkle.hpp — CPU restatement of the reference's SHA3 Merkle channel.
//
// TEST INFRASTRUCTURE ONLY (part of the oracle; never linked into the product).
//
// Follows merkle/src/lib.rs:
//   :95-113   DsLabel = le64(arity) || le64(level) || le64(position) || le64(tree_label)
//   :115      LEAF_LEVEL_DS = u32::MAX
//   :185-217  leaf = SHA3(DsLabel{arities[0], u32::MAX, i, label} || le64 canonical values)
//   :219-238  node = SHA3(DsLabel{arity, parent_level, parent_pos, label} || children)
//   :423-476  finalize: pad each level with copies of its last node to a multiple of the
//             level's arity; parent level index = child level index + 1
//   :478-512  open: siblings of the group, padding read as the last node
//   :754-800  verify_opening
// and deep_ali/src/fri.rs:950-959 (merkle_depth), :1094-1103 (pick_arity_for_layer).
#pragma once
#include <array>
#include <vector>
#include "gl.hpp"
#include "keccak.hpp"

namespace orc {

using Digest = std::array<uint8_t, HASH_BYTES>;

inline size_t pick_arity_for_layer(size_t n, size_t m) {
  const size_t cands[] = {128, 64, 32, 16, 8, 4};
  for (size_t c : cands)
    if (m >= c && n % c == 0) return c;
  return n % 2 == 0 ? 2 : 1;
}

inline size_t merkle_depth(size_t leaves, size_t arity) {
  size_t depth = 1, cur = leaves;
  while (cur > arity) {
    cur = (cur + arity - 1) / arity;
    ++depth;
  }
  return depth;
}

inline void ds_label(uint8_t out[32], uint64_t arity, uint64_t level, uint64_t pos, uint64_t label) {
  memcpy(out, &arity, 8);
  memcpy(out + 8, &level, 8);
  memcpy(out + 16, &pos, 8);
  memcpy(out + 24, &label, 8);
}

inline Digest leaf_hash(size_t arity0, uint64_t label, uint64_t pos, const Fp* vals, size_t n) {
  uint8_t ds[32];
  ds_label(ds, arity0, 0xFFFFFFFFull, pos, label);
  SelectedHasher h;
  h.update(ds, 32);
  for (size_t i = 0; i < n; ++i) h.update(&vals[i].v, 8);
  Digest d;
  h.finalize(d.data());
  return d;
}

inline Digest node_hash(size_t arity, uint64_t label, uint64_t level, uint64_t pos, const Digest* ch) {
  uint8_t ds[32];
  ds_label(ds, arity, level, pos, label);
  SelectedHasher h;
  h.update(ds, 32);
  for (size_t i = 0; i < arity; ++i) h.update(ch[i].data(), HASH_BYTES);
  Digest d;
  h.finalize(d.data());
  return d;
}

struct MerkleOpening {
  Digest leaf;
  std::vector<std::vector<Digest>> path;
  uint64_t index;
};

struct MerkleTree {
  std::vector<size_t> arities;
  uint64_t label;
  std::vector<std::vector<Digest>> levels;

  MerkleTree(std::vector<size_t> ar, uint64_t lbl) : arities(std::move(ar)), label(lbl) {}

  // leaves: n_leaves rows of `width` values each (row-major)
  void build(const std::vector<Fp>& leaves_rm, size_t width) {
    size_t n = width ? leaves_rm.size() / width : 0;
    levels.assign(1, std::vector<Digest>(n));
#pragma omp parallel for schedule(static) if (n >= 256)
    for (long i = 0; i < (long)n; ++i)
      levels[0][i] = leaf_hash(arities[0], label, i, &leaves_rm[i * width], width);
    finalize();
  }
  void finalize() {
    size_t level = 0;
    while (levels[level].size() > 1) {
      size_t ar = arities.at(level);
      auto& cur = levels[level];
      if (cur.size() % ar) {
        Digest last = cur.back();
        cur.resize(cur.size() + (ar - cur.size() % ar), last);
      }
      size_t np = cur.size() / ar;
      std::vector<Digest> par(np);
#pragma omp parallel for schedule(static) if (np >= 256)
      for (long i = 0; i < (long)np; ++i) par[i] = node_hash(ar, label, level + 1, i, &cur[i * ar]);
      levels.push_back(std::move(par));
      ++level;
    }
  }
  Digest root() const { return levels.back()[0]; }
  MerkleOpening open(size_t index) const {
    MerkleOpening o;
    o.leaf = levels[0][index];
    o.index = index;
    size_t idx = index;
    for (size_t lv = 0; lv + 1 < levels.size(); ++lv) {
      const auto& nodes = levels[lv];
      size_t ar = arities[lv];
      size_t g = (idx / ar) * ar;
      std::vector<Digest> sib;
      for (size_t i = 0; i < ar; ++i) {
        size_t pos = g + i;
        if (pos == idx) continue;
        sib.push_back(pos < nodes.size() ? nodes[pos] : nodes.back());
      }
      o.path.push_back(sib);
      idx /= ar;
    }
    return o;
  }
};

inline bool verify_opening(const std::vector<size_t>& arities, uint64_t label, const Digest& root,
                           const MerkleOpening& o) {
  Digest cur = o.leaf;
  size_t idx = o.index;
  for (size_t lv = 0; lv < o.path.size(); ++lv) {
    if (lv >= arities.size()) return false;
    size_t ar = arities[lv], pos = idx % ar;
    std::vector<Digest> ch;
    size_t k = 0;
    for (size_t i = 0; i < ar; ++i) {
      if (i == pos) ch.push_back(cur);
      else {
        if (k >= o.path[lv].size()) return false;
        ch.push_back(o.path[lv][k++]);
      }
    }
    cur = node_hash(ar, label, lv + 1, idx / ar, ch.data());
    idx /= ar;
  }
  return cur == root;
}

}  // namespace orc

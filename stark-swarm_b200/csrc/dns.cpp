// dns.cpp — the DNS-shard steps either side of the prover (swarm-dns/src/dns.rs,
// swarm-dns/src/prover.rs): doubly salted record leaf hashes, the domain-separated
// binary SHA3-256 Merkle tree over them, its inclusion paths, and the shard
// pi_hash. Host code: a zone's records are hashed with one thread per core.
#include <algorithm>
#include <cstring>
#include <thread>
#include <vector>

#include "dns.hpp"
#include "keccak.cuh"

namespace sg {
namespace {

void sha3_parts(std::initializer_list<std::pair<const void*, size_t>> parts, uint8_t out[32]) {
  kc::Sha3 h;
  for (auto& p : parts) h.update(p.first, p.second);
  h.finalize(out);
}

void dns_node(const uint8_t l[32], const uint8_t r[32], uint8_t out[32]) {
  sha3_parts({{"DNS-NODE-V1", 11}, {l, 32}, {r, 32}}, out);
}

}  // namespace

// DnsRecord::h1 / leaf_hash (dns.rs:56-79):
//   h1 = SHA3("DNS-LEAF-V1" || salt || canonical), h2 = SHA3("DNS-LEAF-DOUBLE-V1" || salt || h1)
void dns_record_leaves(const uint8_t* canon, const size_t* offsets, size_t n, const uint8_t salt[16],
                       uint8_t* out) {
  auto run = [&](size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; ++i) {
      uint8_t h1[32];
      sha3_parts({{"DNS-LEAF-V1", 11}, {salt, 16}, {canon + offsets[i], offsets[i + 1] - offsets[i]}}, h1);
      sha3_parts({{"DNS-LEAF-DOUBLE-V1", 18}, {salt, 16}, {h1, 32}}, out + 32 * i);
    }
  };
  const size_t hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t nt = std::min<size_t>(hw, n / 1024);
  if (nt <= 1) return run(0, n);
  std::vector<std::thread> th;
  const size_t chunk = (n + nt - 1) / nt;
  for (size_t t = 0; t < nt; ++t) th.emplace_back(run, t * chunk, std::min(n, (t + 1) * chunk));
  for (auto& x : th) x.join();
}

// merkle_build (dns.rs:85-102): level l+1 pairs level l, an odd last node with itself.
std::vector<std::vector<uint8_t>> dns_merkle_levels(const uint8_t* leaves, size_t n) {
  std::vector<std::vector<uint8_t>> lv(1, std::vector<uint8_t>(leaves, leaves + 32 * n));
  while (lv.back().size() > 32) {
    const std::vector<uint8_t>& prev = lv.back();
    const size_t m = prev.size() / 32;
    std::vector<uint8_t> next(32 * ((m + 1) / 2));
    for (size_t i = 0; i < m; i += 2) {
      const uint8_t* l = prev.data() + 32 * i;
      const uint8_t* r = i + 1 < m ? l + 32 : l;
      dns_node(l, r, next.data() + 32 * (i / 2));
    }
    lv.push_back(std::move(next));
  }
  return lv;
}

// merkle_path (dns.rs:104-114): the sibling at each level (the node itself when it has none).
std::vector<uint8_t> dns_merkle_path(const std::vector<std::vector<uint8_t>>& lv, size_t index) {
  std::vector<uint8_t> path;
  for (size_t l = 0; l + 1 < lv.size(); ++l) {
    const size_t m = lv[l].size() / 32, sib = index ^ 1;
    const uint8_t* d = lv[l].data() + 32 * (sib < m ? sib : index);
    path.insert(path.end(), d, d + 32);
    index /= 2;
  }
  return path;
}

// merkle_verify (dns.rs:116-131)
bool dns_merkle_verify(const uint8_t leaf[32], size_t index, const uint8_t* path, size_t depth,
                       const uint8_t root[32]) {
  uint8_t cur[32];
  memcpy(cur, leaf, 32);
  for (size_t l = 0; l < depth; ++l) {
    uint8_t nx[32];
    if (index & 1)
      dns_node(path + 32 * l, cur, nx);
    else
      dns_node(cur, path + 32 * l, nx);
    memcpy(cur, nx, 32);
    index /= 2;
  }
  return memcmp(cur, root, 32) == 0;
}

// prove_inner_shard's pi_hash (prover.rs:207-214)
void shard_pi_hash(const uint8_t salt[16], uint64_t count, const uint8_t root[32], const uint8_t root_f0[32],
                   const uint8_t fs_binding[32], uint8_t out[32]) {
  uint8_t cnt[8];
  for (int i = 0; i < 8; ++i) cnt[i] = (uint8_t)(count >> (8 * i));
  sha3_parts({{"DNS-SHARD-PIHASH-V1", 19}, {salt, 16}, {cnt, 8}, {root, 32}, {root_f0, 32}, {fs_binding, 32}},
             out);
}

}  // namespace sg

// dns.hpp — DNS-shard helpers around the prover (swarm-dns/src/dns.rs, prover.rs).
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

namespace sg {

// Doubly salted leaf hashes of n records in canonical form (record i is
// canon[offsets[i] .. offsets[i+1])); out: n x 32 bytes.
void dns_record_leaves(const uint8_t* canon, const size_t* offsets, size_t n, const uint8_t salt[16],
                       uint8_t* out);
// All levels of the DNS Merkle tree over n leaf hashes (level 0 = the leaves).
std::vector<std::vector<uint8_t>> dns_merkle_levels(const uint8_t* leaves, size_t n);
// Inclusion path of leaf `index`: one 32-byte sibling per level below the root.
std::vector<uint8_t> dns_merkle_path(const std::vector<std::vector<uint8_t>>& levels, size_t index);
bool dns_merkle_verify(const uint8_t leaf[32], size_t index, const uint8_t* path, size_t depth,
                       const uint8_t root[32]);
// pi_hash of an inner shard: SHA3("DNS-SHARD-PIHASH-V1" || salt || le64(count) || root || root_f0 || fs_binding)
void shard_pi_hash(const uint8_t salt[16], uint64_t count, const uint8_t root[32], const uint8_t root_f0[32],
                   const uint8_t fs_binding[32], uint8_t out[32]);

}  // namespace sg

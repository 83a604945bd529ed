"""Synthetic DNS zone and shard inputs for the golden-proof fixtures.

Restates, for test-input generation only, the reference code that produced
the committed golden proofs (paths relative to stark-stir-swarm/crates/):
  swarm-ctrl/src/main.rs:1331-1355  build_synthetic_zone
  swarm-ctrl/src/main.rs:1317-1329  split_evenly; shard_id = index + 1 (:820)
  swarm-dns/src/dns.rs:41-79        DnsRecord::canonical_bytes / h1 / leaf_hash
  swarm-dns/src/dns.rs:85-102       merkle_build (DNS-NODE-V1, odd node duplicated)
  swarm-proto/src/messages.rs:162-176 shard_fs_binding
  swarm-dns/src/prover.rs:207-214   pi_hash
  deep_ali/src/air_workloads.rs:611-620 pack_hash_to_leaves (4 x le64 per digest)
"""
import hashlib
import struct


def sha3(*parts: bytes) -> bytes:
    h = hashlib.sha3_256()
    for p in parts:
        h.update(p)
    return h.digest()


def canonical_bytes(domain: str, rtype: int, ttl: int, rdata: bytes) -> bytes:
    d = domain.encode()
    return (b"DNS-RECORD-V1" + struct.pack("<I", len(d)) + d + struct.pack("<H", rtype)
            + struct.pack("<I", ttl) + struct.pack("<I", len(rdata)) + rdata)


def synthetic_zone(n: int):
    recs = []
    for i in range(n):
        k = i % 4
        if k == 0:
            recs.append((f"host-{i:08x}.example.com", 1, 300,
                         bytes([10, (i >> 16) & 0xFF, (i >> 8) & 0xFF, i & 0xFF])))
        elif k == 1:
            recs.append((f"v6-{i:08x}.example.com", 28, 300,
                         struct.pack(">Q", i) + struct.pack(">Q", i ^ 0xCAFEBABEDEADBEEF)))
        elif k == 2:
            recs.append((f"txt-{i:08x}.example.com", 16, 60, f"v=auth1;rec={i}".encode()))
        else:
            recs.append((f"mail-{i:08x}.example.com", 15, 300,
                         struct.pack(">H", i % 1000) + f"mx{i & 0xFF}.example.com".encode()))
    return recs


def split_evenly(records, n_shards):
    base, rem = divmod(len(records), n_shards)
    out, i = [], 0
    for s in range(n_shards):
        ln = base + (1 if s < rem else 0)
        out.append(records[i:i + ln])
        i += ln
    return out


def record_leaf_hash(rec, salt: bytes) -> bytes:
    h1 = sha3(b"DNS-LEAF-V1", salt, canonical_bytes(*rec))
    return sha3(b"DNS-LEAF-DOUBLE-V1", salt, h1)


def dns_merkle_root(leaves):
    lv = list(leaves)
    while len(lv) > 1:
        nxt = []
        for i in range(0, len(lv), 2):
            left = lv[i]
            right = lv[i + 1] if i + 1 < len(lv) else lv[i]
            nxt.append(sha3(b"DNS-NODE-V1", left, right))
        lv = nxt
    return lv[0]


def shard_fs_binding(pk_hash: bytes, job_id: bytes, shard_id: int, nonce: bytes) -> bytes:
    return sha3(b"DNS-SWARM-SHARD-FS-V1", pk_hash, job_id, struct.pack("<I", shard_id), nonce)


def pack_hashes_to_leaves(hashes):
    out = []
    for h in hashes:
        out.extend(struct.unpack("<4Q", h))
    return out


def shard_pi_hash(salt, count, root, root_f0, fs_binding) -> bytes:
    return sha3(b"DNS-SHARD-PIHASH-V1", salt, struct.pack("<Q", count), root, root_f0, fs_binding)


def inner_shard_inputs(fx: dict, shard: dict):
    """Return (rollup leaves, fs_binding, dns merkle root) for one fixture shard."""
    salt = bytes.fromhex(fx["zone_salt_hex"])
    recs = split_evenly(synthetic_zone(fx["record_count"]), fx["shard_count"])[shard["shard_id"] - 1]
    lh = [record_leaf_hash(r, salt) for r in recs]
    fsb = shard_fs_binding(bytes.fromhex(fx["authority_pk_hash_hex"]), bytes.fromhex(fx["job_id_hex"]),
                           shard["shard_id"], bytes.fromhex(shard["shard_nonce_hex"]))
    return pack_hashes_to_leaves(lh), fsb, dns_merkle_root(lh), len(recs)


def outer_rollup_inputs(fx: dict):
    pis = [bytes.fromhex(h) for h in fx["inner_pi_hashes_hex"]]
    return pack_hashes_to_leaves(pis), bytes.fromhex(fx["authority_pk_hash_hex"])

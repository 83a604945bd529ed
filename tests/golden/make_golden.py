"""Regenerate tests/golden/golden_proofs.json from the reference checkout.

Reads stark-stir-swarm/primary-state/zone_bundle.json and the four proof
files it names (reference-produced: proofs/outer-rollup.bin and
proofs/inner-shard-000{1,2,3}.bin) and records, per proof, its inputs, byte
length, SHA3-256 digest and a few decoded fields. The tests then check that
the oracle and the GPU library reproduce each proof byte for byte without
the reference being present.

Usage: python tests/golden/make_golden.py path/to/stark-stir-swarm

The path of the reference checkout is required.
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py path/to/stark-stir-swarm")
    root = sys.argv[1]
    state = os.path.join(root, "primary-state")
    b = json.load(open(os.path.join(state, "zone_bundle.json")))

    def proof_entry(path):
        data = open(os.path.join(state, path), "rb").read()
        return {
            "path": path,
            "len": len(data),
            "sha3_256": hashlib.sha3_256(data).hexdigest(),
            "root_f0_hex": data[:32].hex(),
            "head_hex": data[:256].hex(),
        }

    fx = {
        "source": "stark-stir-swarm/primary-state/zone_bundle.json",
        "zone_salt_hex": b["zone_salt_hex"],
        "record_count": b["record_count"],
        "shard_count": b["shard_count"],
        "ldt": b["ldt"],
        "authority_pk_hash_hex": b["authority_pk_hash_hex"],
        "job_id_hex": b["job_id_hex"],
        "inner_pi_hashes_hex": b["inner_pi_hashes_hex"],
        "outer": dict(proof_entry(b["outer_proof_path"]), n_trace=b["outer_n_trace"], n0=b["outer_n0"],
                      root_f0_expected_hex=b["outer_root_f0_hex"]),
        "shards": [],
    }
    for w in b["inner_workers"]:
        e = proof_entry(w["proof_path"])
        e.update(shard_id=w["shard_id"], shard_nonce_hex=w["shard_nonce_hex"], pi_hash_hex=w["pi_hash_hex"],
                 merkle_root_hex=w["merkle_root_hex"], record_count=w["record_count"], n_trace=w["n_trace"],
                 n0=w["n_trace"] * 32)
        fx["shards"].append(e)
    out = os.path.join(HERE, "golden_proofs.json")
    with open(out, "w") as f:
        json.dump(fx, f, indent=1)
    print("wrote", out)


if __name__ == "__main__":
    main()

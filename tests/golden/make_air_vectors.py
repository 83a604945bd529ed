"""Regenerate tests/golden/air_vectors.json from the reference's own AIR sources.

For each wide AIR the reference's constraint evaluator -- the Rust function
itself, run by the subset interpreter in rust_subset.py -- is evaluated on
rows of uniformly random field elements (seeded numpy draws), at rows chosen
to hit every phase of the AIR's row gating. Random rows make every constraint
polynomial non-zero, so the recorded vectors fix the emission order, the
column offsets each constraint reads and the exact polynomial of each
constraint (b·(1−b) and b² − b differ in sign, and λ_j = j + 1 multiplies
the j-th value). Each case records the row, the seed, the vector's length,
the SHA3-256 of its little-endian u64 encoding, its first values and its
λ-weighted sum Σ (j+1)·c_j.

Evaluators (paths within stark-stir-swarm/crates/deep_ali/src):
  sha256  eval_sha256_constraints              sha256_air.rs:956
  sha512  eval_sha512_constraints              sha512_air.rs:909
  rsa     eval_rsa_stacked_per_row             rsa2048_stacked_air.rs:84
          (layout build_rsa_stacked_layout, rsa2048_stacked_air.rs:44)
  p256    eval_ecdsa_double_multirow_per_row   p256_ecdsa_double_multirow_air.rs:236
          (layout build_ecdsa_double_multirow_layout(0), :63)
  ed25519 eval_verify_air_v16_per_row          ed25519_verify_air.rs:4870
          (layout verify_air_layout_v16, :4741, from a signature made by the
          RFC 8032 signer in tests/oracle_ed25519.py; the layout builder's
          decompressions run in the interpreter too)

For the Ed25519 files the interpreter is given one native routine in Python:
FieldElement::mul (ed25519_field.rs:296-347) as the exact product mod 2^255 - 19
in tight limbs. The Rust routine packs a u256 product with u128 wrapping
arithmetic that the untyped interpreter cannot model; its result is that
product (it can differ only by representing one of the 19 values below 19 as
that value + p, which none of these inputs reaches).

The test tests/test_air_vectors.py regenerates the same rows and checks the
oracle's evaluators against these records; the reference is not read then.

Usage: python tests/golden/make_air_vectors.py path/to/stark-stir-swarm [air ...]
(with AIR names, only those entries are regenerated; the others are kept)
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))
import rust_subset as R  # noqa: E402

P = R.P

# (air, evaluator inputs) cases; the rows cover every gating phase
SHA256_CASES = [(0, 1), (5, 1), (14, 1), (15, 1), (20, 1), (62, 1), (63, 1), (64, 1), (65, 1), (127, 1),
                (148, 2), (192, 2), (300, 2)]
SHA512_CASES = [(0, 1), (15, 1), (16, 1), (40, 1), (78, 1), (79, 1), (80, 1), (81, 1), (127, 1), (150, 2),
                (300, 2)]
RSA_CASES = [(1, 0), (1, 7), (1, 16), (1, 30), (1, 31), (2, 16), (2, 31)]
P256_CASES = [(256, 0), (256, 129), (256, 255), (8, 7)]
# (key seed tag, message, k_scalar, rows): one SHA-512 block with K = 8 and K = 256, two blocks with K = 16;
# the rows hit every gate: SHA-512 rows, the digest row, reduction, both decompressions, the first, a
# middle and the last row of both ladders, the residual row, the three doublings, the result row and idle rows
ED25519_CASES = [
    ("k0", b"m" * 32, 8, [0, 15, 16, 80, 126, 127, 128, 129, 130, 131, 135, 138, 139, 146, 147, 148, 149, 150,
                           151, 152, 255]),
    ("k1", bytes(range(32)), 256, [0, 126, 127, 128, 129, 130, 131, 300, 386, 387, 500, 642, 643, 644, 645, 646,
                                   647, 648, 1023]),
    ("k2", b"two sha-512 blocks: " + bytes(range(80)), 16, [0, 127, 128, 254, 255, 256, 257, 258, 259, 274, 275,
                                                           290, 291, 292, 294, 295, 296, 511]),
]


def rows_for(seed, width):
    """the case's (cur, nxt) rows: uniform field elements from numpy's PCG64 stream"""
    rng = np.random.default_rng(seed)
    return (rng.integers(0, P, width, dtype=np.uint64), rng.integers(0, P, width, dtype=np.uint64))


def record(vals, row, seed, extra):
    v = np.array(vals, dtype=np.uint64)
    lam = sum((j + 1) * int(x) for j, x in enumerate(v)) % P
    return dict(extra, row=row, seed=seed, n=int(v.size), sha3_256=hashlib.sha3_256(v.tobytes()).hexdigest(),
                head=[int(x) for x in v[:4]], lambda_sum=lam)


def fe_list(a):
    return [R.Fe(int(x)) for x in a]


ED_OFF = [0, 26, 51, 77, 102, 128, 153, 179, 204, 230]
ED_W = [26, 25] * 5
ED_P = 2 ** 255 - 19


def _fe25519_mul(a, b):
    """FieldElement::mul as the exact product mod 2^255 - 19 in tight limbs (see the module docstring)"""
    va = sum(l << ED_OFF[i] for i, l in enumerate(a.limbs)) % ED_P
    vb = sum(l << ED_OFF[i] for i, l in enumerate(b.limbs)) % ED_P
    v = va * vb % ED_P
    return R.Struct("FieldElement", {"limbs": [(v >> ED_OFF[i]) & ((1 << ED_W[i]) - 1) for i in range(10)]})


def ed25519_entry(src):
    import hashlib as _h
    import oracle_ed25519 as OE
    files = ("ed25519_field.rs", "ed25519_field_air.rs", "ed25519_group.rs", "ed25519_group_air.rs",
             "ed25519_scalar.rs", "ed25519_scalar_air.rs", "ed25519_scalar_mult_air.rs", "sha512_air.rs",
             "ed25519_verify_air.rs")
    it = R.Interp(R.parse_sources([open(os.path.join(src, f)).read() for f in files]),
                  extra_builtins={"FieldElement::mul": _fe25519_mul})
    layouts, cases = [], []
    for li, (tag, msg, K, rows) in enumerate(ED25519_CASES):
        seed_key = _h.sha256(tag.encode()).digest()
        _, _, pub = OE.keypair(seed_key)
        sig = OE.sign(seed_key, msg)
        s_bits = [bool(b) for b in OE.ladder_bits(sig[32:], K)]
        k_bits = [bool(b) for b in OE.ladder_bits(OE.k_scalar_bytes(sig, pub, msg), K)]
        lay = it.call("verify_air_layout_v16", 64 + len(msg), s_bits, k_bits, list(sig[:32]), list(pub))
        n = it.call("verify_v16_per_row_constraints", K)
        layouts.append({"key_tag": tag, "msg_hex": msg.hex(), "k_scalar": K, "width": lay.width,
                        "height": lay.height, "constraints": n,
                        "rows": {k: getattr(lay, k) for k in ("k_hash", "reduce_row", "decompress_R_row",
                                                               "decompress_A_row", "sB_first_row", "kA_first_row",
                                                               "residual_row", "dbl_1_row", "dbl_2_row",
                                                               "dbl_3_row", "result_row")}})
        for j, row in enumerate(rows):
            seed = 25519000 + 100 * li + j
            cur, nxt = rows_for(seed, lay.width)
            vals = it.call("eval_verify_air_v16_per_row", fe_list(cur), fe_list(nxt), row, lay)
            cases.append(record([x.v for x in vals], row, seed, {"layout": li}))
    return {"evaluator": "ed25519_verify_air.rs:eval_verify_air_v16_per_row", "layouts": layouts, "cases": cases}


def main():
    if len(sys.argv) < 2:
        sys.exit("usage: make_air_vectors.py path/to/stark-stir-swarm [air ...]")
    src = os.path.join(sys.argv[1], "crates", "deep_ali", "src")
    only = set(sys.argv[2:])
    path = os.path.join(HERE, "air_vectors.json")

    def module(*files):
        return R.Interp(R.parse_sources([open(os.path.join(src, f)).read() for f in files]))

    out = {"source": "stark-stir-swarm/crates/deep_ali/src (evaluated by tests/golden/rust_subset.py)",
           "p": P, "airs": {}}
    if only:
        with open(path) as f:
            out = json.load(f)
    t0 = time.time()
    if not only or "ed25519" in only:
        out["airs"]["ed25519"] = ed25519_entry(src)
    if only:
        with open(path, "w") as f:
            json.dump(out, f, indent=1)
        print(f"wrote {path} in {time.time() - t0:.0f} s")
        return

    it = module("sha256_air.rs")
    w = it.const("WIDTH")
    cases = []
    for i, (row, nb) in enumerate(SHA256_CASES):
        seed = 256000 + i
        cur, nxt = rows_for(seed, w)
        cases.append(record([x.v for x in it.call("eval_sha256_constraints", fe_list(cur), fe_list(nxt), row, nb)],
                            row, seed, {"n_blocks": nb}))
    out["airs"]["sha256"] = {"width": w, "constraints": it.const("NUM_CONSTRAINTS"),
                             "evaluator": "sha256_air.rs:eval_sha256_constraints", "cases": cases}

    it = module("sha512_air.rs")
    w = it.const("WIDTH")
    cases = []
    for i, (row, nb) in enumerate(SHA512_CASES):
        seed = 512000 + i
        cur, nxt = rows_for(seed, w)
        cases.append(record([x.v for x in it.call("eval_sha512_constraints", fe_list(cur), fe_list(nxt), row, nb)],
                            row, seed, {"n_blocks": nb}))
    out["airs"]["sha512"] = {"width": w, "constraints": it.const("NUM_CONSTRAINTS"),
                             "evaluator": "sha512_air.rs:eval_sha512_constraints", "cases": cases}

    it = module("rsa2048_field_air.rs", "rsa2048_exp_air.rs", "rsa2048_stacked_air.rs")
    cases = []
    for i, (nrec, row) in enumerate(RSA_CASES):
        lay = it.call("build_rsa_stacked_layout", nrec)
        seed = 2048000 + i
        cur, nxt = rows_for(seed, lay.width)
        vals = it.call("eval_rsa_stacked_per_row", fe_list(cur), fe_list(nxt), row, 32, lay)
        cases.append(record([x.v for x in vals], row, seed, {"records": nrec, "n_trace": 32, "width": lay.width}))
    out["airs"]["rsa2048"] = {"width_per_record": it.call("build_rsa_stacked_layout", 1).width,
                              "evaluator": "rsa2048_stacked_air.rs:eval_rsa_stacked_per_row", "cases": cases}

    it = module("p256_field.rs", "p256_field_air.rs", "p256_group_air.rs", "p256_scalar_mul_air.rs",
                "p256_ecdsa_double_multirow_air.rs")
    lay, w = it.call("build_ecdsa_double_multirow_layout", 0)
    cases = []
    for i, (n_trace, row) in enumerate(P256_CASES):
        seed = 256256 + i
        cur, nxt = rows_for(seed, w)
        vals = it.call("eval_ecdsa_double_multirow_per_row", fe_list(cur), fe_list(nxt), row, n_trace, lay)
        cases.append(record([x.v for x in vals], row, seed, {"n_trace": n_trace}))
    out["airs"]["p256_ecdsa"] = {"width": w, "constraints": it.call("ecdsa_double_multirow_constraints", lay),
                                 "evaluator": "p256_ecdsa_double_multirow_air.rs:eval_ecdsa_double_multirow_per_row",
                                 "cases": cases}

    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {path} in {time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()

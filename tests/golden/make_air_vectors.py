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

The test tests/test_air_vectors.py regenerates the same rows and checks the
oracle's evaluators against these records; the reference is not read then.

Usage: python tests/golden/make_air_vectors.py path/to/stark-stir-swarm
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import rust_subset as R  # noqa: E402

P = R.P

# (air, evaluator inputs) cases; the rows cover every gating phase
SHA256_CASES = [(0, 1), (5, 1), (14, 1), (15, 1), (20, 1), (62, 1), (63, 1), (64, 1), (65, 1), (127, 1),
                (148, 2), (192, 2), (300, 2)]
SHA512_CASES = [(0, 1), (15, 1), (16, 1), (40, 1), (78, 1), (79, 1), (80, 1), (81, 1), (127, 1), (150, 2),
                (300, 2)]
RSA_CASES = [(1, 0), (1, 7), (1, 16), (1, 30), (1, 31), (2, 16), (2, 31)]
P256_CASES = [(256, 0), (256, 129), (256, 255), (8, 7)]


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


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_air_vectors.py path/to/stark-stir-swarm")
    src = os.path.join(sys.argv[1], "crates", "deep_ali", "src")

    def module(*files):
        return R.Interp(R.parse_sources([open(os.path.join(src, f)).read() for f in files]))

    out = {"source": "stark-stir-swarm/crates/deep_ali/src (evaluated by tests/golden/rust_subset.py)",
           "p": P, "airs": {}}
    t0 = time.time()

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

    path = os.path.join(HERE, "air_vectors.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {path} in {time.time() - t0:.0f} s")


if __name__ == "__main__":
    main()

"""The oracle's AIR constraint evaluators against the reference's own.

tests/golden/air_vectors.json holds, per AIR, the output of the reference's
Rust constraint evaluator (run by the subset interpreter in
tests/golden/rust_subset.py when the fixture was made) on rows of uniformly
random field elements, at rows covering every phase of the AIR's gating.
Here the same rows are drawn again from their seeds and fed to the oracle's
evaluators (the restatements the GPU kernels are checked against); the
vectors must be identical: same length, same digest of every value, same
λ-weighted sum with λ_j = j + 1. Random rows make every constraint non-zero,
so this pins the emission order, the cells each constraint reads and each
constraint's polynomial.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle_lib as O
import oracle_p256 as E
import oracle_rsa as ORSA

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = json.load(open(os.path.join(HERE, "golden", "air_vectors.json")))
P = O.P


def rows_for(seed, width):
    rng = np.random.default_rng(seed)
    return (rng.integers(0, P, width, dtype=np.uint64), rng.integers(0, P, width, dtype=np.uint64))


def check(vals, case):
    v = np.ascontiguousarray(vals, dtype=np.uint64)
    assert v.size == case["n"]
    assert [int(x) for x in v[:4]] == case["head"]
    assert sum((j + 1) * int(x) for j, x in enumerate(v)) % P == case["lambda_sum"]
    assert hashlib.sha3_256(v.tobytes()).hexdigest() == case["sha3_256"]


def _ids(air):
    return [f"{air}-{i}" for i in range(len(FIX["airs"][air]["cases"]))]


@pytest.mark.parametrize("case", FIX["airs"]["sha256"]["cases"], ids=_ids("sha256"))
def test_sha256_evaluator_matches_reference(case):
    a = FIX["airs"]["sha256"]
    assert (a["width"], a["constraints"]) == (O.SHA_WIDTH, O.SHA_K)
    cur, nxt = rows_for(case["seed"], a["width"])
    check(O.sha256_eval(cur, nxt, case["row"], case["n_blocks"]), case)


@pytest.mark.parametrize("case", FIX["airs"]["sha512"]["cases"], ids=_ids("sha512"))
def test_sha512_evaluator_matches_reference(case):
    a = FIX["airs"]["sha512"]
    cur, nxt = rows_for(case["seed"], a["width"])
    check(O.sha512_eval(cur, nxt, case["row"], case["n_blocks"]), case)


@pytest.mark.parametrize("case", FIX["airs"]["rsa2048"]["cases"], ids=_ids("rsa2048"))
def test_rsa2048_evaluator_matches_reference(case):
    assert FIX["airs"]["rsa2048"]["width_per_record"] == ORSA.WIDTH
    cur, nxt = rows_for(case["seed"], case["width"])
    check(ORSA.eval_row(cur, nxt, case["row"], case["records"], case["n_trace"]), case)


@pytest.mark.parametrize("case", FIX["airs"]["p256_ecdsa"]["cases"], ids=_ids("p256_ecdsa"))
def test_p256_ecdsa_evaluator_matches_reference(case):
    a = FIX["airs"]["p256_ecdsa"]
    lay = E.Layout()
    assert (lay.width, lay.n_constraints) == (a["width"], a["constraints"])
    cur, nxt = rows_for(case["seed"], a["width"])
    check(E.eval_row(lay, cur, nxt, case["row"], case["n_trace"]), case)


def test_fixture_shapes():
    # the fixture itself: one case per gating phase, digests of full-length vectors
    assert FIX["airs"]["sha256"]["constraints"] == 766 and FIX["airs"]["sha512"]["constraints"] == 1526
    assert FIX["airs"]["p256_ecdsa"]["constraints"] == 155774
    for a in FIX["airs"].values():
        assert len({c["sha3_256"] for c in a["cases"]}) == len(a["cases"])

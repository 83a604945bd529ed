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

import oracle_ed25519 as OE
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


_ED_PROGRAMS = {}


def _ed25519_program(li):
    """the oracle's layout and constraint program for the fixture's li-th signature"""
    if li not in _ED_PROGRAMS:
        L = FIX["airs"]["ed25519"]["layouts"][li]
        seed = hashlib.sha256(L["key_tag"].encode()).digest()
        msg = bytes.fromhex(L["msg_hex"])
        _, _, pub = OE.keypair(seed)
        sig = OE.sign(seed, msg)
        _ED_PROGRAMS[li] = OE.layout_program(pub, sig, msg, L["k_scalar"])[:2]
    return _ED_PROGRAMS[li]


@pytest.mark.parametrize("li", range(len(FIX["airs"]["ed25519"]["layouts"])))
def test_ed25519_layout_matches_reference(li):
    L = FIX["airs"]["ed25519"]["layouts"][li]
    lay, pr = _ed25519_program(li)
    assert (lay.width, lay.height, pr.n) == (L["width"], L["height"], L["constraints"])
    assert pr.n == OE.n_constraints(L["k_scalar"])
    rows = L["rows"]
    assert (lay.k_hash, lay.reduce_row, lay.decomp_R_row, lay.decomp_A_row) == (
        rows["k_hash"], rows["reduce_row"], rows["decompress_R_row"], rows["decompress_A_row"])
    assert (lay.sB_first, lay.kA_first, lay.residual_row, lay.result_row) == (
        rows["sB_first_row"], rows["kA_first_row"], rows["residual_row"], rows["result_row"])
    assert lay.dbl_rows == (rows["dbl_1_row"], rows["dbl_2_row"], rows["dbl_3_row"])


@pytest.mark.parametrize("case", FIX["airs"]["ed25519"]["cases"], ids=_ids("ed25519"))
def test_ed25519_evaluator_matches_reference(case):
    lay, pr = _ed25519_program(case["layout"])
    cur, nxt = rows_for(case["seed"], lay.width)
    check(OE.eval_row(pr, cur, nxt, case["row"]), case)


def test_fixture_shapes():
    # the fixture itself: one case per gating phase, digests of full-length vectors
    assert FIX["airs"]["sha256"]["constraints"] == 766 and FIX["airs"]["sha512"]["constraints"] == 1526
    assert FIX["airs"]["p256_ecdsa"]["constraints"] == 155774
    assert [L["constraints"] for L in FIX["airs"]["ed25519"]["layouts"]] == [68870, 70606, 68926]
    for a in FIX["airs"].values():
        assert len({c["sha3_256"] for c in a["cases"]}) == len(a["cases"])

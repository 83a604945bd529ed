"""The GPU constraint merges on random input, against the oracle.

The merge tests elsewhere feed honest (or lightly tampered) traces, on which
most constraints vanish. Here every LDE column is uniformly random, so every
constraint value at every point is a generic field element and Φ = Σ λ_j C_j
depends on each constraint's position and polynomial. The oracle's
evaluators are in turn checked against the reference's own Rust evaluators on
random rows (tests/test_air_vectors.py), which closes the chain
GPU = oracle = reference for the constraint systems. Exact equality of the
whole c_eval (Φ, the quotient by Z_H and its evaluation) is required.
"""
import numpy as np
import pytest

import oracle_lib as O
import oracle_p256 as E
import oracle_rsa as ORSA

pytestmark = pytest.mark.gpu
P = O.P


def rand_lde(seed, w, n):
    return np.random.default_rng(seed).integers(0, P, size=(w, n), dtype=np.uint64)


@pytest.mark.parametrize("n_trace,blowup,n_blocks", [(128, 4, 1), (256, 2, 2), (128, 32, 1)])
def test_sha256_merge_random_input(ctx, n_trace, blowup, n_blocks):
    lam = np.arange(1, O.SHA_K + 1, dtype=np.uint64)
    lde = rand_lde(n_trace + blowup, O.SHA_WIDTH, n_trace * blowup)
    want = O.merge_sha256(lde, n_trace, blowup, lam, n_blocks, O.PHI_ALWAYS)
    assert np.array_equal(ctx.merge_sha256(lde, n_trace, blowup, lam, n_blocks, O.PHI_ALWAYS), want)


@pytest.mark.parametrize("n_trace,blowup,n_blocks", [(128, 4, 1), (256, 2, 2)])
def test_sha512_merge_random_input(ctx, n_trace, blowup, n_blocks):
    lam = np.arange(1, 1527, dtype=np.uint64)
    lde = rand_lde(7 * n_trace + blowup, 1510, n_trace * blowup)
    want = O.merge_sha512(lde, n_trace, blowup, lam, n_blocks, O.PHI_ALWAYS)
    assert np.array_equal(ctx.merge_sha512(lde, n_trace, blowup, lam, n_blocks, O.PHI_ALWAYS), want)


@pytest.mark.parametrize("records,blowup", [(1, 4), (2, 4), (1, 32)])
def test_rsa2048_merge_random_input(ctx, records, blowup):
    lde = rand_lde(2048 + records * blowup, records * ORSA.WIDTH, 32 * blowup)
    want = ORSA.merge(lde, records, 32, blowup)
    assert np.array_equal(ctx.merge_rsa2048(lde, records, 32, blowup), want)


@pytest.mark.parametrize("n_trace,blowup", [(8, 4), (4, 32)])
def test_p256_merge_random_input(ctx, n_trace, blowup):
    lay = E.Layout()
    lde = rand_lde(256 + n_trace, lay.width, n_trace * blowup)
    want = E.merge(lay, lde, n_trace, blowup)
    assert np.array_equal(ctx.merge_p256_ecdsa(lde, n_trace, blowup), want)

"""NTT / LDE / Merkle on inputs built from the field's edge values, against the oracle.

Uniform random field elements almost never come near the carries and borrows the
device arithmetic takes care of: a 64-bit value above p - 2^32, a sum that wraps
2^64 exactly, a difference of equal values, a product whose high word is all ones.
Columns drawn from a small set of such values (0, 1, p - 1, p - 2, 2^32 - 1, 2^32,
2^63, p - 2^32, ...) and from runs of one value reach those cases in every pass
and every butterfly; bit-exact equality with the oracle is required.
"""
import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu
P = O.P

EDGE = np.array([0, 1, 2, P - 1, P - 2, P - 3, (1 << 32) - 1, 1 << 32, (1 << 32) + 1, 1 << 63, (1 << 63) - 1,
                 P - (1 << 32), P - (1 << 32) + 1, (1 << 64) - (1 << 33) + 1, 0xFFFFFFFE00000001, 0x00000000FFFFFFFE,
                 0x8000000000000001, 0x7FFFFFFF80000000],
                dtype=np.uint64)


def edge_cols(rng, cols, n):
    x = EDGE[rng.integers(0, EDGE.size, size=(cols, n))]
    # runs of one value (constant blocks make whole butterflies see equal inputs)
    if n >= 64:
        for c in range(cols):
            s = int(rng.integers(0, n - 32))
            x[c, s:s + 32] = EDGE[int(rng.integers(0, EDGE.size))]
    assert (x < np.uint64(P)).all()
    return x


@pytest.mark.parametrize("log_n", [1, 4, 7, 8, 10, 11, 12, 13, 16, 20])
@pytest.mark.parametrize("inverse", [False, True])
def test_ntt_edge_values_match_oracle(ctx, log_n, inverse):
    rng = np.random.default_rng(900 + log_n)
    cols = 2
    x = edge_cols(rng, cols, 1 << log_n)
    got = ctx.ntt(x, log_n, inverse)
    for c in range(cols):
        assert np.array_equal(got[c], O.ntt(x[c], inverse)), c


@pytest.mark.parametrize("w,log_n,blowup,shift", [(3, 10, 8, 7), (2, 14, 8, 7), (1, 16, 4, 3), (16, 12, 8, 7)])
def test_lde_edge_values_match_oracle(ctx, w, log_n, blowup, shift):
    rng = np.random.default_rng(w * 10 + log_n)
    tr = edge_cols(rng, w, 1 << log_n)
    assert np.array_equal(ctx.lde(tr, blowup, shift), O.lde(tr, blowup, shift))


def test_all_max_and_all_zero_columns(ctx):
    n = 1 << 12
    x = np.stack([np.full(n, P - 1, dtype=np.uint64), np.zeros(n, dtype=np.uint64),
                  np.full(n, (1 << 32), dtype=np.uint64)])
    for inverse in (False, True):
        got = ctx.ntt(x, 12, inverse)
        for c in range(3):
            assert np.array_equal(got[c], O.ntt(x[c], inverse))
    assert np.array_equal(ctx.lde(x, 8, 7), O.lde(x, 8, 7))


def test_lde_commit_edge_values_match_oracle(ctx):
    # the fused path (last pass hashes the rows) on the same kind of input
    rng = np.random.default_rng(77)
    w, log_n, blowup = 16, 12, 8
    tr = edge_cols(rng, w, 1 << log_n)
    lde = O.lde(tr, blowup, 7)
    arities = [16, 16, 16, 8]
    root = ctx.lde_commit(tr, blowup, 7, arities, 0)
    assert root == ctx.merkle_commit(lde, arities, 0)
    assert root == O.merkle_root(np.ascontiguousarray(lde.T), arities, 0)

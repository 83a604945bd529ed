"""The benchmarked workload itself, compared with the oracle at full size.

bench.py's step is: 64 columns x 2^20 rows (seed 3) -> coset LDE x8 (shift 7)
-> SHA3-256 Merkle root over the 2^23 LDE rows (arity 16 x 6, tree label 0)
-> STIR proof of LDE column 0 with build_params(2^23, bench pi hash). Every
output of that step is compared here byte for byte with the oracle on the
same inputs: all 64 LDE columns, the root, the proof. A uniformly random 2^23
column (not of low degree, unlike an LDE column) is proved too, and the full
2^23 forward and inverse NTTs are compared point by point. The oracle runs
multi-threaded on the host; these cases take tens of seconds.
"""
import numpy as np
import pytest

import bench
import oracle_lib as O

pytestmark = pytest.mark.gpu
P = O.P


@pytest.fixture(scope="module")
def step_inputs():
    trace = bench.make_trace(0)
    assert trace.shape == (bench.W, bench.N) == (64, 1 << 20)
    return trace


@pytest.mark.parametrize("inverse", [False, True])
def test_ntt_2p23_full_transform_matches_oracle(ctx, inverse):
    rng = np.random.default_rng(2300 + inverse)
    x = rng.integers(0, P, size=(1, 1 << 23), dtype=np.uint64)
    got = ctx.ntt(x, 23, inverse)
    assert np.array_equal(got[0], O.ntt(x[0], inverse))


def test_bench_step_lde_root_and_proof_match_oracle(sgpu, ctx, step_inputs):
    trace = step_inputs
    lde = ctx.lde(trace, bench.BLOWUP, bench.SHIFT)
    want = O.lde(trace, bench.BLOWUP, bench.SHIFT)
    for c in range(bench.W):
        assert np.array_equal(lde[c], want[c]), f"LDE column {c}"
    del want
    root = ctx.merkle_commit(lde, bench.ARITIES, bench.TREE_LABEL)
    rows = np.ascontiguousarray(lde.T)
    assert root == O.merkle_root(rows, bench.ARITIES, bench.TREE_LABEL)
    del rows
    # the fused pipeline the bench times: the LDE's last pass hashes the rows
    root_fused, col0 = ctx.lde_commit(trace, bench.BLOWUP, bench.SHIFT, bench.ARITIES, bench.TREE_LABEL, keep_cols=1)
    assert root_fused == root
    assert np.array_equal(col0[0], lde[0])
    n0 = bench.N0
    proof = ctx.deep_fri_prove(lde[0], n0, sgpu.build_params(n0, bench.PI_HASH))
    assert proof == O.stir_prove(lde[0], O.build_params(n0, bench.PI_HASH))
    assert sgpu.deep_fri_verify(sgpu.build_params(n0, bench.PI_HASH), proof)


def test_stir_proof_of_random_2p23_column_matches_oracle(sgpu, ctx):
    n0 = 1 << 23
    rng = np.random.default_rng(8023)
    f0 = rng.integers(0, P, size=n0, dtype=np.uint64)
    pi = rng.bytes(32)
    got = ctx.deep_fri_prove(f0, n0, sgpu.build_params(n0, pi))
    assert got == O.stir_prove(f0, O.build_params(n0, pi))

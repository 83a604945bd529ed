"""STIR proofs of one shape in lockstep (sg_stir_prove_group): every stage one
launch over all proofs, one host round trip per fold layer for all transcripts.
Each proof must equal, byte for byte, the same proof made alone (and the
oracle's)."""
import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu
P = O.P


@pytest.mark.parametrize("log_n0,G", [(3, 2), (6, 5), (9, 16), (13, 3), (17, 8), (14, 1)])
def test_group_stir_matches_single_proofs(sgpu, ctx, log_n0, G):
    n0 = 1 << log_n0
    rng = np.random.default_rng(400 + log_n0 * 10 + G)
    f0s = rng.integers(0, P, size=(G, n0), dtype=np.uint64)
    pis = [rng.bytes(32) for _ in range(G)]
    ps = [sgpu.build_params(n0, pi) for pi in pis]
    got = ctx.deep_fri_prove_group(f0s, ps)
    alone = [ctx.deep_fri_prove(f0s[g], n0, ps[g]) for g in range(G)]
    assert got == alone
    g = G - 1
    assert got[g] == O.stir_prove(f0s[g], O.build_params(n0, pis[g]))


@pytest.mark.parametrize("sched,cc", [([4, 2, 8], True), ([2, 2, 2, 2], False), ([16, 4], True), ([8], False)])
def test_group_stir_other_schedules(sgpu, ctx, sched, cc):
    n0 = 4
    for m in sched:
        n0 *= m
    rng = np.random.default_rng(n0 + len(sched))
    G = 4
    f0s = rng.integers(0, P, size=(G, n0), dtype=np.uint64)
    ps = [sgpu.FriParams.new(sched, coeff_commit_final=cc, public_inputs_hash=rng.bytes(32)) for _ in range(G)]
    assert ctx.deep_fri_prove_group(f0s, ps) == [ctx.deep_fri_prove(f0s[g], n0, ps[g]) for g in range(G)]


def test_group_stir_device_input_and_low_degree_accepted(sgpu, ctx):
    torch = pytest.importorskip("torch")
    n0, G = 1 << 12, 6
    rng = np.random.default_rng(12)
    coeffs = np.zeros((G, n0), dtype=np.uint64)
    coeffs[:, :64] = rng.integers(0, P, size=(G, 64), dtype=np.uint64)
    f0s = np.stack([O.ntt(coeffs[g]) for g in range(G)])
    ps = [sgpu.build_params(n0, rng.bytes(32)) for _ in range(G)]
    d = torch.from_numpy(f0s.view(np.int64)).cuda()
    got = ctx.deep_fri_prove_group(d, ps)
    assert got == ctx.deep_fri_prove_group(f0s, ps)
    assert all(sgpu.deep_fri_verify(ps[g], got[g]) for g in range(G))


def test_group_stir_refuses_mixed_shapes(sgpu, ctx):
    n0 = 1 << 9
    f0s = np.zeros((2, n0), dtype=np.uint64)
    ps = [sgpu.build_params(n0, bytes(32)), sgpu.FriParams.new([8, 8, 2, 2, 2], public_inputs_hash=bytes(32))]
    with pytest.raises(sgpu.StarkGpuError):
        ctx.deep_fri_prove_group(f0s, ps)

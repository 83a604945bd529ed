"""SHA-512 AIR on the GPU vs the oracle (bit-exact): the device trace expansion
against the oracle's fill_block trace, deep_ali_merge_sha512 for 1..3-block
messages in every Phi mode, the coset-sliced merge against the materialised one,
and full proofs byte for byte, accepted by the oracle's verifier."""
import hashlib

import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu

LAM = np.arange(1, 1527, dtype=np.uint64)


@pytest.mark.parametrize("msg", [b"", b"abc", b"b" * 112, bytes(range(256)) + b"q" * 60, b"m" * 700])
def test_device_trace_expansion_matches_oracle(sgpu, ctx, msg):
    want, wnb = O.sha512_trace(msg)
    got, nb, dg = ctx.sha512_trace(msg)
    assert nb == wnb and got.shape == want.shape
    assert np.array_equal(got, want)
    assert dg == hashlib.sha512(msg).digest()


@pytest.mark.parametrize("msg,mode", [(b"abc", O.PHI_PARALLEL_GATE), (b"b" * 112, O.PHI_PARALLEL_GATE),
                                      (bytes(range(200)), O.PHI_ALWAYS), (b"d" * 300, O.PHI_PARALLEL_GATE),
                                      (b"abc", O.PHI_NEVER)])
def test_merge_sha512_matches_oracle(sgpu, ctx, msg, mode):
    tr, nb, _ = sgpu.build_sha512_trace_multi(msg)
    n_trace = tr.shape[1]
    lde = O.lde(tr, 32)
    want = O.merge_sha512(lde, n_trace, 32, LAM, nb, mode)
    got = ctx.merge_sha512(lde, n_trace, 32, LAM, nb, mode)
    assert np.array_equal(got, want)


def test_merge_sha512_random_lambdas(sgpu, ctx):
    rng = np.random.default_rng(512)
    lam = rng.integers(0, O.P, 1526, dtype=np.uint64)
    tr, nb, _ = sgpu.build_sha512_trace_multi(b"lambda")
    lde = O.lde(tr, 32)
    assert np.array_equal(ctx.merge_sha512(lde, tr.shape[1], 32, lam, nb, O.PHI_ALWAYS),
                          O.merge_sha512(lde, tr.shape[1], 32, lam, nb, O.PHI_ALWAYS))


@pytest.mark.parametrize("msg", [b"abc", bytes(range(130))])
def test_prove_sha512_matches_oracle(sgpu, ctx, msg):
    fsb = hashlib.sha3_256(b"fs512" + msg).digest()
    proof, digest = ctx.prove_sha512(msg, fsb)
    want, wdigest = O.prove_sha512(msg, fsb)
    assert digest == wdigest == hashlib.sha512(msg).digest()
    assert proof == want
    assert O.stir_verify(proof, O.build_params(len(O.sha512_trace(msg)[0][0]) * 32, fsb))


def test_coset_sliced_merge_matches_materialised(sgpu, ctx):
    msg = b"cosets" * 50
    fsb = hashlib.sha3_256(b"c512").digest()
    want = O.prove_sha512(msg, fsb)
    try:
        ctx.set_option(sgpu.OPT_WIDE_MERGE, sgpu.WIDE_MERGE_COSETS)
        got = ctx.prove_sha512(msg, fsb)
    finally:
        ctx.set_option(sgpu.OPT_WIDE_MERGE, sgpu.WIDE_MERGE_AUTO)
    assert got == want

"""SHA-256 AIR on the GPU vs the oracle (bit-exact): deep_ali_merge_sha256 for
1..5-block messages in every Phi mode, the AIR-registry merge (n_blocks = 1),
and full prove_ds_ksk_binding proofs byte for byte, accepted by both verifiers."""
import hashlib

import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu

LAM = np.arange(1, 767, dtype=np.uint64)


@pytest.mark.parametrize("msg,mode", [(b"abc", O.PHI_PARALLEL_GATE), (bytes(range(64)), O.PHI_PARALLEL_GATE),
                                      (b"c" * 120, O.PHI_ALWAYS), (bytes(range(250)), O.PHI_PARALLEL_GATE),
                                      (b"abc", O.PHI_NEVER)])
def test_merge_sha256_matches_oracle(sgpu, ctx, msg, mode):
    tr, nb, _ = sgpu.build_sha256_trace_multi(msg)
    n_trace = tr.shape[1]
    lde = O.lde(tr, 32)
    want = O.merge_sha256(lde, n_trace, 32, LAM, nb, mode)
    got = ctx.merge_sha256(lde, n_trace, 32, LAM, nb, mode)
    assert np.array_equal(got, want)


def test_merge_registry_sha256_matches_oracle(ctx):
    # AirType::Sha256DsKsk through the generic merge: n_blocks fixed to 1
    tr, _ = O.sha256_trace(b"registry")
    lde = O.lde(tr, 32)
    rng = np.random.default_rng(5)
    lam = rng.integers(0, O.P, 766, dtype=np.uint64)
    want = O.merge(O.AIR_SHA256, lde, tr.shape[1], 32, lam, O.PHI_ALWAYS)
    got = ctx.merge(6, lde, tr.shape[1], 32, lam, O.PHI_ALWAYS)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("msg", [b"abc", bytes(range(64)), b"dnskey" * 40])
def test_prove_sha256_matches_oracle(sgpu, ctx, msg):
    fsb = hashlib.sha3_256(b"fs-binding" + msg).digest()
    proof, digest = ctx.prove_sha256(msg, fsb)
    want, wdigest = O.prove_sha256(msg, fsb)
    assert digest == wdigest == hashlib.sha256(msg).digest()
    assert proof == want
    tr, nb, _ = sgpu.build_sha256_trace_multi(msg)
    n0 = tr.shape[1] * 32
    assert sgpu.deep_fri_verify(sgpu.build_params(n0, fsb), proof)
    assert O.stir_verify(proof, O.build_params(n0, fsb))


@pytest.mark.parametrize("msg", [b"abc", bytes(range(200)), b"w" * 2000])
def test_coset_sliced_merge_matches_materialised(sgpu, ctx, msg):
    fsb = hashlib.sha3_256(b"coset" + msg).digest()
    want, wd = O.prove_sha256(msg, fsb)
    try:
        ctx.set_option(sgpu.OPT_WIDE_MERGE, sgpu.WIDE_MERGE_COSETS)
        got, gd = ctx.prove_sha256(msg, fsb)
    finally:
        ctx.set_option(sgpu.OPT_WIDE_MERGE, sgpu.WIDE_MERGE_AUTO)
    assert got == want and gd == wd


def test_large_sha256_trace_proof(sgpu, ctx):
    # 2^14-row trace (128 blocks): n0 = 2^19, taken by the coset path; digest and
    # self-verification (inside the call) and acceptance by the oracle verifier
    msg = bytes(np.random.default_rng(14).integers(0, 256, 128 * 64 - 9, dtype=np.uint8))
    fsb = hashlib.sha3_256(b"large").digest()
    ctx.set_option(sgpu.OPT_WIDE_MERGE, sgpu.WIDE_MERGE_COSETS)
    try:
        proof, digest = ctx.prove_sha256(msg, fsb)
    finally:
        ctx.set_option(sgpu.OPT_WIDE_MERGE, sgpu.WIDE_MERGE_AUTO)
    assert digest == hashlib.sha256(msg).digest()
    assert O.stir_verify(proof, O.build_params(1 << 19, fsb))


@pytest.mark.parametrize("msg", [b"", b"abc", bytes(range(64)), bytes(range(256)) * 3, b"p" * 1000])
def test_device_trace_expansion_matches_oracle(sgpu, ctx, msg):
    # host compressions + device column expansion == the oracle's fill_block trace,
    # padding rows included
    want, wnb = O.sha256_trace(msg)
    got, nb, dg = ctx.sha256_trace(msg)
    assert nb == wnb and got.shape == want.shape
    assert np.array_equal(got, want)
    assert dg == hashlib.sha256(msg).digest()


def test_device_trace_expansion_into_device_buffer(sgpu, ctx):
    torch = pytest.importorskip("torch")
    msg = bytes(np.random.default_rng(9).integers(0, 256, 700, dtype=np.uint8))
    want, _ = O.sha256_trace(msg)
    d = torch.empty(want.size, dtype=torch.int64, device="cuda")
    ctx.sha256_trace(msg, out=d)
    torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy().view(np.uint64).reshape(want.shape), want)

"""P-256 ECDSA double-chain AIR on the GPU vs the oracle (bit-exact): the device
trace expansion, the gadget-interpreter merge (Phi at every LDE point, then the
quotient) on honest and tampered traces, and whole chain proofs byte for byte.
The full-size ECDSA proof (K = 256 rows, n0 = 8192) is checked through its
chain outputs: R = A + B - 2^256 (G + Q) must have x(R) = r mod n."""
import hashlib
import random

import numpy as np
import pytest

import oracle_lib as O
import oracle_p256 as E

pytestmark = pytest.mark.gpu

Q2 = E._affine_add(E.G, E.G)


def _bits(seed, k):
    rng = random.Random(seed)
    return [rng.randrange(2) for _ in range(k)], [rng.randrange(2) for _ in range(k)]


def test_device_trace_matches_oracle(sgpu, ctx):
    a, b = _bits(3, 8)
    d, q = E.keypair(0x1357)
    want, _ = E.trace(E.G, a, q, b)
    assert np.array_equal(ctx.p256_chain_trace(E.G, a, q, b), want)


@pytest.mark.parametrize("k", [4, 8])
def test_merge_matches_oracle(sgpu, ctx, k):
    a, b = _bits(k, k)
    tr, lay = E.trace(E.G, a, Q2, b)
    lde = O.lde(tr, E.BLOWUP)
    assert np.array_equal(ctx.merge_p256_ecdsa(lde, k), E.merge(lay, lde, k))


def test_merge_of_tampered_trace_matches_oracle(sgpu, ctx):
    a, b = _bits(11, 4)
    tr, lay = E.trace(E.G, a, Q2, b)
    rng = np.random.default_rng(5)
    for c in rng.integers(0, lay.width, 40):
        tr[c, int(rng.integers(0, 4))] ^= 1
    lde = O.lde(tr, E.BLOWUP)
    assert np.array_equal(ctx.merge_p256_ecdsa(lde, 4), E.merge(lay, lde, 4))


def test_chain_proof_matches_oracle(sgpu, ctx):
    a, b = _bits(21, 8)
    d, q = E.keypair(0x2468)
    pi = hashlib.sha3_256(b"p256 chains").digest()
    tr, lay = E.trace(E.G, a, q, b)
    got = ctx.prove_p256_chains(E.G, a, q, b, pi)
    assert got == E.prove(lay, tr, pi)
    assert O.stir_verify(got, O.build_params(8 * E.BLOWUP, pi))


def test_full_ecdsa_proof(sgpu, ctx):
    d, q = E.keypair(0xDEC0DE)
    digest = hashlib.sha256(b"DNSSEC-RRSIG-V0|google.com.|A|142.251.46.142|epoch-0").digest()
    r, s = E.sign(digest, d, 0x0BADC0FFEE)
    pi = sgpu.p256_ecdsa_pi(q[0], q[1], r, s, digest)
    proof = ctx.prove_p256_ecdsa(q, r, s, digest, pi)
    assert O.stir_verify(proof, O.build_params(256 * E.BLOWUP, pi))
    assert sgpu.deep_fri_verify(sgpu.build_params(256 * E.BLOWUP, pi), proof)
    # the trace's chain outputs finish the verification natively
    u1, u2 = sgpu.p256_u_bits(digest, r, s)
    tr = ctx.p256_chain_trace(E.G, u1, q, u2)
    lay = E.Layout()
    out = [sum(int(tr[lay.r_proj[j] + i, 0]) << (26 * i) for i in range(10)) for j in range(6)]
    ra = (out[0] * pow(out[2], -1, E.P) % E.P, out[1] * pow(out[2], -1, E.P) % E.P)
    rb = (out[3] * pow(out[5], -1, E.P) % E.P, out[4] * pow(out[5], -1, E.P) % E.P)
    shift = E.scalar_mul(1 << 256, E._affine_add(E.G, q))
    R = E._affine_add(E._affine_add(ra, rb), (shift[0], (-shift[1]) % E.P))
    assert R[0] % E.N == r


def test_full_ecdsa_proof_matches_oracle_bytes(sgpu, ctx):
    # the full-size record proof (K = 256 rows, n0 = 8192, a 9.9 GB LDE in the
    # oracle) byte for byte against the oracle fed the Python-integer trace; the
    # proof commits to every value of the merge output (c_eval), so equal bytes
    # also pin the merge at full size
    d, q = E.keypair(0xFACADE)
    digest = hashlib.sha256(b"DNSSEC-RRSIG-V0|example.org.|A|93.184.216.34|epoch-1").digest()
    r, s = E.sign(digest, d, 0x5EED)
    pi = sgpu.p256_ecdsa_pi(q[0], q[1], r, s, digest)
    u1, u2 = sgpu.p256_u_bits(digest, r, s)
    assert (u1, u2) == E.u_bits(digest, r, s)
    tr, lay = E.trace(E.G, u1, q, u2)
    assert np.array_equal(ctx.p256_chain_trace(E.G, u1, q, u2), tr)
    want = E.prove(lay, tr, pi)
    assert ctx.prove_p256_ecdsa(q, r, s, digest, pi) == want
    assert ctx.prove_p256_chains(E.G, u1, q, u2, pi) == want


def test_coset_streamed_merge_matches_materialised(sgpu, ctx):
    # SG_WIDE_MERGE_COSETS never stores the LDE (one coset at a time); its proofs
    # equal the materialised merge's and the oracle's, for K = 8 chains at blowup
    # 32 and for a full K = 256 signature check at blowup 4
    a, b = _bits(48, 8)
    d, q = E.keypair(0x7777)
    pi = hashlib.sha3_256(b"coset p256").digest()
    tr, lay = E.trace(E.G, a, q, b)
    want_chain = E.prove(lay, tr, pi)
    d2, q2 = E.keypair(0x8888)
    digest = hashlib.sha256(b"coset ecdsa").digest()
    r, s_ = E.sign(digest, d2, 0x99)
    pi2 = sgpu.p256_ecdsa_pi(q2[0], q2[1], r, s_, digest)
    u1, u2 = E.u_bits(digest, r, s_)
    tr2, _ = E.trace(E.G, u1, q2, u2)
    want_sig = E.prove(lay, tr2, pi2, blowup=4)
    try:
        for mode in (sgpu.WIDE_MERGE_COSETS, sgpu.WIDE_MERGE_LDE):
            ctx.set_option(sgpu.OPT_WIDE_MERGE, mode)
            assert ctx.prove_p256_chains(E.G, a, q, b, pi) == want_chain, mode
            (got, res), = ctx.prove_batch([(sgpu.JOB_P256_ECDSA, (q2, r, s_, digest), pi2, 0, 4)], n_streams=1)
            assert res.status == 0 and got == want_sig, mode
    finally:
        ctx.set_option(sgpu.OPT_WIDE_MERGE, sgpu.WIDE_MERGE_AUTO)

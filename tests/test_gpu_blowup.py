"""Proofs at LDE blowup 4 (the batched record-check workload's setting) against
the oracle, byte for byte, through the batch API's per-job blowup.

Blowup changes n0 = n_trace * blowup, hence the LDE, the Phi gate of the hash
AIRs (Phi = 0 below n0 = 4096 in the reference's parallel build), the
quotient, the STIR schedule make_schedule(n0) and every transcript value.
"""
import hashlib

import numpy as np
import pytest

import oracle_lib as O
import oracle_p256 as E
import oracle_rsa as ORSA

pytestmark = pytest.mark.gpu


def _one(ctx, job):
    (proof, res), = ctx.prove_batch([job], n_streams=1)
    assert res.status == 0
    return proof, res


@pytest.mark.parametrize("length", [40, 300, 600])
def test_sha256_record_proof_at_blowup_4(sgpu, ctx, length):
    # 1, 5 and 10 blocks: n0 = 512 (Phi gated to zero), 4096 and 8192 (Phi live)
    msg = np.random.default_rng(length).integers(0, 256, length, dtype=np.uint8).tobytes()
    fsb = hashlib.sha3_256(b"b4" + msg).digest()
    proof, res = _one(ctx, (sgpu.JOB_SHA256, msg, fsb, 0, 4))
    want, dg = O.prove_sha256(msg, fsb, O.PHI_PARALLEL_GATE, 4)
    assert proof == want
    assert bytes(res.digest[:32]) == dg == hashlib.sha256(msg).digest()
    n_trace = 128
    while n_trace < 128 * ((length + 9 + 63) // 64):
        n_trace *= 2
    assert sgpu.deep_fri_verify(sgpu.build_params(4 * n_trace, fsb), proof)


def test_sha512_record_proof_at_blowup_4(sgpu, ctx):
    msg = bytes(range(200))
    fsb = hashlib.sha3_256(b"b4-512").digest()
    proof, res = _one(ctx, (sgpu.JOB_SHA512, msg, fsb, 0, 4))
    assert proof == O.prove_sha512(msg, fsb, O.PHI_PARALLEL_GATE, 4)[0]


def test_rsa2048_proof_at_blowup_4(sgpu, ctx):
    keys = ORSA.keys()
    rec = ORSA.record(b"DNSSEC-RRSIG-V0|b4.example.|A|10.0.0.4", keys[0])[0]
    pi = hashlib.sha3_256(b"rsa b4").digest()
    proof, _ = _one(ctx, (sgpu.JOB_RSA2048, [rec], pi, 0, 4))
    assert proof == ORSA.prove(ORSA.trace([rec]), pi, blowup=4)
    assert sgpu.deep_fri_verify(sgpu.build_params(32 * 4, pi), proof)


def test_ecdsa_proof_at_blowup_4(sgpu, ctx):
    d, q = E.keypair(0xB10)
    digest = hashlib.sha256(b"DNSSEC-RRSIG-V0|b4.example.|A|10.0.0.4|alg-13").digest()
    r, s = E.sign(digest, d, 0x44)
    pi = sgpu.p256_ecdsa_pi(q[0], q[1], r, s, digest)
    proof, _ = _one(ctx, (sgpu.JOB_P256_ECDSA, (q, r, s, digest), pi, 0, 4))
    u1, u2 = E.u_bits(digest, r, s)
    tr, lay = E.trace(E.G, u1, q, u2)
    assert proof == E.prove(lay, tr, pi, blowup=4)
    assert sgpu.deep_fri_verify(sgpu.build_params(256 * 4, pi), proof)


def test_blowup_mix_batched_equals_alone(sgpu, ctx):
    # jobs of different blowups side by side: each proof equals the same job alone
    keys = ORSA.keys()
    jobs = []
    for i in range(6):
        msg = bytes([i]) * (50 + 90 * i)
        jobs.append((sgpu.JOB_SHA256, msg, hashlib.sha3_256(msg).digest(), 0, [4, 8, 32][i % 3]))
        rec = ORSA.record(msg, keys[i % len(keys)])[0]
        jobs.append((sgpu.JOB_RSA2048, [rec], hashlib.sha3_256(b"r" + msg).digest(), 0, [4, 16][i % 2]))
    alone = [_one(ctx, j)[0] for j in jobs]
    batched = ctx.prove_batch(jobs, n_streams=8)
    assert [p for p, _ in batched] == alone


def test_bad_blowup_is_refused(sgpu, ctx):
    for bad in (3, 1, 2048):
        with pytest.raises(sgpu.StarkGpuError) as ei:
            ctx.prove_batch([(sgpu.JOB_SHA256, b"abc", bytes(32), 0, bad)], n_streams=1)
        assert ei.value.code == sgpu.SG_EINVAL

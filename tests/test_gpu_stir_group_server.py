"""The serving loop with lockstep STIR groups (SG_OPT_STIR_GROUP): a worker takes
queued jobs whose proofs share n0 and proves their STIR phases together. Every
proof must equal the same job proved alone, failures stay with their own job."""
import hashlib

import numpy as np
import pytest

import oracle_p256 as E
import oracle_rsa as ORSA

pytestmark = pytest.mark.gpu


def _mix(sg):
    keys = ORSA.keys()
    jobs = []
    for i in range(18):
        msg = np.random.default_rng(i).integers(0, 256, 40 + 37 * i, dtype=np.uint8).tobytes()
        bu = 4 if i % 3 else 32
        jobs.append((sg.JOB_SHA256, msg, hashlib.sha3_256(b"g%d" % i).digest(), 0, bu))
        if i % 2:
            rec = ORSA.record(msg, keys[i % len(keys)])[0]
            jobs.append((sg.JOB_RSA2048, [rec], hashlib.sha3_256(b"r%d" % i).digest(), 0, bu))
    for i in range(3):
        d, q = E.keypair(0x600 + i)
        dg = hashlib.sha256(b"grouped ecdsa %d" % i).digest()
        r, s_ = E.sign(dg, d, 0x77 + i)
        jobs.append((sg.JOB_P256_ECDSA, (q, r, s_, dg), sg.p256_ecdsa_pi(q[0], q[1], r, s_, dg), 0, 4))
    jobs.append((sg.JOB_SHA512, b"x" * 300, hashlib.sha3_256(b"s512").digest(), 0, 4))
    return jobs


def test_grouped_batch_equals_jobs_alone(sgpu, ctx):
    jobs = _mix(sgpu)
    alone = [p for p, _ in ctx.prove_batch(jobs, n_streams=1)]
    try:
        for group, streams in ((8, 4), (64, 2), (3, 8)):
            ctx.set_option(sgpu.OPT_STIR_GROUP, group)
            got = ctx.prove_batch(jobs, n_streams=streams, hbm_budget_bytes=32 << 30)
            assert all(r.status == 0 for _, r in got)
            assert [p for p, _ in got] == alone, (group, streams)
    finally:
        ctx.set_option(sgpu.OPT_STIR_GROUP, 1)


def test_grouped_server_failures_stay_with_their_job(sgpu, ctx):
    jobs = [(sgpu.JOB_SHA256, bytes([i]) * 64, hashlib.sha3_256(b"f%d" % i).digest(), 0, 4) for i in range(10)]
    alone = [p for p, _ in ctx.prove_batch(jobs, n_streams=1)]
    try:
        ctx.set_option(sgpu.OPT_STIR_GROUP, 16)
        with sgpu.Server(ctx, n_streams=1) as srv:
            srv.set_retries(1)
            flags = [0] * 10
            flags[2] = sgpu.JOB_FAULT_VERIFY
            flags[5] = sgpu.JOB_FAULT_ALLOC
            t = [srv.submit(*(j + (flags[i],))) for i, j in enumerate(jobs)]
            for i, x in enumerate(t):
                if i == 2:
                    with pytest.raises(sgpu.StarkGpuError) as ei:
                        srv.wait(x)
                    assert ei.value.code == sgpu.SG_EVERIFY
                else:
                    assert srv.wait(x)[0] == alone[i]
    finally:
        ctx.set_option(sgpu.OPT_STIR_GROUP, 1)
    with pytest.raises(sgpu.StarkGpuError):
        ctx.set_option(sgpu.OPT_STIR_GROUP, 0)

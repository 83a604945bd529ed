"""Failure handling of the serving loop, with faults made on the host only.

The reference's controller gives each shard a deadline, reopens failed shards
and has workers self-verify (swarm-ctrl/src/main.rs:94-99, 1085;
swarm-dns/src/prover.rs:189-192). Here: a wait with a time limit, cancelling
queued and running jobs, re-running a job whose attempt failed with a
transient error, a job whose proof fails self-verification, and a job larger
than the HBM budget admitted only once the others are done. Every fault is
raised by the host (SG_JOB_FAULT_* flags raise the error where the named call
would have failed); no kernel is made to fault, trap or wait.
"""
import hashlib

import pytest

pytestmark = pytest.mark.gpu


def _sha_job(sg, i, flags=0, length=64):
    msg = bytes([i % 256]) * length
    return (sg.JOB_SHA256, msg, hashlib.sha3_256(b"fault-%d" % i).digest(), 0, 0, flags)


def test_wait_with_time_limit(sgpu, ctx):
    with sgpu.Server(ctx, n_streams=1) as srv:
        big = srv.submit(*_sha_job(sgpu, 1, length=20000)[:3])
        with pytest.raises(sgpu.StarkGpuError) as ei:
            srv.wait(big, timeout_ms=0)
        assert ei.value.code == sgpu.SG_ETIMEDOUT
        proof, res = srv.wait(big, timeout_ms=600000)  # the ticket is still valid
        assert res.status == 0 and proof


def test_cancel_queued_and_running(sgpu, ctx):
    alone = ctx.prove_batch([_sha_job(sgpu, 3)], n_streams=1)[0][0]
    with sgpu.Server(ctx, n_streams=1) as srv:
        first = srv.submit(*_sha_job(sgpu, 2, length=20000)[:3])
        queued = srv.submit(*_sha_job(sgpu, 3)[:3])
        last = srv.submit(*_sha_job(sgpu, 4)[:3])
        assert srv.cancel(queued) == 0
        with pytest.raises(sgpu.StarkGpuError) as ei:
            srv.wait(queued)
        assert ei.value.code == sgpu.SG_ECANCELED
        assert srv.wait(first)[1].status == 0
        assert srv.wait(last)[1].status == 0
        # a running job (the only one, on an idle worker): its result is discarded
        run = srv.submit(*_sha_job(sgpu, 5, length=20000)[:3])
        assert srv.cancel(run) in (0, 1)
        with pytest.raises(sgpu.StarkGpuError) as ei:
            srv.wait(run)
        assert ei.value.code == sgpu.SG_ECANCELED
        # the server keeps serving: the cancelled job's slot and memory are free again
        again = srv.submit(*_sha_job(sgpu, 3)[:3])
        assert srv.wait(again)[0] == alone
        with pytest.raises(sgpu.StarkGpuError):
            srv.cancel(987654321)


def test_transient_failure_is_retried(sgpu, ctx):
    jobs = [_sha_job(sgpu, i) for i in range(6)]
    alone = [p for p, _ in ctx.prove_batch(jobs, n_streams=1)]
    with sgpu.Server(ctx, n_streams=4) as srv:
        srv.set_retries(1)
        t = [srv.submit(*(j[:3] + (0, 0, sgpu.JOB_FAULT_ALLOC if i % 2 else 0))) for i, j in enumerate(jobs)]
        got = [srv.wait(x) for x in t]
    assert [p for p, _ in got] == alone
    # without retries the failure is reported and the other jobs still complete
    with sgpu.Server(ctx, n_streams=4) as srv:
        t = [srv.submit(*(j[:3] + (0, 0, sgpu.JOB_FAULT_ALLOC if i == 2 else 0))) for i, j in enumerate(jobs)]
        for i, x in enumerate(t):
            if i == 2:
                with pytest.raises(sgpu.StarkGpuError) as ei:
                    srv.wait(x)
                assert ei.value.code == sgpu.SG_ENOMEM
            else:
                assert srv.wait(x)[0] == alone[i]


def test_proof_failing_self_verification_is_reported(sgpu, ctx):
    jobs = [_sha_job(sgpu, 10 + i) for i in range(8)]
    jobs[3] = jobs[3][:5] + (sgpu.JOB_FAULT_VERIFY,)
    with pytest.raises(sgpu.StarkGpuError) as ei:
        ctx.prove_batch(jobs, n_streams=4)
    assert ei.value.code == sgpu.SG_EVERIFY
    with sgpu.Server(ctx, n_streams=4) as srv:
        srv.set_retries(3)  # a failed self-verification is deterministic: never retried
        t = [srv.submit(*j) for j in jobs]
        for i, x in enumerate(t):
            if i == 3:
                with pytest.raises(sgpu.StarkGpuError) as ei:
                    srv.wait(x)
                assert ei.value.code == sgpu.SG_EVERIFY
            else:
                proof, res = srv.wait(x)
                assert res.status == 0
                assert proof == ctx.prove_batch([jobs[i]], n_streams=1)[0][0]


def test_job_over_budget_runs_alone(sgpu, ctx):
    # budget below the large job's footprint: it is admitted only when nothing else runs
    small = [_sha_job(sgpu, 20 + i) for i in range(6)]
    big = _sha_job(sgpu, 30, length=8000)
    jobs = small[:3] + [big] + small[3:]
    res = ctx.prove_batch(jobs, n_streams=4, hbm_budget_bytes=2 << 30)
    spans = [(r.queue_ms, r.latency_ms) for _, r in res]
    b0, b1 = spans[3]
    for i, (s0, s1) in enumerate(spans):
        if i != 3:
            assert s1 <= b0 + 0.5 or s0 >= b1 - 0.5, (i, spans[i], spans[3])
    assert all(r.status == 0 for _, r in res)

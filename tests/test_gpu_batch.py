"""Batched and served proving: every proof made in a mix of concurrent jobs
(SHA-256, SHA-512, HashRollup and RSA-2048 signature checks) is
byte-identical to the same job proved alone (oracle), under several stream
counts and an HBM budget tight enough to serialise admission; the server
accepts submissions while earlier jobs are running. ECDSA-P256 jobs, whose
full-size proof is beyond the oracle's reach, match the same job proved alone
on the GPU (that path is pinned to the oracle at smaller chain lengths)."""
import hashlib
import time

import numpy as np
import pytest

import oracle_lib as O
import oracle_p256 as E
import oracle_rsa as R

pytestmark = pytest.mark.gpu


def _mix(n, seed):
    rng = np.random.default_rng(seed)
    jobs, want = [], []
    keys = R.keys()
    for i in range(n):
        pi = hashlib.sha3_256(b"job%d" % i).digest()
        if i % 5 == 4:
            k = 1 + i % 2
            recs = [R.record(b"job%d rec%d" % (i, r), keys[(i + r) % 4])[0] for r in range(k)]
            jobs.append((4, recs, pi))
            want.append((R.prove(R.trace(recs), pi), None))
        elif i % 4 == 2:
            leaves = rng.integers(0, O.P, int(rng.integers(1, 3000)), dtype=np.uint64)
            jobs.append((2, leaves, pi))
            want.append((O.prove_hash_rollup(leaves, pi), None))
        elif i % 4 == 3:
            msg = rng.integers(0, 256, int(rng.integers(1, 240)), dtype=np.uint8).tobytes()
            jobs.append((3, msg, pi))
            want.append(O.prove_sha512(msg, pi))
        else:
            ln = int(np.clip(rng.lognormal(np.log(120), 0.6), 40, 600))
            msg = rng.integers(0, 256, ln, dtype=np.uint8).tobytes()
            jobs.append((1, msg, pi))
            proof, dg = O.prove_sha256(msg, pi)
            want.append((proof, dg))
    return jobs, want


@pytest.mark.parametrize("streams,budget", [(1, 0), (4, 0), (16, 0), (8, 64 << 20)])
def test_batch_matches_single_proofs(ctx, streams, budget):
    jobs, want = _mix(12, streams)
    out = ctx.prove_batch(jobs, n_streams=streams, hbm_budget_bytes=budget)
    for (proof, res), (wproof, wdg) in zip(out, want):
        assert res.status == 0
        assert proof == wproof
        if wdg is not None:
            assert bytes(res.digest)[:len(wdg)] == wdg
        assert res.latency_ms >= res.run_ms >= 0


def test_server_admits_while_running(sgpu, ctx):
    jobs, want = _mix(10, 99)
    with sgpu.Server(ctx, n_streams=4) as srv:
        tickets = [srv.submit(*jobs[i]) for i in range(5)]
        first, _ = srv.wait(tickets[0])
        assert first == want[0][0]
        time.sleep(0.01)
        tickets += [srv.submit(*jobs[i]) for i in range(5, 10)]  # arrive while others are on the GPU
        for i, t in enumerate(tickets[1:], start=1):
            proof, res = srv.wait(t)
            assert res.status == 0 and proof == want[i][0]


def _ecdsa_jobs(sgpu, n):
    out = []
    for i in range(n):
        d, q = E.keypair(0xEC0000 + i)
        digest = hashlib.sha256(b"DNSSEC-RRSIG-V0|rec%03d.example.|A|10.0.0.%d" % (i, i)).digest()
        r, s = E.sign(digest, d, 0x5000 + 7 * i)
        out.append((sgpu.JOB_P256_ECDSA, (q, r, s, digest), sgpu.p256_ecdsa_pi(q[0], q[1], r, s, digest)))
    return out


def test_batch_with_ecdsa_jobs(sgpu, ctx):
    ecdsa = _ecdsa_jobs(sgpu, 3)
    alone = [ctx.prove_p256_ecdsa(q, r, s, dg, pi) for _, (q, r, s, dg), pi in ecdsa]
    for proof, (_, _, pi) in zip(alone, ecdsa):
        assert O.stir_verify(proof, O.build_params(256 * E.BLOWUP, pi))
    jobs, want = _mix(5, 3)
    jobs = [jobs[0], ecdsa[0], jobs[1], ecdsa[1], jobs[2], ecdsa[2], jobs[3], jobs[4]]
    want = [want[0][0], alone[0], want[1][0], alone[1], want[2][0], alone[2], want[3][0], want[4][0]]
    out = ctx.prove_batch(jobs, n_streams=4)
    for (proof, res), w in zip(out, want):
        assert res.status == 0 and proof == w
    with sgpu.Server(ctx, n_streams=2) as srv:
        tickets = [srv.submit(*j) for j in jobs]
        for t, w in zip(tickets, want):
            proof, res = srv.wait(t)
            assert res.status == 0 and proof == w


def test_ecdsa_job_rejects_bad_input(sgpu, ctx):
    with pytest.raises(sgpu.StarkGpuError):
        ctx.prove_batch([(sgpu.JOB_P256_ECDSA, b"\x00" * 159, bytes(32))])


def test_pool_reserve_then_batch(ctx):
    ctx.pool_reserve(2 << 30)
    ctx.pool_reserve(1 << 30)  # already reserved: nothing to do
    jobs, want = _mix(6, 17)
    out = ctx.prove_batch(jobs, n_streams=4, hbm_budget_bytes=3 << 30)
    for (proof, res), (wproof, _) in zip(out, want):
        assert res.status == 0 and proof == wproof

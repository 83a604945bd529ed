"""Ed25519 verify AIR (v16) on the GPU vs the oracle (bit-exact): the device trace
expansion, the gated block-interpreter merge (Phi at every LDE point, then the
quotient) on random and honest LDEs, proofs byte for byte through the
materialised and the coset-streamed merge, the full-size proof (k_scalar = 256,
n0 = 32768) byte for byte, and prove_zsk_ksk_binding_v2's native check and
pi_hash."""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle_ed25519 as OE
import oracle_lib as O

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
VEC = json.load(open(os.path.join(HERE, "golden", "ed25519_vectors.json")))["vectors"]


def _signed(tag: bytes, msg: bytes):
    seed = hashlib.sha256(tag).digest()
    _, _, pub = OE.keypair(seed)
    return pub, OE.sign(seed, msg), msg


@pytest.mark.parametrize("tag,msg,k", [(b"t1", b"m" * 32, 8), (b"t2", bytes(range(100)), 16), (b"t3", b"", 256)])
def test_device_trace_matches_oracle(sgpu, ctx, tag, msg, k):
    pub, sig, msg = _signed(tag, msg)
    _lay, _pr, want = OE.build(pub, sig, msg, k)
    assert np.array_equal(ctx.ed25519_trace(pub, sig, msg, k), want)


def test_merge_of_random_lde_matches_oracle(sgpu, ctx):
    # uniformly random LDE columns: every constraint of every row class is non-zero
    pub, sig, msg = _signed(b"rnd", b"r" * 32)
    lay, pr, _s, _k = OE.layout_program(pub, sig, msg, 8)
    blowup = 4
    rng = np.random.default_rng(25519)
    lde = rng.integers(0, O.P, size=(lay.width, lay.height * blowup), dtype=np.uint64)
    got = ctx.merge_ed25519(pub, sig, msg, lde, blowup, 8)
    assert np.array_equal(got, OE.merge(lay, pr, lde, lay.height, blowup))


@pytest.mark.parametrize("tag,msg,k", [(b"h1", b"h" * 32, 8), (b"h2", bytes(range(120)), 8),
                                       (b"h3", bytes(range(250)), 8)])
def test_merge_of_honest_lde_matches_oracle(sgpu, ctx, tag, msg, k):
    pub, sig, msg = _signed(tag, msg)
    lay, pr, tr = OE.build(pub, sig, msg, k)
    lde = O.lde(tr, 4)
    assert np.array_equal(ctx.merge_ed25519(pub, sig, msg, lde, 4, k), OE.merge(lay, pr, lde, lay.height, 4))


def test_merge_of_tampered_trace_matches_oracle(sgpu, ctx):
    pub, sig, msg = _signed(b"tmp", b"t" * 32)
    lay, pr, tr = OE.build(pub, sig, msg, 8)
    rng = np.random.default_rng(7)
    for c in rng.integers(0, lay.width, 60):
        tr[c, int(rng.integers(0, lay.height))] ^= 1
    lde = O.lde(tr, 4)
    assert np.array_equal(ctx.merge_ed25519(pub, sig, msg, lde, 4, 8), OE.merge(lay, pr, lde, lay.height, 4))


@pytest.mark.parametrize("blowup", [4, 32])
def test_proof_matches_oracle(sgpu, ctx, blowup):
    pub, sig, msg = _signed(b"prf", b"p" * 32)
    fs = hashlib.sha3_256(b"ed25519 fs binding").digest()
    lay, pr, tr = OE.build(pub, sig, msg, 8)
    got = ctx.prove_ed25519(pub, sig, msg, fs, 8, blowup)
    assert got == OE.prove(lay, pr, tr, fs, blowup)
    assert O.stir_verify(got, O.build_params(lay.height * blowup, fs))


def test_coset_streamed_merge_matches_materialised(sgpu, ctx):
    pub, sig, msg = _signed(b"cos", b"c" * 40)
    fs = hashlib.sha3_256(b"coset ed25519").digest()
    proofs = []
    for mode in (sgpu.WIDE_MERGE_LDE, sgpu.WIDE_MERGE_COSETS):
        ctx.set_option(sgpu.OPT_WIDE_MERGE, mode)
        try:
            proofs.append(ctx.prove_ed25519(pub, sig, msg, fs, 16, 32))
        finally:
            ctx.set_option(sgpu.OPT_WIDE_MERGE, sgpu.WIDE_MERGE_AUTO)
    assert proofs[0] == proofs[1]
    lay, pr, tr = OE.build(pub, sig, msg, 16)
    assert proofs[0] == OE.prove(lay, pr, tr, fs, 32)


def test_full_proof_matches_oracle_bytes(sgpu, ctx):
    # prove_zsk_ksk_binding_v2's shape: k_scalar = 256, blowup 32 (1024 rows, n0 = 32768,
    # a 10.9 GB LDE in the oracle) for RFC 8032 TEST 3's signature
    v = VEC[2]
    pub, sig, msg = bytes.fromhex(v["pub"]), bytes.fromhex(v["sig"]), bytes.fromhex(v["msg"])
    fs = hashlib.sha3_256(b"zsk-ksk fs binding").digest()
    mr = hashlib.sha3_256(b"domain to ip tree").digest()
    proof, pi = ctx.prove_zsk_ksk_binding_v2(pub, sig, msg, fs, mr)
    assert O.stir_verify(proof, O.build_params(1024 * 32, fs))
    assert pi == OE.pi_hash(pub, sig, msg, fs, mr, proof[:32])
    lay, pr, tr = OE.build(pub, sig, msg, 256)
    assert proof == OE.prove(lay, pr, tr, fs, 32)


def test_binding_refuses_an_invalid_signature(sgpu, ctx):
    pub, sig, msg = _signed(b"bad", b"zone")
    bad = bytearray(sig)
    bad[50] ^= 4
    fs = mr = bytes(32)
    with pytest.raises(sgpu.StarkGpuError) as e:
        ctx.prove_zsk_ksk_binding_v2(pub, bytes(bad), msg, fs, mr)
    assert e.value.code == sgpu.SG_EVERIFY


def test_batch_and_server_jobs(sgpu, ctx):
    # SG_JOB_ED25519 (k_scalar 256) in a batch beside a SHA-256 job, and in the server,
    # where a signature that does not verify is refused (SG_EVERIFY) without blocking the queue
    signed = [_signed(b"srv%d" % i, b"zone record %d" % i) for i in range(3)]
    fs = [hashlib.sha3_256(b"fs%d" % i).digest() for i in range(3)]
    want = [ctx.prove_ed25519(p, s, m, f, 256, 4) for (p, s, m), f in zip(signed, fs)]
    jobs = [(sgpu.JOB_ED25519, psm, f, sgpu.PHI_PARALLEL_GATE, 4) for psm, f in zip(signed, fs)]
    jobs.append((sgpu.JOB_SHA256, b"record bytes", fs[0]))
    out = ctx.prove_batch(jobs, n_streams=4)
    for i in range(3):
        assert out[i][1].status == sgpu.SG_OK and out[i][0] == want[i]
    pub, sig, msg = signed[0]
    bad = bytearray(sig)
    bad[40] ^= 1
    with sgpu.Server(ctx, n_streams=2) as srv:
        t_bad = srv.submit(sgpu.JOB_ED25519, (pub, bytes(bad), msg), fs[0], blowup=4)
        t_ok = srv.submit(sgpu.JOB_ED25519, signed[1], fs[1], blowup=4)
        with pytest.raises(sgpu.StarkGpuError) as ei:
            srv.wait(t_bad)
        assert ei.value.code == sgpu.SG_EVERIFY
        assert srv.wait(t_ok)[0] == want[1]


def test_grouped_batch_equals_proofs_alone(sgpu, ctx):
    # Ed25519 jobs (k_scalar 256, blowup 4: n0 = 4096) beside SHA-256 jobs of the same
    # n0 (480-byte messages: 8 blocks, 1024 rows) proved with lockstep STIR groups:
    # every proof equals the same job proved alone
    signed = [_signed(b"grp%d" % i, b"grouped zone record %d" % i) for i in range(4)]
    fs = [hashlib.sha3_256(b"gfs%d" % i).digest() for i in range(4)]
    jobs = [(sgpu.JOB_ED25519, psm, f, sgpu.PHI_PARALLEL_GATE, 4) for psm, f in zip(signed, fs)]
    jobs += [(sgpu.JOB_SHA256, bytes([7 + i]) * 480, fs[i], sgpu.PHI_PARALLEL_GATE, 4) for i in range(2)]
    alone = [p for p, _ in ctx.prove_batch(jobs, n_streams=1)]
    try:
        ctx.set_option(sgpu.OPT_STIR_GROUP, 8)
        got = ctx.prove_batch(jobs, n_streams=2, hbm_budget_bytes=48 << 30)
    finally:
        ctx.set_option(sgpu.OPT_STIR_GROUP, 1)
    assert all(r.status == sgpu.SG_OK for _, r in got)
    assert [p for p, _ in got] == alone

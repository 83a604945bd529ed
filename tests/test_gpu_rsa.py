"""RSA-2048 AIR on the GPU vs the oracle (bit-exact): the device trace expansion
against the host and oracle traces, the RSA merge (Phi at every LDE point, then
the quotient) against the oracle's, and whole proofs byte for byte for one record
(prove_rsa2048_record_v1.rs) and stacked records (stacked_rsa_zone_prover.rs),
including a record whose EM does not match its signature."""
import numpy as np
import pytest

import oracle_lib as O
import oracle_rsa as R

pytestmark = pytest.mark.gpu

MSG = b"DNSSEC-RRSIG-V0|google.com.|A|142.251.46.142|epoch-0"


def _records(k):
    keys = R.keys()
    return [R.record(b"rec%04d.example.com.|A|10.0.0.%d" % (i, i), keys[i % 4]) for i in range(k)]


def test_device_trace_matches_oracle(sgpu, ctx):
    recs = [r[0] for r in _records(3)]
    want = R.trace(recs)
    assert np.array_equal(ctx.rsa2048_trace(recs[:1]), want[:R.WIDTH])
    assert np.array_equal(ctx.rsa2048_trace(recs), want)


@pytest.mark.parametrize("k", [1, 2])
def test_merge_matches_oracle(sgpu, ctx, k):
    recs = [r[0] for r in _records(k)]
    lde = O.lde(R.trace(recs), R.BLOWUP)
    want = R.merge(lde, k)
    got = ctx.merge_rsa2048(lde, k)
    assert np.array_equal(got, want)


def test_merge_of_invalid_trace_matches_oracle(sgpu, ctx):
    (n, s, em), *_ = _records(1)[0]
    tr = R.trace([(n, s, (em + 7) % n)])
    tr[R.CARRY + 100, 3] ^= 1  # a carry bit flipped as well
    lde = O.lde(tr, R.BLOWUP)
    assert np.array_equal(ctx.merge_rsa2048(lde, 1), R.merge(lde, 1))


def test_single_record_proof_matches_oracle(sgpu, ctx):
    (rec, n_be, sig, em) = R.record(MSG, R.keys()[0])
    assert sgpu.rsa2048_verify(n_be, sig, em)
    pi = sgpu.rsa2048_pi_record(n_be, sig, MSG, em)
    got = ctx.prove_rsa2048([rec], pi)
    want = R.prove(R.trace([rec]), pi)
    assert got == want
    assert O.stir_verify(got, O.build_params(1024, pi))


def test_stacked_proof_matches_oracle(sgpu, ctx):
    key = R.keys()[3]
    recs, ems = [], []
    for i in range(3):
        rec, n_be, sig, em = R.record(b"DNSSEC-RRSIG-V0|rec%04d.example.com.|A|10.0.0.%d|epoch-0|alg-8" % (i, i), key)
        recs.append(rec)
        ems.append(em)
    pi = sgpu.rsa2048_pi_stacked(n_be, ems)
    got = ctx.prove_rsa2048(recs, pi)
    assert got == R.prove(R.trace(recs), pi)


def test_wrong_em_proof_matches_oracle(sgpu, ctx):
    (n, s, em), n_be, sig, emb = R.record(MSG, R.keys()[2])
    rec = (n, s, (em + 1) % n)
    assert not sgpu.rsa2048_verify(n, s, rec[2])
    pi = sgpu.rsa2048_pi_record(n_be, sig, MSG, emb)
    assert ctx.prove_rsa2048([rec], pi) == R.prove(R.trace([rec]), pi)


def test_prove_rejects_bad_records(sgpu, ctx):
    n = R.keys()[0][0]
    with pytest.raises(sgpu.StarkGpuError):
        ctx.prove_rsa2048([(n, n, 0)], bytes(32))

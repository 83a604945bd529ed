"""The RSA-2048 oracle against the properties the reference's own tests assert
(deep_ali/src/rsa2048_field_air.rs:414-620, rsa2048_exp_air.rs:288-393,
rsa2048_stacked_air.rs:72-158, rsa2048.rs:129-222): exact constraint counts, a
valid chain satisfies every constraint, a tampered c or a wrong EM does not,
the row-16 output is s^65537 mod n, limbs round-trip, and the PKCS#1 encoding
has its fixed shape. These pin the oracle; the GPU tests then compare against it."""
import hashlib
import random

import numpy as np
import pytest

import oracle_lib as O
import oracle_rsa as R

MSG = b"DNSSEC-RRSIG-V0|google.com.|A|142.251.46.142|epoch-0"


def _nonzero(tr, n_records=1, rows=range(R.N_TRACE)):
    total = 0
    for r in rows:
        cv = R.eval_row(tr[:, r], tr[:, (r + 1) % R.N_TRACE], r, n_records)
        total += int(np.count_nonzero(cv))
    return total


def test_constraint_and_cell_counts():
    assert R.WIDTH == 11041
    assert R.CONSTRAINTS == 1 + 80 + 10799 + 80 + 320
    assert 2 * 80 * 27 + 159 + 158 * 40 == 10799  # constraint_count_exact
    assert R.CARRY - R.C == 80 + 80 + 2 * 2080  # c, q, both bit blocks


def test_limb_roundtrip():
    rng = random.Random(0xCAFEF00D)
    for _ in range(16):
        x = rng.getrandbits(2040)
        limbs = R.limbs80(x)
        assert all(0 <= l < 1 << 26 for l in limbs)
        assert sum(l << (26 * i) for i, l in enumerate(limbs)) == x


def test_pkcs1_encoding_shape():
    em = R.em_encode(MSG)
    assert len(em) == 256 and em[:2] == b"\x00\x01"
    ps = 256 - 51 - 3
    assert em[2:2 + ps] == b"\xff" * ps and em[2 + ps] == 0
    assert em[3 + ps:3 + ps + 19] == R.DIGEST_INFO_SHA256
    assert em[-32:] == hashlib.sha256(MSG).digest()


def test_keys_and_signatures_are_valid():
    for key in R.keys():
        n, d = key
        assert n.bit_length() == 2048 and pow(pow(12345, 65537, n), d, n) == 12345
        (nn, s, em), _, sig, emb = R.record(MSG, key)
        assert pow(s, 65537, nn) == em


def test_valid_chain_satisfies_every_constraint_and_outputs_s_e():
    (n, s, em), *_ = R.record(MSG, R.keys()[0])
    tr = R.trace([(n, s, em)])
    assert _nonzero(tr) == 0
    c16 = sum(int(tr[R.C + i, R.OUTPUT_ROW]) << (26 * i) for i in range(80))
    assert c16 == pow(s, 65537, n)
    # phase is 1 on row 16 only
    assert [int(x) for x in tr[R.PHASE]] == [int(r == 16) for r in range(32)]


def test_small_modulus_and_zero_signature_satisfy():
    n = 0xFFFFFFFF * 0xFFFFFFFE + 3  # mul_gadget_satisfies_on_zero_a's modulus
    for s in (0, 1, 0xCAFEBABE % n):
        tr = R.trace([(n, s, pow(s, 65537, n))])
        assert _nonzero(tr) == 0


def test_tampered_c_violates():
    (n, s, em), *_ = R.record(MSG, R.keys()[1])
    tr = R.trace([(n, s, em)])
    tr[R.C, 5] = (int(tr[R.C, 5]) + 1) % O.P
    assert _nonzero(tr, rows=[4, 5]) > 0


def test_wrong_em_violates_the_row16_boundary():
    (n, s, em), *_ = R.record(MSG, R.keys()[2])
    bogus = (em + 1) % n
    tr = R.trace([(n, s, bogus)])
    cv = R.eval_row(tr[:, 16], tr[:, 17], 16)
    assert np.count_nonzero(cv[10880:10960]) >= 1
    # the other rows are still satisfied
    assert _nonzero(tr, rows=[r for r in range(32) if r != 16]) == 0


def test_stacked_records_all_zero():
    keys = R.keys()
    recs = [R.record(b"rec%04d.example.com." % i, keys[i % len(keys)])[0] for i in range(3)]
    tr = R.trace(recs)
    assert tr.shape == (3 * R.WIDTH, 32)
    assert _nonzero(tr, n_records=3) == 0


def test_oracle_proof_verifies_and_binds_pi():
    (n, s, em), n_be, sig, emb = R.record(MSG, R.keys()[0])
    tr = R.trace([(n, s, em)])
    pi = R.pi_record(n_be, sig, MSG, emb)
    proof = R.prove(tr, pi)
    p = O.build_params(1024, pi)
    assert p.sched == [8, 8, 8, 2]
    assert O.stir_verify(proof, p)
    other = O.build_params(1024, hashlib.sha3_256(b"other").digest())
    assert not O.stir_verify(proof, other)

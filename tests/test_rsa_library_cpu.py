"""Host-side RSA-2048 parts of the library against the oracle (no kernel is
launched): the C++ big-integer witness expanded on the host against the oracle's
Python-integer trace, EM encoding, the native check, the pi_hash recipes and the
argument checks."""
import hashlib

import numpy as np
import pytest

import oracle_rsa as R
from conftest import load_sgpu

MSG = b"DNSSEC-RRSIG-V0|google.com.|A|142.251.46.142|epoch-0"


@pytest.fixture(scope="module")
def sg():
    return load_sgpu()


def test_em_encoding_matches(sg):
    for m in (b"", MSG, bytes(range(256)) * 3):
        assert sg.rsa2048_em(m) == R.em_encode(m)


@pytest.mark.parametrize("k", range(4))
def test_host_trace_matches_oracle(sg, k):
    rec, *_ = R.record(MSG + bytes([k]), R.keys()[k])
    assert np.array_equal(sg.rsa2048_trace([rec]), R.trace([rec]))


def test_stacked_host_trace_matches_oracle(sg):
    keys = R.keys()
    recs = [R.record(b"rec%04d.example.com." % i, keys[i % 4])[0] for i in range(5)]
    assert np.array_equal(sg.rsa2048_trace(recs), R.trace(recs))


def test_edge_values_match_oracle(sg):
    n_small = 0xFFFFFFFF * 0xFFFFFFFE + 3
    n0 = R.keys()[0][0]
    cases = [(n_small, 0, 0), (n_small, 1, 1), (n_small, n_small - 1, pow(n_small - 1, 65537, n_small)),
             (n0, n0 - 1, pow(n0 - 1, 65537, n0)), ((1 << 2048) - 1, (1 << 2048) - 2, 0), (3, 2, 2)]
    for rec in cases:
        assert np.array_equal(sg.rsa2048_trace([rec]), R.trace([rec])), hex(rec[0])[:20]


def test_native_verify(sg):
    (n, s, em), n_be, sig, emb = R.record(MSG, R.keys()[0])
    assert sg.rsa2048_verify(n_be, sig, emb)
    assert not sg.rsa2048_verify(n_be, sig, R.em_encode(MSG + b"x"))
    assert not sg.rsa2048_verify(n_be, (s ^ 1).to_bytes(256, "big"), emb)
    assert not sg.rsa2048_verify(n_be, n_be, emb)  # s >= n
    assert not sg.rsa2048_verify(n_be, bytes(256), emb)  # s = 0


def test_pi_recipes(sg):
    (n, s, em), n_be, sig, emb = R.record(MSG, R.keys()[1])
    assert sg.rsa2048_pi_record(n_be, sig, MSG, emb) == R.pi_record(n_be, sig, MSG, emb)
    ems = [R.em_encode(b"m%d" % i) for i in range(3)]
    assert sg.rsa2048_pi_stacked(n_be, ems) == R.pi_stacked(n_be, 3, b"".join(ems))
    assert sg.rsa2048_pi_stacked(n_be, []) == hashlib.sha3_256(b"RSA2048-STACKED-ZONE" + n_be + bytes(8)).digest()


def test_rejects_bad_records(sg):
    n = R.keys()[0][0]
    for rec in [(n, n, 0), (n, n + 5, 0), (1, 0, 0), (0, 0, 0)]:
        with pytest.raises(sg.StarkGpuError):
            sg.rsa2048_trace([rec])
    with pytest.raises(ValueError):
        sg.rsa2048_trace([])

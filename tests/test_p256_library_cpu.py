"""Host-side P-256 parts of the library against the oracle (no kernel is
launched): the row layout (gadget table and tail bases), the host trace built
from the C++ witness against the oracle's Python-integer trace, the ECDSA
scalars u1/u2, the pi_hash recipe and the argument checks."""
import hashlib
import random

import numpy as np
import pytest

import oracle_p256 as E
from conftest import load_sgpu

Q2 = E._affine_add(E.G, E.G)


@pytest.fixture(scope="module")
def sg():
    return load_sgpu()


def test_layout_matches_oracle(sg):
    w, k, table, tail = sg.p256_layout()
    lay = E.Layout()
    assert (w, k) == (lay.width, lay.n_constraints)
    assert np.array_equal(table.astype(np.uint64), lay.table)
    assert np.array_equal(tail.astype(np.uint64), lay.tail)


@pytest.mark.parametrize("k,seed", [(4, 0), (8, 1), (16, 2)])
def test_host_trace_matches_oracle(sg, k, seed):
    rng = random.Random(seed)
    d, q = E.keypair(0xABCDEF + seed)
    a_bits = [rng.randrange(2) for _ in range(k)]
    b_bits = [rng.randrange(2) for _ in range(k)]
    want, _ = E.trace(E.G, a_bits, q, b_bits)
    assert np.array_equal(sg.p256_chain_trace(E.G, a_bits, q, b_bits), want)


def test_all_zero_and_all_one_bits(sg):
    for bits in ([0] * 8, [1] * 8):
        want, _ = E.trace(E.G, bits, Q2, bits[::-1])
        assert np.array_equal(sg.p256_chain_trace(E.G, bits, Q2, bits[::-1]), want)


def test_u_bits_and_pi(sg):
    d, q = E.keypair(0x5EED)
    digest = hashlib.sha256(b"DNSSEC-RRSIG-V0|rec0001.example.com.|A|10.0.0.1").digest()
    r, s = E.sign(digest, d, 0xFEEDFACE)
    assert sg.p256_u_bits(digest, r, s) == E.u_bits(digest, r, s)
    assert sg.p256_ecdsa_pi(q[0], q[1], r, s, digest) == E.pi_hash(q[0], q[1], r, s, digest)
    # a digest above n is reduced first
    big = (E.N + 5).to_bytes(32, "big")
    assert sg.p256_u_bits(big, r, s) == E.u_bits(big, r, s)


def test_rejects_bad_inputs(sg):
    with pytest.raises(sg.StarkGpuError):
        sg.p256_chain_trace((E.GX, (E.GY + 1) % E.P), [1, 0], E.G, [0, 1])  # off the curve
    with pytest.raises(sg.StarkGpuError):
        sg.p256_chain_trace((E.P, E.GY), [1, 0], E.G, [0, 1])  # coordinate not below p
    with pytest.raises(sg.StarkGpuError):
        sg.p256_chain_trace(E.G, [1, 0, 1], E.G, [0, 1, 1])  # not a power of 2
    digest = bytes(32)
    for r, s in ((0, 1), (1, 0), (E.N, 1), (1, E.N)):
        with pytest.raises(sg.StarkGpuError):
            sg.p256_u_bits(digest, r, s)


def test_ecdsa_job_packing(sg):
    d, q = E.keypair(0x77)
    digest = hashlib.sha256(b"job").digest()
    r, s = E.sign(digest, d, 0x99)
    j, buf = sg.make_job(sg.JOB_P256_ECDSA, (q, r, s, digest), bytes(32))
    want = b"".join(v.to_bytes(32, "big") for v in (q[0], q[1], r, s)) + digest
    assert j.kind == sg.JOB_P256_ECDSA and j.input_len == 160 and bytes(buf)[:160] == want
    j2, _ = sg.make_job(sg.JOB_P256_ECDSA, want, bytes(32))
    assert j2.input_len == 160

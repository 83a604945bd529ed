"""Ed25519 verify AIR (v16) on the CPU: the oracle against the reference's
known answers, and the library's host side against the oracle (no kernel is
launched).

Pins: the oracle's RFC 8032 signer reproduces TEST 1 of the reference's own
tests (tests/golden/ed25519_vectors.json, read from ed25519_verify.rs) and its
verifier accepts TEST 1-3; the traces built from those signatures satisfy every
constraint of the program pinned in tests/test_air_vectors.py on every row.
Library: its constraint program (block records and pairs) and its host trace
are identical to the oracle's; its native verifier and pi_hash recipe agree."""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle_ed25519 as OE
from conftest import load_sgpu

HERE = os.path.dirname(os.path.abspath(__file__))
VEC = json.load(open(os.path.join(HERE, "golden", "ed25519_vectors.json")))["vectors"]


@pytest.fixture(scope="module")
def sg():
    return load_sgpu()


def _vec(v):
    return bytes.fromhex(v["pub"]), bytes.fromhex(v["sig"]), bytes.fromhex(v["msg"])


def _signed(tag: bytes, msg: bytes):
    seed = hashlib.sha256(tag).digest()
    _, _, pub = OE.keypair(seed)
    return pub, OE.sign(seed, msg), msg


def test_oracle_signer_reproduces_rfc8032_test1():
    v = VEC[0]
    secret = bytes.fromhex(v["secret"])
    _, _, pub = OE.keypair(secret)
    assert pub.hex() == v["pub"]
    assert OE.sign(secret, bytes.fromhex(v["msg"])).hex() == v["sig"]


@pytest.mark.parametrize("i", range(len(VEC)))
def test_oracle_verifier_accepts_rfc8032(i):
    pub, sig, msg = _vec(VEC[i])
    assert OE.verify(pub, sig, msg)
    assert not OE.verify(pub, sig, msg + b"\x00")
    bad = bytearray(sig)
    bad[40] ^= 1
    assert not OE.verify(pub, bytes(bad), msg)


def test_constants():
    assert OE.D_INT * 121666 % OE.P == (-121665) % OE.P
    assert OE.SQRT_M1 ** 2 % OE.P == OE.P - 1
    x, y = OE.affine(OE.BASEPOINT)
    assert y == 4 * pow(5, OE.P - 2, OE.P) % OE.P and x % 2 == 0
    assert (-x * x + y * y - 1 - OE.D_INT * x * x * y * y) % OE.P == 0
    # L in the C++ oracle's 16-bit limbs
    assert sum(l << (16 * i) for i, l in enumerate([0xd3ed, 0x5cf5, 0x631a, 0x5812, 0x9cd6, 0xa2f7, 0xf9de, 0x14de,
                                                    0, 0, 0, 0, 0, 0, 0, 0x1000])) == OE.L_ORDER


@pytest.mark.parametrize("i", range(len(VEC)))
def test_rfc8032_traces_satisfy_every_constraint(i):
    pub, sig, msg = _vec(VEC[i])
    lay, pr, tr = OE.build(pub, sig, msg, 256)
    for row in range(lay.height):
        v = OE.eval_row(pr, tr[:, row], tr[:, (row + 1) % lay.height], row)
        assert not v.any(), f"row {row}: constraints {np.nonzero(v)[0][:8]}"


def test_tampered_trace_fires():
    pub, sig, msg = _signed(b"tamper", b"x" * 32)
    lay, pr, tr = OE.build(pub, sig, msg, 8)
    for row, col in ((lay.sB_first + 3, lay.mdbl.mul_X3.c + 2), (lay.residual_row, lay.pa_R2.mul_Z3.carry + 5),
                     (lay.decomp_A_row, lay.decomp.x_bits + 7), (lay.reduce_row, lay.red["q"] + 1),
                     (lay.k_hash - 1, lay.digest_bits + 100)):
        t = tr.copy()
        t[col, row] ^= 1
        v = OE.eval_row(pr, t[:, row], t[:, (row + 1) % lay.height], row)
        assert v.any(), (row, col)


@pytest.mark.parametrize("tag,msg,k", [(b"a", b"m" * 32, 8), (b"b", bytes(range(100)), 16), (b"c", b"", 4),
                                       (b"e", bytes(range(250)), 8)])
def test_library_program_matches_oracle(sg, tag, msg, k):
    pub, sig, msg = _signed(tag, msg)
    lay, pr, _s, _k = OE.layout_program(pub, sig, msg, k)
    recs, pairs = sg.ed25519_program(pub, sig, msg, k)
    assert np.array_equal(recs, pr.records())
    assert np.array_equal(pairs, pr.pair_array())
    w, h, n, rows = sg.ed25519_layout(len(msg), k)
    assert (w, h, n) == (lay.width, lay.height, pr.n)
    assert (rows["residual_row"], rows["result_row"]) == (lay.residual_row, lay.result_row)


@pytest.mark.parametrize("tag,msg,k", [(b"a", b"m" * 32, 8), (b"b", bytes(range(100)), 16), (b"d", b"", 256),
                                       (b"e", bytes(range(250)), 8)])
def test_library_host_trace_matches_oracle(sg, tag, msg, k):
    pub, sig, msg = _signed(tag, msg)
    _lay, _pr, want = OE.build(pub, sig, msg, k)
    assert np.array_equal(sg.ed25519_trace(pub, sig, msg, k), want)


def test_concurrent_host_traces_match_oracle(sg):
    # witnesses built at once from several host threads (as server workers do) share
    # the host's threads and wait row by row for their accumulators: each trace still
    # equals the oracle's
    import threading
    cases = [_signed(b"conc%d" % i, bytes(range(i, i + 40))) for i in range(6)]
    want = [OE.build(p, s, m, 16)[2] for p, s, m in cases]
    got = [None] * len(cases)

    def work(i):
        p, s, m = cases[i]
        got[i] = sg.ed25519_trace(p, s, m, 16)

    th = [threading.Thread(target=work, args=(i,)) for i in range(len(cases))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for i in range(len(cases)):
        assert np.array_equal(got[i], want[i]), i


@pytest.mark.parametrize("i", range(len(VEC)))
def test_library_verify(sg, i):
    pub, sig, msg = _vec(VEC[i])
    assert sg.ed25519_verify(pub, sig, msg)
    assert not sg.ed25519_verify(pub, sig, msg + b"\x01")
    bad = bytearray(pub)
    bad[3] ^= 1
    assert not sg.ed25519_verify(bytes(bad), sig, msg)
    bad_s = bytearray(sig)  # a flipped bit of S (the reference's tamper test)
    bad_s[40] ^= 1
    assert not sg.ed25519_verify(pub, bytes(bad_s), msg)
    assert not OE.verify(pub, bytes(bad_s), msg)
    # S >= L is refused (ed25519_verify.rs:80)
    s = int.from_bytes(sig[32:], "little") + OE.L_ORDER
    if s < 1 << 256:
        assert not sg.ed25519_verify(pub, sig[:32] + s.to_bytes(32, "little"), msg)


def test_library_pi_hash(sg):
    pub, sig, msg = _signed(b"pi", b"zone data")
    fs, mr, rf = (hashlib.sha3_256(t).digest() for t in (b"fs", b"mr", b"rf"))
    assert sg.ed25519_pi_hash(pub, sig, msg, fs, mr, rf) == OE.pi_hash(pub, sig, msg, fs, mr, rf)


def test_library_refuses_bad_encodings(sg):
    pub, sig, msg = _signed(b"enc", b"m")
    y_ge_p = (OE.P + 1).to_bytes(32, "little")  # y >= p
    with pytest.raises(sg.StarkGpuError):
        sg.ed25519_trace(y_ge_p, sig, msg, 8)
    with pytest.raises(sg.StarkGpuError):
        sg.ed25519_trace(pub, y_ge_p + sig[32:], msg, 8)
    # y = 2 is not the y of a curve point (2^2 - 1 over 4d + 1 is not a square)
    assert OE.decompress((2).to_bytes(32, "little")) is None
    with pytest.raises(sg.StarkGpuError):
        sg.ed25519_trace((2).to_bytes(32, "little"), sig, msg, 8)
    with pytest.raises(sg.StarkGpuError):
        sg.ed25519_layout(1, 1)
    with pytest.raises(sg.StarkGpuError):
        sg.ed25519_layout(1, 257)

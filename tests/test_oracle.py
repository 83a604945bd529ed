"""Pins the CPU oracle before it is trusted as the GPU library's checker.

Known answers: the ark-goldilocks test identities (crates/ark-goldilocks/src/lib.rs:54-139),
FIPS 202 via hashlib, RFC 8439 §2.3.2 for the ChaCha block function, the
omega0 fields of the golden proofs, and -- the strongest pin -- byte
identity with the reference-produced golden proofs
primary-state/proofs/{outer-rollup,inner-shard-000[123]}.bin.
"""
import hashlib
import os
import random
import struct

import numpy as np
import pytest

import dnszone
import oracle_lib as O

P = O.P


def test_field_known_answers():
    L = O.lib()
    assert L.orc_fp_add(0, 1) == 1
    assert L.orc_fp_mul(2, 3) == 6
    assert L.orc_fp_sub(0, 5) == P - 5
    # generator 7 has full order p-1 (ark-goldilocks/src/lib.rs:67-73)
    assert L.orc_fp_pow(7, P - 1) == 1
    assert L.orc_fp_pow(7, (P - 1) // 2) != 1
    a = 123456789
    assert L.orc_fp_mul(a, L.orc_fp_inv(a)) == 1
    # Legendre: 25 residue, 11 non-residue (:85-92)
    assert L.orc_fp_pow(25, (P - 1) // 2) == 1
    assert L.orc_fp_pow(11, (P - 1) // 2) == P - 1
    root = L.orc_root_of_unity(32)
    assert root == pow(7, (P - 1) >> 32, P)
    assert L.orc_fp_pow(root, 1 << 32) == 1 and L.orc_fp_pow(root, 1 << 31) != 1
    # omega0 fields of the golden proofs (n0 = 512 and 131072)
    assert L.orc_root_of_unity(9) == 1803076106186727246
    assert L.orc_root_of_unity(17) == 12380578893860276750
    rng = random.Random(1)
    for _ in range(2000):
        x, y = rng.randrange(P), rng.randrange(P)
        assert L.orc_fp_mul(x, y) == x * y % P
        assert L.orc_fp_add(x, y) == (x + y) % P
        assert L.orc_fp_sub(x, y) == (x - y) % P
    for x, y in [(P - 1, P - 1), (P - 1, 2), (1 << 63, 1 << 63), (0xFFFFFFFF, 0xFFFFFFFF00000000)]:
        assert L.orc_fp_mul(x, y) == x * y % P


# Independent Python model of Fp6 = Fp3[u]/(u^2 - a), Fp3 = Fp[a]/(a^3 - 7):
# multiply as polynomials in (a, u) and reduce.
def _f3mul(x, y):
    r = [0] * 5
    for i in range(3):
        for j in range(3):
            r[i + j] += x[i] * y[j]
    return [(r[0] + 7 * r[3]) % P, (r[1] + 7 * r[4]) % P, r[2] % P]


def _f6mul(x, y):
    a0, a1, b0, b1 = x[:3], x[3:], y[:3], y[3:]
    v0, v1 = _f3mul(a0, b0), _f3mul(a1, b1)
    c0 = [(v0[0] + 7 * v1[2]) % P, (v0[1] + v1[0]) % P, (v0[2] + v1[1]) % P]
    c1 = [(s + t) % P for s, t in zip(_f3mul(a0, b1), _f3mul(a1, b0))]
    return c0 + c1


def test_fp6_against_python_model():
    rng = random.Random(2)
    one = [1, 0, 0, 0, 0, 0]
    for _ in range(200):
        a = [rng.randrange(P) for _ in range(6)]
        b = [rng.randrange(P) for _ in range(6)]
        assert O.fp6_mul(a, b) == _f6mul(a, b)
        assert O.fp6_mul(a, O.fp6_inv(a)) == one


def test_sha3_matches_hashlib():
    rng = random.Random(3)
    for n in list(range(0, 300)) + [543, 544, 545, 1000, 4096]:
        m = bytes(rng.randrange(256) for _ in range(n))
        assert O.sha3_256(m) == hashlib.sha3_256(m).digest()


def test_chacha_block_rfc8439():
    # RFC 8439 §2.3.2: key 00..1f, block counter 1, nonce 00:00:00:09:00:00:00:4a:00:00:00:00.
    # In the 64-bit-counter layout: word12 = counter, word13 = first nonce word.
    key = bytes(range(32))
    counter = 1 | (0x09000000 << 32)
    stream = 0x4A000000
    out = O.chacha_block(key, counter, stream, 20)
    assert out == [0xE4E7F110, 0x15593BD1, 0x1FDD0F50, 0xC47120A3, 0xC7F4D1C7, 0x0368C033, 0x9AAA2204,
                   0x4E6CD4C3, 0x466482D2, 0x09AA9F07, 0x05D7C214, 0xA2028BD9, 0xD19C12B5, 0xB94E16DE,
                   0xE883D0CB, 0x4E3C50A2]


def _naive_dft(a, w):
    n = len(a)
    return [sum(int(a[j]) * pow(w, j * k, P) for j in range(n)) % P for k in range(n)]


def test_ntt_matches_naive_dft():
    rng = np.random.default_rng(4)
    L = O.lib()
    for lg in range(0, 8):
        n = 1 << lg
        a = rng.integers(0, P, n, dtype=np.uint64)
        w = L.orc_root_of_unity(lg)
        assert list(O.ntt(a)) == _naive_dft(list(a), w)
        assert list(O.ntt(O.ntt(a), inverse=True)) == list(a)


def test_lde_matches_polynomial_evaluation():
    rng = np.random.default_rng(5)
    L = O.lib()
    n, B = 8, 4
    tr = rng.integers(0, P, (3, n), dtype=np.uint64)
    for shift in (1, 7):
        out = O.lde(tr, B, shift)
        wn = L.orc_root_of_unity(3)
        wN = L.orc_root_of_unity(5)
        for c in range(3):
            coeffs = [x * pow(n, P - 2, P) % P for x in _naive_dft(list(tr[c]), pow(wn, P - 2, P))]
            for i in range(n * B):
                x = shift * pow(wN, i, P) % P
                assert int(out[c, i]) == sum(cf * pow(x, k, P) for k, cf in enumerate(coeffs)) % P


def test_poly_div_zh_matches_naive():
    rng = random.Random(6)
    for n, m in [(32, 8), (64, 4), (16, 16), (8, 16), (128, 32)]:
        d = [rng.randrange(P) for _ in range(n)]
        q = O.poly_div_zh(d, m)
        if n <= m:
            assert list(q) == [0]
            continue
        # long division by X^m - 1, remainder dropped
        rem = list(d)
        quo = [0] * (n - m)
        for k in range(n - 1, m - 1, -1):
            c = rem[k]
            quo[k - m] = c
            rem[k] = 0
            rem[k - m] = (rem[k - m] + c) % P
        assert [int(x) for x in q] == quo


def _py_merkle(rows, arities, label):
    def ds(ar, lvl, pos):
        return struct.pack("<4Q", ar, lvl, pos, label)
    lvl = [hashlib.sha3_256(ds(arities[0], 0xFFFFFFFF, i) + struct.pack(f"<{len(r)}Q", *map(int, r))).digest()
           for i, r in enumerate(rows)]
    li = 0
    while len(lvl) > 1:
        a = arities[li]
        while len(lvl) % a:
            lvl.append(lvl[-1])
        lvl = [hashlib.sha3_256(ds(a, li + 1, j) + b"".join(lvl[j * a:(j + 1) * a])).digest()
               for j in range(len(lvl) // a)]
        li += 1
    return lvl[0]


@pytest.mark.parametrize("n,width,arities,label", [
    (1, 6, [2], 0xFE), (5, 3, [2, 2, 2], 7), (16, 8, [16], 0xFF), (100, 4, [8, 8, 8], 1), (37, 2, [4, 4, 4], 0),
])
def test_merkle_root_matches_python(n, width, arities, label):
    rows = np.random.default_rng(n).integers(0, P, (n, width), dtype=np.uint64)
    assert O.merkle_root(rows, arities, label) == _py_merkle(rows, arities, label)


def test_golden_outer_rollup(golden):
    leaves, pk = dnszone.outer_rollup_inputs(golden)
    proof = O.prove_hash_rollup(leaves, pk)
    e = golden["outer"]
    assert len(proof) == e["len"]
    assert hashlib.sha3_256(proof).hexdigest() == e["sha3_256"]
    assert proof[:32].hex() == e["root_f0_expected_hex"]
    assert O.stir_verify(proof, O.build_params(e["n0"], pk))


@pytest.mark.parametrize("idx", [0, 1, 2])
def test_golden_inner_shard(golden, idx):
    sh = golden["shards"][idx]
    leaves, fsb, root, count = dnszone.inner_shard_inputs(golden, sh)
    assert root.hex() == sh["merkle_root_hex"]
    proof = O.prove_hash_rollup(leaves, fsb)
    assert len(proof) == sh["len"]
    assert hashlib.sha3_256(proof).hexdigest() == sh["sha3_256"]
    pi = dnszone.shard_pi_hash(bytes.fromhex(golden["zone_salt_hex"]), count, root, proof[:32], fsb)
    assert pi.hex() == sh["pi_hash_hex"]
    assert O.stir_verify(proof, O.build_params(sh["n0"], fsb))


def test_phi_gate_modes(golden):
    # n0 = 512 < 4096: the reference's parallel build leaves Φ = 0 (all-zero fz),
    # a sequential build would prove the true quotient.
    leaves, pk = dnszone.outer_rollup_inputs(golden)
    gated = O.prove_hash_rollup(leaves, pk, O.PHI_PARALLEL_GATE)
    never = O.prove_hash_rollup(leaves, pk, O.PHI_NEVER)
    always = O.prove_hash_rollup(leaves, pk, O.PHI_ALWAYS)
    assert gated == never
    assert always != gated
    assert O.stir_verify(always, O.build_params(512, pk))


def test_verifier_rejects_tampering(golden):
    leaves, pk = dnszone.outer_rollup_inputs(golden)
    params = O.build_params(512, pk)
    proof = bytearray(O.prove_hash_rollup(leaves, pk, O.PHI_ALWAYS))
    assert O.stir_verify(bytes(proof), params)
    rng = random.Random(7)
    for _ in range(40):
        i = rng.randrange(len(proof))
        bad = bytearray(proof)
        bad[i] ^= 1 << rng.randrange(8)
        assert not O.stir_verify(bytes(bad), params), i
    other = O.build_params(512, bytes(32))
    assert not O.stir_verify(bytes(proof), other)


@pytest.mark.parametrize("lg", [3, 6, 9, 11, 13])
def test_prove_verify_round_trip_low_degree(lg):
    n0 = 1 << lg
    rng = np.random.default_rng(lg)
    # a degree-0 polynomial passes the d_final = 1 check whatever the schedule
    f0 = np.full(n0, int(rng.integers(0, P, dtype=np.uint64)), dtype=np.uint64)
    params = O.build_params(n0, os.urandom(32))
    proof = O.stir_prove(f0, params)
    assert O.stir_verify(proof, params)


def _low_degree_f0(n0, seed):
    rng = np.random.default_rng(seed)
    c = np.zeros(n0, dtype=np.uint64)
    k = max(1, n0 // 32)
    c[:k] = rng.integers(0, O.P, k, dtype=np.uint64)
    return O.ntt(c)


@pytest.mark.parametrize("log_n0", [2, 4, 7, 10])
def test_classic_fri_oracle_round_trip(log_n0):
    # classic DEEP-FRI branch (params.stir = false): the oracle's proof verifies,
    # and changing a checked byte (root, layer opening, payload, fz, final poly) is rejected
    import hashlib
    n0 = 1 << log_n0
    f0 = _low_degree_f0(n0, log_n0)
    p = O.build_params(n0, hashlib.sha3_256(b"classic").digest(), stir=False)
    assert p.sched == [2] * log_n0
    proof = O.stir_prove(f0, p)
    assert O.stir_verify(proof, p)
    for pos in (5, 40, 300, len(proof) - 60):
        bad = bytearray(proof)
        bad[pos] ^= 0x10
        assert not O.stir_verify(bytes(bad), p), pos
    p2 = O.build_params(n0, hashlib.sha3_256(b"other").digest(), stir=False)
    assert not O.stir_verify(proof, p2)

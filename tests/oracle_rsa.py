"""RSA-2048 part of the CPU oracle (test infrastructure only).

The trace is restated here with Python integers, independent of the library's
C++ big-integer code; the constraint evaluation, merge and proof go through
the C++ oracle (oracle/rsa2048_air.hpp, oracle/oracle.cpp).

Follows (stark-stir-swarm paths):
  crates/deep_ali/src/rsa2048_field_air.rs:190-221  biguint_to_limbs80 (26-bit limbs, little-endian)
  crates/deep_ali/src/rsa2048_field_air.rs:241-326  fill_rsa_mul_gadget (c, q, carry chain, bits)
  crates/deep_ali/src/rsa2048_exp_air.rs:126-204    fill_rsa_exp_multirow (phase 1 only on row 16)
  crates/deep_ali/src/rsa2048.rs:36-41,71-90        SHA-256 DigestInfo prefix, EMSA-PKCS1-v1_5 encode
  crates/swarm-dns/examples/prove_rsa2048_record_v1.rs:178-187  pi_hash "RSA2048-V2-PI-PRE"
  crates/swarm-dns/examples/stacked_rsa_zone_prover.rs:158-165  pi_hash "RSA2048-STACKED-ZONE"
"""
import ctypes
import hashlib
import json
import os

import numpy as np

import oracle_lib as O

LIMBS, LIMB_BITS, SLOTS, CARRY_BITS = 80, 26, 159, 40
CARRY_POS = SLOTS - 1
CARRY_OFFSET = 1 << (CARRY_BITS - 1)
ACC, S, N, PHASE, OP2, EM, C, Q = 0, 80, 160, 240, 241, 321, 401, 481
Q_BITS = 561
C_BITS = Q_BITS + LIMBS * LIMB_BITS
CARRY = C_BITS + LIMBS * LIMB_BITS
WIDTH = CARRY + CARRY_BITS * CARRY_POS
CONSTRAINTS = 11280
N_TRACE, BLOWUP = 32, 32
OUTPUT_ROW = 16
assert WIDTH == 11041

DIGEST_INFO_SHA256 = bytes([0x30, 0x31, 0x30, 0x0D, 0x06, 0x09, 0x60, 0x86, 0x48, 0x01,
                            0x65, 0x03, 0x04, 0x02, 0x01, 0x05, 0x00, 0x04, 0x20])


def limbs80(x: int):
    assert 0 <= x < 1 << (LIMBS * LIMB_BITS)
    return [(x >> (LIMB_BITS * i)) & ((1 << LIMB_BITS) - 1) for i in range(LIMBS)]


def em_encode(msg: bytes, k: int = 256) -> bytes:
    """EMSA-PKCS1-v1_5 of SHA-256(msg) into k bytes (RFC 8017 9.2)."""
    t = DIGEST_INFO_SHA256 + hashlib.sha256(msg).digest()
    assert k >= len(t) + 11
    return b"\x00\x01" + b"\xff" * (k - len(t) - 3) + b"\x00" + t


def pi_record(n_be: bytes, sig: bytes, msg: bytes, em: bytes) -> bytes:
    return hashlib.sha3_256(b"RSA2048-V2-PI-PRE" + n_be + sig + msg + em).digest()


def pi_stacked(n_be: bytes, n_records: int, ems: bytes) -> bytes:
    return hashlib.sha3_256(b"RSA2048-STACKED-ZONE" + n_be + n_records.to_bytes(8, "little") + ems).digest()


def fill_record(cols, base: int, n: int, s: int, em: int, n_trace: int = N_TRACE):
    """fill_rsa_exp_multirow into cols[base + cell][row] (Python ints)."""
    s_l, n_l, em_l = limbs80(s), limbs80(n), limbs80(em)
    acc = s
    radix = 1 << LIMB_BITS
    for r in range(n_trace):
        for i in range(LIMBS):
            cols[base + S + i][r] = s_l[i]
            cols[base + N + i][r] = n_l[i]
            cols[base + EM + i][r] = em_l[i]
        a_l = limbs80(acc)
        for i in range(LIMBS):
            cols[base + ACC + i][r] = a_l[i]
        phase = r == OUTPUT_ROW
        cols[base + PHASE][r] = int(phase)
        op2 = s if phase else acc
        b_l = limbs80(op2)
        for i in range(LIMBS):
            cols[base + OP2 + i][r] = b_l[i]
        prod = acc * op2
        c, q = prod % n, prod // n
        c_l, q_l = limbs80(c), limbs80(q)
        carry = 0
        carries = []
        for k in range(SLOTS):
            lo, hi = max(0, k - (LIMBS - 1)), min(LIMBS - 1, k)
            pab = sum(a_l[i] * b_l[k - i] for i in range(lo, hi + 1))
            pqn = sum(q_l[i] * n_l[k - i] for i in range(lo, hi + 1))
            lhs = pab - pqn - (c_l[k] if k < LIMBS else 0) + carry
            if k < SLOTS - 1:
                assert lhs % radix == 0
                carry = lhs // radix
                assert abs(carry) < CARRY_OFFSET
                carries.append(carry)
            else:
                assert lhs == 0
        for i in range(LIMBS):
            cols[base + C + i][r] = c_l[i]
            cols[base + Q + i][r] = q_l[i]
            for b in range(LIMB_BITS):
                cols[base + C_BITS + i * LIMB_BITS + b][r] = (c_l[i] >> b) & 1
                cols[base + Q_BITS + i * LIMB_BITS + b][r] = (q_l[i] >> b) & 1
        for k in range(CARRY_POS):
            biased = carries[k] + CARRY_OFFSET
            for b in range(CARRY_BITS):
                cols[base + CARRY + k * CARRY_BITS + b][r] = (biased >> b) & 1
        acc = c


def trace(records, n_trace: int = N_TRACE) -> np.ndarray:
    """records = [(n, s, em) ints]; returns (len(records) * 11041, n_trace) uint64."""
    cols = [[0] * n_trace for _ in range(len(records) * WIDTH)]
    for r, (n, s, em) in enumerate(records):
        fill_record(cols, r * WIDTH, n, s, em, n_trace)
    return np.array(cols, dtype=np.uint64)


def _lib():
    L = O.lib()
    if not getattr(L, "_rsa_bound", False):
        L.orc_rsa_eval.argtypes = [O.U64P, O.U64P, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, O.U64P]
        L.orc_merge_rsa.argtypes = [O.U64P, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, O.U64P]
        L.orc_prove_rsa.argtypes = [O.U64P, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_char_p, ctypes.c_size_t,
                                    ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
        L._rsa_bound = True
    return L


def eval_row(cur, nxt, row, n_records=1, n_trace=N_TRACE):
    cur = np.ascontiguousarray(cur, dtype=np.uint64)
    nxt = np.ascontiguousarray(nxt, dtype=np.uint64)
    out = np.zeros(n_records * CONSTRAINTS, dtype=np.uint64)
    _lib().orc_rsa_eval(O._ptr(cur), O._ptr(nxt), row, n_trace, n_records, O._ptr(out))
    return out


def merge(lde_cols, n_records, n_trace=N_TRACE, blowup=BLOWUP):
    lde_cols = np.ascontiguousarray(lde_cols, dtype=np.uint64)
    out = np.zeros(n_trace * blowup, dtype=np.uint64)
    assert _lib().orc_merge_rsa(O._ptr(lde_cols), n_records, n_trace, blowup, O._ptr(out)) == 0
    return out


def prove(tr: np.ndarray, pi: bytes, n_trace=N_TRACE, blowup=BLOWUP) -> bytes:
    tr = np.ascontiguousarray(tr, dtype=np.uint64)
    n_records = tr.shape[0] // WIDTH
    cap = 1 << 24
    buf = ctypes.create_string_buffer(cap)
    ln = ctypes.c_size_t()
    rc = _lib().orc_prove_rsa(O._ptr(tr), n_records, n_trace, pi, blowup, buf, cap, ctypes.byref(ln))
    assert rc == 0, rc
    return buf.raw[:ln.value]


KEYS_JSON = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "rsa2048_keys.json")


def keys():
    """Seeded RSA-2048 test keys (tests/golden/make_rsa_keys.py): [(n, d)]."""
    with open(KEYS_JSON) as f:
        return [(int(k["n"], 16), int(k["d"], 16)) for k in json.load(f)["keys"]]


def sign(msg: bytes, n: int, d: int) -> bytes:
    """RSASSA-PKCS1-v1_5 signature (RSASP1 of the encoded message), 256 bytes big-endian."""
    return pow(int.from_bytes(em_encode(msg), "big"), d, n).to_bytes(256, "big")


def record(msg: bytes, key):
    """(n, s, em) ints and the byte strings the pi recipes hash."""
    n, d = key
    sig = sign(msg, n, d)
    em = em_encode(msg)
    return (n, int.from_bytes(sig, "big"), int.from_bytes(em, "big")), n.to_bytes(256, "big"), sig, em

"""ctypes binding of the CPU oracle (oracle/liboracle.so) for the tests.

The oracle is the checker only: tests compare the GPU library's outputs with
it. It is built on first use with `make -C oracle`.
"""
import ctypes
import os
import subprocess
import threading

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
# The hash profile (the reference's compile-time sha3-256 / sha3-384 / sha3-512
# feature) is chosen per process, as the library's is: STARK_GPU_HASH.
HASH_PROFILE = os.environ.get("STARK_GPU_HASH", "sha3-256")
_SO_NAME = {"sha3-256": "liboracle.so", "sha3-384": "liboracle_sha3_384.so", "sha3-512": "liboracle_sha3_512.so"}
ORACLE_SO = os.path.join(ORACLE_DIR, _SO_NAME[HASH_PROFILE])
HASH_BYTES = {"sha3-256": 32, "sha3-384": 48, "sha3-512": 64}[HASH_PROFILE]
P = 0xFFFFFFFF00000001

PHI_PARALLEL_GATE, PHI_ALWAYS, PHI_NEVER = 0, 1, 2
AIR_HASH_ROLLUP, AIR_SHA256 = 4, 6


class FriParams(ctypes.Structure):
    _fields_ = [
        ("schedule", ctypes.c_uint64 * 64),
        ("schedule_len", ctypes.c_uint64),
        ("r", ctypes.c_uint64),
        ("s0", ctypes.c_uint64),
        ("seed_z", ctypes.c_uint64),
        ("d_final", ctypes.c_uint64),
        ("coeff_commit_final", ctypes.c_int32),
        ("stir", ctypes.c_int32),
        ("has_pi", ctypes.c_int32),
        ("pi_hash", ctypes.c_uint8 * 32),
    ]

    @property
    def sched(self):
        return [self.schedule[i] for i in range(self.schedule_len)]


_lock = threading.Lock()
_lib = None

U64P = ctypes.POINTER(ctypes.c_uint64)


def _ptr(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(U64P)


def lib():
    global _lib
    with _lock:
        if _lib is None:
            subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
            L = ctypes.CDLL(ORACLE_SO)
            assert L.orc_hash_bytes() == HASH_BYTES, "oracle library of another hash profile"
            L.orc_fp_add.restype = L.orc_fp_sub.restype = L.orc_fp_mul.restype = ctypes.c_uint64
            L.orc_fp_pow.restype = L.orc_fp_inv.restype = ctypes.c_uint64
            for f in ("orc_fp_add", "orc_fp_sub", "orc_fp_mul", "orc_fp_pow"):
                getattr(L, f).argtypes = [ctypes.c_uint64, ctypes.c_uint64]
            L.orc_fp_inv.argtypes = [ctypes.c_uint64]
            L.orc_root_of_unity.restype = ctypes.c_uint64
            L.orc_root_of_unity.argtypes = [ctypes.c_uint]
            L.orc_stdrng_first_u64.restype = ctypes.c_uint64
            L.orc_lde.argtypes = [U64P, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_uint64, U64P]
            L.orc_ntt.argtypes = [U64P, ctypes.c_size_t, ctypes.c_int]
            L.orc_merge.argtypes = [ctypes.c_int, U64P, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, U64P,
                                    ctypes.c_size_t, ctypes.c_int, U64P]
            L.orc_poly_div_zh.argtypes = [U64P, ctypes.c_size_t, ctypes.c_size_t, U64P]
            L.orc_merkle_root.argtypes = [U64P, ctypes.c_size_t, ctypes.c_size_t, U64P, ctypes.c_size_t,
                                          ctypes.c_uint64, ctypes.c_char_p]
            L.orc_hash_rollup_trace.argtypes = [U64P, ctypes.c_size_t, ctypes.c_size_t, U64P]
            L.orc_build_params.argtypes = [ctypes.c_size_t, ctypes.c_char_p, ctypes.c_int,
                                           ctypes.POINTER(FriParams)]
            L.orc_stir_prove.argtypes = [U64P, ctypes.c_size_t, ctypes.POINTER(FriParams), ctypes.c_char_p,
                                         ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
            L.orc_stir_verify.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(FriParams)]
            L.orc_prove_hash_rollup.argtypes = [U64P, ctypes.c_size_t, ctypes.c_char_p, ctypes.c_int,
                                                ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]
            L.orc_chacha_block.argtypes = [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_uint32)]
            L.orc_merge_sha256.argtypes = [U64P, ctypes.c_size_t, ctypes.c_size_t, U64P, ctypes.c_size_t,
                                           ctypes.c_int, U64P]
            L.orc_sha256_trace.argtypes = [ctypes.c_char_p, ctypes.c_size_t, U64P, ctypes.c_size_t,
                                           ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]
            L.orc_sha256_eval.argtypes = [U64P, U64P, ctypes.c_size_t, ctypes.c_size_t, U64P]
            L.orc_prove_sha256.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p, ctypes.c_int,
                                           ctypes.c_size_t, ctypes.c_char_p, ctypes.c_size_t,
                                           ctypes.POINTER(ctypes.c_size_t), ctypes.c_char_p]
            L.orc_merge_sha512.argtypes = L.orc_merge_sha256.argtypes
            L.orc_sha512_trace.argtypes = L.orc_sha256_trace.argtypes
            L.orc_sha512_eval.argtypes = L.orc_sha256_eval.argtypes
            L.orc_prove_sha512.argtypes = L.orc_prove_sha256.argtypes
            _lib = L
    return _lib


def set_threads(n: int):
    lib().orc_set_threads(n)


def ntt(a, inverse=False):
    a = np.ascontiguousarray(a, dtype=np.uint64).copy()
    assert lib().orc_ntt(_ptr(a), a.size, int(inverse)) == 0
    return a


def lde(trace: np.ndarray, blowup: int, shift: int = 1) -> np.ndarray:
    """trace: (w, n) uint64 -> (w, n*blowup)"""
    trace = np.ascontiguousarray(trace, dtype=np.uint64)
    w, n = trace.shape
    out = np.zeros((w, n * blowup), dtype=np.uint64)
    rc = lib().orc_lde(_ptr(trace), w, n, blowup, shift, _ptr(out))
    assert rc == 0, rc
    return out


def merge(air: int, lde_cols: np.ndarray, n_trace: int, blowup: int, lambdas, phi_mode=PHI_PARALLEL_GATE):
    lde_cols = np.ascontiguousarray(lde_cols, dtype=np.uint64)
    lam = np.ascontiguousarray(lambdas, dtype=np.uint64)
    out = np.zeros(n_trace * blowup, dtype=np.uint64)
    rc = lib().orc_merge(air, _ptr(lde_cols), lde_cols.shape[0], n_trace, blowup, _ptr(lam), lam.size, phi_mode,
                         _ptr(out))
    assert rc == 0, rc
    return out


def poly_div_zh(coeffs, m):
    c = np.ascontiguousarray(coeffs, dtype=np.uint64)
    q = np.zeros(max(1, c.size), dtype=np.uint64)
    k = lib().orc_poly_div_zh(_ptr(c), c.size, m, _ptr(q))
    return q[:k]


def merkle_root(rows: np.ndarray, arities, label: int) -> bytes:
    rows = np.ascontiguousarray(rows, dtype=np.uint64)
    ar = np.ascontiguousarray(arities, dtype=np.uint64)
    out = ctypes.create_string_buffer(HASH_BYTES)
    rc = lib().orc_merkle_root(_ptr(rows), rows.shape[0], rows.shape[1], _ptr(ar), ar.size, label, out)
    assert rc == 0, rc
    return out.raw


def hash_rollup_trace(leaves, n_trace):
    lv = np.ascontiguousarray(leaves, dtype=np.uint64)
    tr = np.zeros((4, n_trace), dtype=np.uint64)
    lib().orc_hash_rollup_trace(_ptr(lv), lv.size, n_trace, _ptr(tr))
    return tr


def build_params(n0: int, pi: bytes = None, stir=True) -> FriParams:
    p = FriParams()
    lib().orc_build_params(n0, pi, int(stir), ctypes.byref(p))
    return p


def stir_prove(f0: np.ndarray, params: FriParams) -> bytes:
    f0 = np.ascontiguousarray(f0, dtype=np.uint64)
    cap = 1 << 26
    buf = ctypes.create_string_buffer(cap)
    ln = ctypes.c_size_t()
    rc = lib().orc_stir_prove(_ptr(f0), f0.size, ctypes.byref(params), buf, cap, ctypes.byref(ln))
    assert rc == 0, rc
    return buf.raw[:ln.value]


def stir_verify(proof: bytes, params: FriParams) -> bool:
    return lib().orc_stir_verify(proof, len(proof), ctypes.byref(params)) == 1


def prove_hash_rollup(leaves, pi: bytes, phi_mode=PHI_PARALLEL_GATE) -> bytes:
    lv = np.ascontiguousarray(leaves, dtype=np.uint64)
    cap = 1 << 26
    buf = ctypes.create_string_buffer(cap)
    ln = ctypes.c_size_t()
    rc = lib().orc_prove_hash_rollup(_ptr(lv), lv.size, pi, phi_mode, buf, cap, ctypes.byref(ln))
    assert rc == 0, rc
    return buf.raw[:ln.value]


SHA_WIDTH, SHA_K = 756, 766
SHA_H0 = 534


def sha256_trace(msg: bytes):
    """build_sha256_trace_multi -> ((756, height) uint64, n_blocks)"""
    n_blocks_max = (len(msg) + 9 + 63) // 64
    height = 128
    while height < 128 * n_blocks_max:
        height *= 2
    out = np.zeros(SHA_WIDTH * height, dtype=np.uint64)
    h, nb = ctypes.c_size_t(), ctypes.c_size_t()
    rc = lib().orc_sha256_trace(msg, len(msg), _ptr(out), out.size, ctypes.byref(h), ctypes.byref(nb))
    assert rc == 0, rc
    return out[: SHA_WIDTH * h.value].reshape(SHA_WIDTH, h.value), nb.value


def sha256_eval(cur, nxt, row, n_blocks):
    cur = np.ascontiguousarray(cur, dtype=np.uint64)
    nxt = np.ascontiguousarray(nxt, dtype=np.uint64)
    out = np.zeros(SHA_K, dtype=np.uint64)
    lib().orc_sha256_eval(_ptr(cur), _ptr(nxt), row, n_blocks, _ptr(out))
    return out


def merge_sha256(lde_cols, n_trace, blowup, lambdas, n_blocks, phi_mode=PHI_PARALLEL_GATE):
    lde_cols = np.ascontiguousarray(lde_cols, dtype=np.uint64)
    lam = np.ascontiguousarray(lambdas, dtype=np.uint64)
    out = np.zeros(n_trace * blowup, dtype=np.uint64)
    rc = lib().orc_merge_sha256(_ptr(lde_cols), n_trace, blowup, _ptr(lam), n_blocks, phi_mode, _ptr(out))
    assert rc == 0, rc
    return out


def prove_sha256(msg: bytes, fs_binding: bytes, phi_mode=PHI_PARALLEL_GATE, blowup: int = 32):
    """prove_ds_ksk_binding core -> (proof bytes, asserted digest)"""
    cap = 1 << 26
    buf = ctypes.create_string_buffer(cap)
    ln = ctypes.c_size_t()
    dg = ctypes.create_string_buffer(32)
    rc = lib().orc_prove_sha256(msg, len(msg), fs_binding, phi_mode, blowup, buf, cap, ctypes.byref(ln), dg)
    assert rc == 0, rc
    return buf.raw[:ln.value], dg.raw


def sha3_256(msg: bytes) -> bytes:
    out = ctypes.create_string_buffer(32)
    lib().orc_sha3_256(msg, len(msg), out)
    return out.raw


def stdrng_first_u64(seed: bytes) -> int:
    return lib().orc_stdrng_first_u64(seed)


def chacha_block(key: bytes, counter: int, stream: int, rounds: int):
    out = (ctypes.c_uint32 * 16)()
    lib().orc_chacha_block(key, counter, stream, rounds, out)
    return list(out)


def fp6_mul(a, b):
    A = (ctypes.c_uint64 * 6)(*a)
    B = (ctypes.c_uint64 * 6)(*b)
    O = (ctypes.c_uint64 * 6)()
    lib().orc_fp6_mul(A, B, O)
    return list(O)


def fp6_inv(a):
    A = (ctypes.c_uint64 * 6)(*a)
    O = (ctypes.c_uint64 * 6)()
    assert lib().orc_fp6_inv(A, O) == 0
    return list(O)


SHA512_WIDTH, SHA512_K = 1510, 1526
SHA512_H0_LO = 1066


def sha512_trace(msg: bytes):
    """build_sha512_trace_multi -> ((1510, height) uint64, n_blocks)"""
    nb = (len(msg) + 17 + 127) // 128
    height = 128
    while height < 128 * nb:
        height *= 2
    out = np.zeros(SHA512_WIDTH * height, dtype=np.uint64)
    h, n = ctypes.c_size_t(), ctypes.c_size_t()
    rc = lib().orc_sha512_trace(msg, len(msg), _ptr(out), out.size, ctypes.byref(h), ctypes.byref(n))
    assert rc == 0, rc
    return out[: SHA512_WIDTH * h.value].reshape(SHA512_WIDTH, h.value), n.value


def sha512_eval(cur, nxt, row, n_blocks):
    cur = np.ascontiguousarray(cur, dtype=np.uint64)
    nxt = np.ascontiguousarray(nxt, dtype=np.uint64)
    out = np.zeros(SHA512_K, dtype=np.uint64)
    lib().orc_sha512_eval(_ptr(cur), _ptr(nxt), row, n_blocks, _ptr(out))
    return out


def merge_sha512(lde_cols, n_trace, blowup, lambdas, n_blocks, phi_mode=PHI_PARALLEL_GATE):
    lde_cols = np.ascontiguousarray(lde_cols, dtype=np.uint64)
    lam = np.ascontiguousarray(lambdas, dtype=np.uint64)
    out = np.zeros(n_trace * blowup, dtype=np.uint64)
    rc = lib().orc_merge_sha512(_ptr(lde_cols), n_trace, blowup, _ptr(lam), n_blocks, phi_mode, _ptr(out))
    assert rc == 0, rc
    return out


def prove_sha512(msg: bytes, fs_binding: bytes, phi_mode=PHI_PARALLEL_GATE, blowup: int = 32):
    """SHA-512 AIR proof -> (proof bytes, 64-byte digest read from the H-state)"""
    cap = 1 << 26
    buf = ctypes.create_string_buffer(cap)
    ln = ctypes.c_size_t()
    dg = ctypes.create_string_buffer(64)
    rc = lib().orc_prove_sha512(msg, len(msg), fs_binding, phi_mode, blowup, buf, cap, ctypes.byref(ln), dg)
    assert rc == 0, rc
    return buf.raw[:ln.value], dg.raw

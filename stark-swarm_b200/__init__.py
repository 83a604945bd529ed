"""B200 (sm_100a) drop-in for the stark-stir-swarm prover hot path.

Host-side mirror of the reference's Rust entry points (paths relative to
stark-stir-swarm/crates/), each a thin ctypes call into libstarkgpu.so whose
C ABI is declared in include/stark_gpu.h:

  lde_trace_columns      deep_ali/src/trace_import.rs:251-281
  deep_ali_merge_general deep_ali/src/lib.rs:343-437
  deep_fri_prove         deep_ali/src/fri.rs:1900-2055 (STIR and classic branches, SexticExt)
  deep_fri_verify        deep_ali/src/fri.rs:2136-2707 (STIR and classic branches)
  MerkleTreeChannel      merkle/src/lib.rs:356-512
  make_schedule / build_params / prove_hash_rollup   swarm-dns/src/prover.rs:53-304
  prove_inner_shard / prove_outer_rollup             swarm-dns/src/prover.rs:148-304
  DnsRecord::leaf_hash, merkle_build/path/verify     swarm-dns/src/dns.rs:43-131
  deep_ali_merge_sha256 / prove_sha256 (prove_ds_ksk_binding core)
                         deep_ali/src/lib.rs:453-545, swarm-dns/src/prover.rs:512-585
  deep_ali_merge_sha512  deep_ali/src/lib.rs:561-641 (and a SHA-512 proof with the same parameters)
  build_sha256_trace_multi / build_sha512_trace_multi
                         deep_ali/src/sha256_air.rs:429-472, sha512_air.rs:551-578
  prove_rsa2048 / rsa2048_trace / merge_rsa2048
                         swarm-dns/examples/prove_rsa2048_record_v1.rs, stacked_rsa_zone_prover.rs,
                         deep_ali/src/rsa2048_exp_air.rs, lib.rs:1694-2070
  prove_p256_ecdsa / p256_chain_trace / merge_p256_ecdsa
                         swarm-dns/examples/prove_ecdsa_record_v1.rs:97-240,
                         deep_ali/src/p256_ecdsa_double_multirow_air.rs, lib.rs:1421-1681
  prove_ed25519 / ed25519_trace / merge_ed25519 / prove_zsk_ksk_binding_v2
                         deep_ali/src/ed25519_verify_air.rs (v16), lib.rs:707-974,
                         swarm-dns/src/prover.rs:763-951
  Server / prove_batch   many proofs in flight on one GPU (worker loop, swarm-worker/src/main.rs:355)

The Merkle / transcript hash profile (sha3-256, sha3-384 or sha3-512: the
reference's compile-time hash feature, hash/src/selected.rs) is one library build
each, chosen per process with STARK_GPU_HASH.

Field elements are canonical uint64 (numpy uint64 arrays on the host, or CUDA
tensors / raw device pointers that the library uses in place). Errors that the
reference reports with panics or Err(String) raise exceptions here. The
library must be built (`make -C stark-swarm_b200`); there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# The hash profile is fixed per build, as the reference's hash feature is per
# compile (hash/src/selected.rs:8-48); a process picks one with STARK_GPU_HASH
# (sha3-256, the default, sha3-384 or sha3-512) before it first uses the library.
HASH_PROFILE = os.environ.get("STARK_GPU_HASH", "sha3-256")
_LIB_NAME = {"sha3-256": "libstarkgpu.so", "sha3-384": "libstarkgpu_sha3_384.so",
             "sha3-512": "libstarkgpu_sha3_512.so"}
if HASH_PROFILE not in _LIB_NAME:
    raise ValueError(f"STARK_GPU_HASH must be one of {sorted(_LIB_NAME)}")
HASH_BYTES = {"sha3-256": 32, "sha3-384": 48, "sha3-512": 64}[HASH_PROFILE]
LIB_PATH = os.path.join(_HERE, _LIB_NAME[HASH_PROFILE])
P = 0xFFFFFFFF00000001

SG_OK, SG_EINVAL, SG_ECUDA, SG_ENOMEM, SG_ESPACE, SG_EVERIFY, SG_ELIMIT = 0, -1, -2, -3, -4, -5, -6
SG_ETIMEDOUT, SG_ECANCELED = -7, -8
NOALLOC_MAX_ELEMS = 1 << 20  # sg_ntt_noalloc: n_cols * 2^log_n limit for log_n > 12
PHI_PARALLEL_GATE, PHI_ALWAYS, PHI_NEVER = 0, 1, 2
AIR_HASH_ROLLUP = 4

BLOWUP = 32
NUM_QUERIES = 54
SEED_Z = 0xDEEFBAAD


class StarkGpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class FriParams(ctypes.Structure):
    """sg_fri_params == DeepFriParams (deep_ali/src/fri.rs:1303-1314)."""
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

    @classmethod
    def new(cls, schedule, r=NUM_QUERIES, seed_z=SEED_Z, coeff_commit_final=True, d_final=1, stir=True, s0=None,
            public_inputs_hash=None):
        p = cls()
        if len(schedule) > 64:
            raise ValueError("schedule longer than 64 layers")
        for i, m in enumerate(schedule):
            p.schedule[i] = m
        p.schedule_len = len(schedule)
        p.r = r
        p.s0 = r if s0 is None else s0
        p.seed_z = seed_z
        p.d_final = d_final
        p.coeff_commit_final = int(bool(coeff_commit_final))
        p.stir = int(bool(stir))
        if public_inputs_hash is not None:
            if len(public_inputs_hash) != 32:
                raise ValueError("public_inputs_hash must be 32 bytes")
            p.has_pi = 1
            ctypes.memmove(p.pi_hash, bytes(public_inputs_hash), 32)
        return p

    @property
    def schedule_list(self):
        return [self.schedule[i] for i in range(self.schedule_len)]


DeepFriParams = FriParams

_U64P = ctypes.POINTER(ctypes.c_uint64)
_lib = None

class ProfileEntry(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 48), ("launches", ctypes.c_uint64), ("total_ms", ctypes.c_double)]


# Every symbol declared in include/stark_gpu.h.
EXPORTS = (
    "sg_ctx_create", "sg_ctx_destroy", "sg_ctx_set_stream", "sg_ctx_set_option", "sg_last_error",
    "sg_kernel_launches",
    "sg_profile_enable", "sg_profile_read", "sg_profile_reset", "sg_ntt", "sg_ntt_noalloc",
    "sg_lde", "sg_lde_commit", "sg_merge", "sg_merge_sha256", "sg_sha256_trace", "sg_sha256_trace_gpu", "sg_prove_sha256",
    "sg_merge_sha512", "sg_sha512_trace", "sg_sha512_trace_gpu", "sg_prove_sha512",
    "sg_dns_record_leaves", "sg_dns_merkle_root", "sg_dns_merkle_path", "sg_dns_merkle_verify", "sg_shard_pi_hash",
    "sg_prove_inner_shard", "sg_prove_outer_rollup",
    "sg_rsa2048_em", "sg_rsa2048_verify", "sg_rsa2048_pi_record", "sg_rsa2048_pi_stacked", "sg_rsa2048_trace",
    "sg_rsa2048_trace_gpu", "sg_merge_rsa2048", "sg_prove_rsa2048",
    "sg_p256_layout", "sg_p256_u_bits", "sg_p256_ecdsa_pi", "sg_p256_chain_trace", "sg_p256_chain_trace_gpu",
    "sg_merge_p256_ecdsa", "sg_prove_p256_chains", "sg_prove_p256_ecdsa",
    "sg_ed25519_layout", "sg_ed25519_program", "sg_ed25519_trace", "sg_ed25519_trace_gpu", "sg_merge_ed25519",
    "sg_prove_ed25519", "sg_ed25519_verify", "sg_ed25519_pi_hash", "sg_prove_zsk_ksk_binding_v2",
    "sg_merkle_commit",
    "sg_merkle_open", "sg_merkle_free", "sg_build_params", "sg_stir_prove", "sg_stir_prove_group", "sg_stir_verify", "sg_prove_hash_rollup",
    "sg_server_create", "sg_server_destroy", "sg_server_submit", "sg_server_poll", "sg_server_wait", "sg_prove_batch",
    "sg_server_wait_for", "sg_server_cancel", "sg_server_set_retries",
    "sg_pool_reserve", "sg_hash_bytes", "sg_ntt_autotune", "sg_ntt_set_split",
)
JOB_SHA256, JOB_HASH_ROLLUP, JOB_SHA512, JOB_RSA2048, JOB_P256_ECDSA, JOB_ED25519 = 1, 2, 3, 4, 5, 6
# sg_job.flags: host-side fault injection for tests of the serving loop
JOB_FAULT_ALLOC, JOB_FAULT_VERIFY = 1, 2
OPT_WIDE_MERGE = 1
OPT_STIR_GROUP = 2  # servers from this context prove up to this many same-n0 STIR phases in lockstep
WIDE_MERGE_AUTO, WIDE_MERGE_LDE, WIDE_MERGE_COSETS = 0, 1, 2


class Job(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("phi_mode", ctypes.c_int32), ("input", ctypes.c_void_p),
                ("input_len", ctypes.c_size_t), ("pi", ctypes.c_uint8 * 32), ("blowup", ctypes.c_uint32),
                ("flags", ctypes.c_uint32)]


class JobResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("reserved", ctypes.c_uint32), ("proof_len", ctypes.c_size_t),
                ("digest", ctypes.c_uint8 * 64), ("queue_ms", ctypes.c_double), ("run_ms", ctypes.c_double),
                ("latency_ms", ctypes.c_double)]
AIR_SHA256 = 6
SHA256_WIDTH, SHA256_CONSTRAINTS = 756, 766
SHA512_WIDTH, SHA512_CONSTRAINTS = 1510, 1526
# per hash AIR: width, constraints, digest bytes, block bytes, padding overhead (0x80 + length field)
_HASH = {"sha256": (SHA256_WIDTH, SHA256_CONSTRAINTS, 32, 64, 9),
         "sha512": (SHA512_WIDTH, SHA512_CONSTRAINTS, 64, 128, 17)}


def _trace_height(hash_name: str, message: bytes) -> int:
    _, _, _, block, pad = _HASH[hash_name]
    nb = (len(message) + pad + block - 1) // block
    height = 128
    while height < 128 * nb:
        height *= 2
    return height


def lib():
    """Load libstarkgpu.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C {_HERE} all`")
    L = ctypes.CDLL(LIB_PATH)
    L.sg_hash_bytes.restype = ctypes.c_int
    if L.sg_hash_bytes() != HASH_BYTES:
        raise ImportError(f"{LIB_PATH} is not a {HASH_PROFILE} build")
    vp, sz, u64, i32 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_int
    L.sg_ctx_create.argtypes = [i32, ctypes.POINTER(vp)]
    L.sg_ctx_destroy.argtypes = [vp]
    L.sg_ctx_destroy.restype = None
    L.sg_ctx_set_stream.argtypes = [vp, vp]
    L.sg_ctx_set_option.argtypes = [vp, i32, ctypes.c_int64]
    L.sg_pool_reserve.argtypes = [vp, u64]
    L.sg_ntt_autotune.argtypes = [vp, sz, sz, i32, sz, ctypes.POINTER(ctypes.c_int)]
    L.sg_ntt_set_split.argtypes = [sz, i32, i32]
    L.sg_last_error.argtypes = [vp]
    L.sg_last_error.restype = ctypes.c_char_p
    L.sg_kernel_launches.argtypes = [vp]
    L.sg_kernel_launches.restype = u64
    L.sg_profile_enable.argtypes = [i32]
    L.sg_profile_read.argtypes = [ctypes.POINTER(ProfileEntry), sz, ctypes.POINTER(sz)]
    L.sg_profile_reset.argtypes = []
    L.sg_profile_reset.restype = None
    L.sg_ntt.argtypes = [vp, vp, vp, sz, sz, i32]
    L.sg_ntt_noalloc.argtypes = [vp, vp, sz, sz, i32, vp]
    L.sg_lde.argtypes = [vp, vp, sz, sz, sz, u64, vp]
    L.sg_merge.argtypes = [vp, i32, vp, sz, sz, sz, vp, sz, i32, vp]
    L.sg_merge_sha256.argtypes = [vp, vp, sz, sz, vp, sz, i32, vp]
    L.sg_server_create.argtypes = [vp, i32, u64, ctypes.POINTER(vp)]
    L.sg_server_destroy.argtypes = [vp]
    L.sg_server_destroy.restype = None
    L.sg_server_submit.argtypes = [vp, ctypes.POINTER(Job), ctypes.POINTER(u64)]
    L.sg_server_poll.argtypes = [vp, u64]
    L.sg_server_wait.argtypes = [vp, u64, ctypes.POINTER(JobResult), ctypes.c_char_p, sz]
    L.sg_server_wait_for.argtypes = [vp, u64, ctypes.c_int64, ctypes.POINTER(JobResult), ctypes.c_char_p, sz]
    L.sg_server_cancel.argtypes = [vp, u64]
    L.sg_server_set_retries.argtypes = [vp, i32]
    L.sg_prove_batch.argtypes = [vp, ctypes.POINTER(Job), sz, i32, u64, ctypes.c_char_p, sz,
                                 ctypes.POINTER(JobResult)]
    L.sg_sha256_trace.argtypes = [ctypes.c_char_p, sz, vp, sz, ctypes.POINTER(sz), ctypes.POINTER(sz),
                                  ctypes.c_char_p]
    L.sg_sha256_trace_gpu.argtypes = [vp] + L.sg_sha256_trace.argtypes
    L.sg_prove_sha256.argtypes = [vp, ctypes.c_char_p, sz, ctypes.c_char_p, i32, ctypes.c_char_p, sz,
                                  ctypes.POINTER(sz), ctypes.c_char_p]
    L.sg_dns_record_leaves.argtypes = [ctypes.c_char_p, ctypes.POINTER(sz), sz, ctypes.c_char_p, ctypes.c_char_p]
    L.sg_dns_merkle_root.argtypes = [ctypes.c_char_p, sz, ctypes.c_char_p]
    L.sg_dns_merkle_path.argtypes = [ctypes.c_char_p, sz, sz, ctypes.c_char_p, sz, ctypes.POINTER(sz)]
    L.sg_dns_merkle_verify.argtypes = [ctypes.c_char_p, sz, ctypes.c_char_p, sz, ctypes.c_char_p]
    L.sg_shard_pi_hash.argtypes = [ctypes.c_char_p, u64, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                   ctypes.c_char_p]
    L.sg_shard_pi_hash.restype = None
    L.sg_prove_inner_shard.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(sz), sz, ctypes.c_char_p, ctypes.c_char_p,
                                       i32, ctypes.c_char_p, sz, ctypes.POINTER(sz), ctypes.c_char_p, ctypes.c_char_p]
    L.sg_prove_outer_rollup.argtypes = [vp, ctypes.c_char_p, sz, ctypes.c_char_p, i32, ctypes.c_char_p, sz,
                                        ctypes.POINTER(sz)]
    L.sg_rsa2048_em.argtypes = [ctypes.c_char_p, sz, ctypes.c_char_p]
    L.sg_rsa2048_verify.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p]
    L.sg_rsa2048_pi_record.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, sz, ctypes.c_char_p,
                                       ctypes.c_char_p]
    L.sg_rsa2048_pi_stacked.argtypes = [ctypes.c_char_p, sz, ctypes.c_char_p, ctypes.c_char_p]
    L.sg_rsa2048_trace.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, sz, vp, sz]
    L.sg_rsa2048_trace_gpu.argtypes = [vp] + L.sg_rsa2048_trace.argtypes
    L.sg_merge_rsa2048.argtypes = [vp, vp, sz, sz, sz, vp]
    L.sg_prove_rsa2048.argtypes = [vp, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, sz, ctypes.c_char_p,
                                   ctypes.c_char_p, sz, ctypes.POINTER(sz)]
    cp = ctypes.c_char_p
    L.sg_p256_layout.argtypes = [ctypes.POINTER(ctypes.c_uint32)] * 3 + [vp, sz, vp]
    L.sg_p256_u_bits.argtypes = [cp, cp, cp, cp, cp]
    L.sg_p256_ecdsa_pi.argtypes = [cp, cp, cp, cp, cp, cp]
    L.sg_p256_chain_trace.argtypes = [cp, cp, cp, cp, cp, cp, sz, vp, sz]
    L.sg_p256_chain_trace_gpu.argtypes = [vp] + L.sg_p256_chain_trace.argtypes
    L.sg_merge_p256_ecdsa.argtypes = [vp, vp, sz, sz, vp]
    L.sg_prove_p256_chains.argtypes = [vp, cp, cp, cp, cp, cp, cp, sz, cp, cp, sz, ctypes.POINTER(sz)]
    L.sg_prove_p256_ecdsa.argtypes = [vp, cp, cp, cp, cp, cp, cp, cp, sz, ctypes.POINTER(sz)]
    u32 = ctypes.c_uint32
    u32p = ctypes.POINTER(u32)
    L.sg_ed25519_layout.argtypes = [u32, sz, u32p, u32p, u32p, vp]
    L.sg_ed25519_program.argtypes = [cp, cp, cp, sz, u32, vp, sz, ctypes.POINTER(sz), vp, sz, ctypes.POINTER(sz)]
    L.sg_ed25519_trace.argtypes = [cp, cp, cp, sz, u32, vp, sz]
    L.sg_ed25519_trace_gpu.argtypes = [vp] + L.sg_ed25519_trace.argtypes
    L.sg_merge_ed25519.argtypes = [vp, cp, cp, cp, sz, u32, vp, sz, vp]
    L.sg_prove_ed25519.argtypes = [vp, cp, cp, cp, sz, cp, u32, sz, cp, sz, ctypes.POINTER(sz)]
    L.sg_ed25519_verify.argtypes = [cp, cp, cp, sz]
    L.sg_ed25519_pi_hash.argtypes = [cp, cp, cp, sz, cp, cp, cp, cp]
    L.sg_prove_zsk_ksk_binding_v2.argtypes = [vp, cp, cp, cp, sz, cp, cp, u32, cp, sz, ctypes.POINTER(sz), cp]
    L.sg_merge_sha512.argtypes = L.sg_merge_sha256.argtypes
    L.sg_sha512_trace.argtypes = L.sg_sha256_trace.argtypes
    L.sg_sha512_trace_gpu.argtypes = L.sg_sha256_trace_gpu.argtypes
    L.sg_prove_sha512.argtypes = L.sg_prove_sha256.argtypes
    L.sg_merkle_commit.argtypes = [vp, vp, sz, sz, sz, vp, sz, u64, ctypes.c_char_p, ctypes.POINTER(vp)]
    L.sg_lde_commit.argtypes = [vp, vp, sz, sz, sz, u64, vp, sz, u64, ctypes.c_char_p, vp, sz, ctypes.POINTER(vp)]
    L.sg_merkle_open.argtypes = [vp, vp, sz, ctypes.c_char_p, sz, ctypes.POINTER(sz)]
    L.sg_merkle_free.argtypes = [vp]
    L.sg_merkle_free.restype = None
    L.sg_build_params.argtypes = [sz, ctypes.c_char_p, i32, ctypes.POINTER(FriParams)]
    L.sg_build_params.restype = None
    L.sg_stir_prove.argtypes = [vp, vp, sz, ctypes.POINTER(FriParams), ctypes.c_char_p, sz, ctypes.POINTER(sz)]
    L.sg_stir_prove_group.argtypes = [vp, vp, sz, sz, ctypes.POINTER(FriParams), ctypes.c_char_p, sz,
                                      ctypes.POINTER(sz)]
    L.sg_stir_verify.argtypes = [ctypes.c_char_p, sz, ctypes.POINTER(FriParams)]
    L.sg_prove_hash_rollup.argtypes = [vp, vp, sz, ctypes.c_char_p, i32, ctypes.c_char_p, sz, ctypes.POINTER(sz)]
    _lib = L
    return L


_PROOF_CAP = 1 << 24  # proof buffer size; untouched pages of np.empty cost nothing, a larger proof is retried


def _out_buffer(cap):
    """An uninitialised byte buffer for a C call to write into: (numpy array, char pointer).
    Only the prefix the call reports as written is read back, so nothing is zero-filled
    or copied beyond the proof itself."""
    arr = np.empty(max(1, cap), dtype=np.uint8)
    return arr, ctypes.cast(arr.ctypes.data, ctypes.c_char_p)


def _addr(x):
    """(pointer, keepalive, is_numpy) for a numpy uint64 array, a CUDA tensor or an int device pointer."""
    if isinstance(x, np.ndarray):
        if x.dtype != np.uint64:
            raise TypeError("host buffers must be numpy uint64")
        if not x.flags["C_CONTIGUOUS"]:
            raise ValueError("host buffers must be C-contiguous")
        return x.ctypes.data, x, True
    if hasattr(x, "data_ptr"):
        if not x.is_contiguous():
            raise ValueError("tensors must be contiguous")
        if x.element_size() != 8:
            raise TypeError("tensors must hold 64-bit elements")
        return x.data_ptr(), x, False
    if isinstance(x, int):
        return x, None, False
    raise TypeError(f"unsupported buffer type {type(x)!r}")


def make_schedule(n0: int, stir: bool = True):
    """swarm-dns/src/prover.rs:53-67"""
    if n0 <= 0 or n0 & (n0 - 1):
        raise ValueError("n0 must be a power of 2")
    lg = n0.bit_length() - 1
    if not stir:
        return [2] * lg
    s = [8] * (lg // 3)
    if lg % 3:
        s.append(1 << (lg % 3))
    return s


def build_params(n0: int, pk_hash_32: bytes = None, stir: bool = True) -> FriParams:
    """swarm-dns/src/prover.rs:89-98"""
    p = FriParams()
    lib().sg_build_params(n0, pk_hash_32, int(stir), ctypes.byref(p))
    return p


def ntt_set_split(log_n: int, padded: bool, log_n1: int):
    """sg_ntt_set_split: pin the four-step split of 2^log_n transforms (0 = default)."""
    rc = lib().sg_ntt_set_split(log_n, int(padded), log_n1)
    if rc != SG_OK:
        raise StarkGpuError(rc, "sg_ntt_set_split: size or split out of range")


def profile_enable(on: bool = True):
    lib().sg_profile_enable(int(on))


def profile_reset():
    lib().sg_profile_reset()


def profile_read():
    """{kernel family: (launches, total device ms)} since the last reset."""
    arr = (ProfileEntry * 64)()
    n = ctypes.c_size_t()
    lib().sg_profile_read(arr, 64, ctypes.byref(n))
    return {arr[i].name.decode(): (arr[i].launches, arr[i].total_ms) for i in range(min(n.value, 64))}


def ntt_noalloc(d_in, d_out, log_n: int, inverse: bool = False, stream_ptr: int = 0, n_cols: int = None) -> int:
    """sg_ntt_noalloc on device buffers, for callers that must not let the library
    allocate device memory. `d_in` / `d_out` are CUDA tensors of 64-bit elements
    holding n_cols columns of 2^log_n (a tensor's element count fixes n_cols), or
    raw device pointers, in which case `n_cols` must be given. Sizes are checked
    here before anything reaches the device: a buffer shorter than one column,
    an element count that is not a whole number of columns, or an output
    shorter than the input raises ValueError. Returns the SG_* code; the
    transform is ordered on `stream_ptr` (0 = the legacy default stream)."""
    if not 0 <= log_n <= 28:
        raise ValueError("log_n must be in [0, 28]")
    n = 1 << log_n
    ip, _ki, host_in = _addr(d_in)
    op, _ko, host_out = _addr(d_out)
    if host_in or host_out:
        raise ValueError("sg_ntt_noalloc takes device buffers, not host arrays")
    counts = [x.numel() if hasattr(x, "numel") else None for x in (d_in, d_out)]
    if counts[0] is not None:
        if counts[0] < n or counts[0] % n:
            raise ValueError(f"input holds {counts[0]} elements, not a whole number of 2^{log_n}-point columns")
        cols = counts[0] // n
        if n_cols is not None and n_cols != cols:
            raise ValueError(f"n_cols={n_cols} but the input holds {cols} columns")
    elif n_cols is None:
        raise ValueError("a raw device pointer needs an explicit n_cols")
    else:
        cols = n_cols
    if cols < 1:
        raise ValueError("n_cols must be at least 1")
    for c in counts:
        if c is not None and c < cols * n:
            raise ValueError(f"a buffer holds {c} elements, fewer than n_cols * 2^log_n = {cols * n}")
    return lib().sg_ntt_noalloc(ip, op, cols, log_n, int(inverse), stream_ptr or None)


def _build_trace_multi(hash_name: str, message: bytes):
    width, _, dbytes, _, _ = _HASH[hash_name]
    height = _trace_height(hash_name, message)
    out = np.zeros(width * height, dtype=np.uint64)
    h, n = ctypes.c_size_t(), ctypes.c_size_t()
    dg = ctypes.create_string_buffer(dbytes)
    fn = getattr(lib(), f"sg_{hash_name}_trace")
    rc = fn(message, len(message), out.ctypes.data, out.size, ctypes.byref(h), ctypes.byref(n), dg)
    if rc != SG_OK:
        raise StarkGpuError(rc, f"sg_{hash_name}_trace failed")
    return out[: width * h.value].reshape(width, h.value), n.value, dg.raw


def build_sha256_trace_multi(message: bytes):
    """sha256_air.rs:429-472 on the host -> ((756, height) uint64 trace, n_blocks, asserted digest)."""
    return _build_trace_multi("sha256", message)


def build_sha512_trace_multi(message: bytes):
    """sha512_air.rs:551-578 on the host -> ((1510, height) uint64 trace, n_blocks, 64-byte digest)."""
    return _build_trace_multi("sha512", message)


RSA_WIDTH, RSA_CONSTRAINTS, RSA_N_TRACE, RSA_BLOWUP = 11041, 11280, 32, 32


def _be256(x) -> bytes:
    """an int or a 256-byte big-endian string -> 256 bytes"""
    if isinstance(x, int):
        return x.to_bytes(256, "big")
    b = bytes(x)
    if len(b) != 256:
        raise ValueError("RSA-2048 values are 256-byte big-endian strings")
    return b


def rsa2048_em(message: bytes) -> bytes:
    """EMSA-PKCS1-v1_5 of SHA-256(message) for a 256-byte modulus (deep_ali/src/rsa2048.rs:71-90)."""
    em = ctypes.create_string_buffer(256)
    rc = lib().sg_rsa2048_em(message, len(message), em)
    if rc != SG_OK:
        raise StarkGpuError(rc, "sg_rsa2048_em failed")
    return em.raw


def rsa2048_verify(n, s, em) -> bool:
    """Native RSASSA-PKCS1-v1_5 check s^65537 mod n == em (deep_ali/src/rsa2048.rs:92-127)."""
    return lib().sg_rsa2048_verify(_be256(n), _be256(s), _be256(em)) == 1


def rsa2048_pi_record(n, s, message: bytes, em) -> bytes:
    """pi_hash of one RSA record (prove_rsa2048_record_v1.rs:178-187)."""
    out = ctypes.create_string_buffer(32)
    rc = lib().sg_rsa2048_pi_record(_be256(n), _be256(s), message, len(message), _be256(em), out)
    if rc != SG_OK:
        raise StarkGpuError(rc, "sg_rsa2048_pi_record failed")
    return out.raw


def rsa2048_pi_stacked(n, ems) -> bytes:
    """pi_hash of a stacked zone under one modulus (stacked_rsa_zone_prover.rs:158-165)."""
    out = ctypes.create_string_buffer(32)
    blob = b"".join(_be256(e) for e in ems)
    rc = lib().sg_rsa2048_pi_stacked(_be256(n), len(ems), blob, out)
    if rc != SG_OK:
        raise StarkGpuError(rc, "sg_rsa2048_pi_stacked failed")
    return out.raw


def _rsa_records(records):
    """[(n, s, em)] (ints or 256-byte strings) -> concatenated n, s, em arrays"""
    if not records:
        raise ValueError("need at least one RSA record")
    ns = b"".join(_be256(r[0]) for r in records)
    ss = b"".join(_be256(r[1]) for r in records)
    es = b"".join(_be256(r[2]) for r in records)
    return ns, ss, es


def rsa2048_trace(records) -> np.ndarray:
    """fill_rsa_exp_multirow / fill_rsa_stacked on the host -> (len(records) * 11041, 32) uint64."""
    ns, ss, es = _rsa_records(records)
    out = np.empty(len(records) * RSA_WIDTH * RSA_N_TRACE, dtype=np.uint64)
    rc = lib().sg_rsa2048_trace(ns, ss, es, len(records), out.ctypes.data, out.size)
    if rc != SG_OK:
        raise StarkGpuError(rc, "sg_rsa2048_trace failed")
    return out.reshape(len(records) * RSA_WIDTH, RSA_N_TRACE)


P256_BLOWUP = 32


def _be32(x) -> bytes:
    if isinstance(x, int):
        return x.to_bytes(32, "big")
    b = bytes(x)
    if len(b) != 32:
        raise ValueError("P-256 values are 32-byte big-endian strings")
    return b


def _bits(bits) -> bytes:
    return bytes(1 if b else 0 for b in bits)


def p256_layout():
    """-> (width, constraints per row, (n_gadgets, 8) uint32 table, 18 tail bases)."""
    L = lib()
    w, g, k = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
    rc = L.sg_p256_layout(ctypes.byref(w), ctypes.byref(g), ctypes.byref(k), None, 0, None)
    if rc != SG_OK:
        raise StarkGpuError(rc, "sg_p256_layout failed")
    table = np.zeros((g.value, 8), dtype=np.uint32)
    tail = np.zeros(18, dtype=np.uint32)
    rc = L.sg_p256_layout(ctypes.byref(w), ctypes.byref(g), ctypes.byref(k), table.ctypes.data, g.value,
                          tail.ctypes.data)
    if rc != SG_OK:
        raise StarkGpuError(rc, "sg_p256_layout failed")
    return w.value, k.value, table, tail


def p256_u_bits(digest: bytes, r, s):
    """u1 = e s^-1, u2 = r s^-1 mod n as MSB-first bit lists (prove_ecdsa_record_v1.rs:97-118)."""
    u1, u2 = ctypes.create_string_buffer(256), ctypes.create_string_buffer(256)
    rc = lib().sg_p256_u_bits(_be32(digest), _be32(r), _be32(s), u1, u2)
    if rc != SG_OK:
        raise StarkGpuError(rc, "sg_p256_u_bits failed")
    return list(u1.raw), list(u2.raw)


def p256_ecdsa_pi(qx, qy, r, s, digest: bytes) -> bytes:
    """pi_hash of prove_ecdsa_record_v1.rs:213-222."""
    out = ctypes.create_string_buffer(32)
    rc = lib().sg_p256_ecdsa_pi(_be32(qx), _be32(qy), _be32(r), _be32(s), _be32(digest), out)
    if rc != SG_OK:
        raise StarkGpuError(rc, "sg_p256_ecdsa_pi failed")
    return out.raw


def p256_chain_trace(a_point, a_bits, b_point, b_bits) -> np.ndarray:
    """fill_ecdsa_double_multirow on the host: chains from (x, y, 1) of two affine
    points, one bit per row -> (151334, len(bits)) uint64."""
    k = len(a_bits)
    width = p256_layout()[0]
    out = np.empty(width * k, dtype=np.uint64)
    rc = lib().sg_p256_chain_trace(_be32(a_point[0]), _be32(a_point[1]), _bits(a_bits), _be32(b_point[0]),
                                   _be32(b_point[1]), _bits(b_bits), k, out.ctypes.data, out.size)
    if rc != SG_OK:
        raise StarkGpuError(rc, "sg_p256_chain_trace failed")
    return out.reshape(width, k)


ED25519_K = 256
ED25519_BLOWUP = 32


def _ed_args(pub, sig, msg):
    pub, sig, msg = bytes(pub), bytes(sig), bytes(msg)
    if len(pub) != 32 or len(sig) != 64:
        raise ValueError("Ed25519 keys are 32 bytes and signatures 64 bytes (R || S)")
    return pub, sig, msg


def ed25519_layout(msg_len: int, k_scalar: int = ED25519_K):
    """verify_air_layout_v16 -> (width, height, constraints per row, dict of phase rows)."""
    w, h, k = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
    rows = (ctypes.c_uint32 * 11)()
    rc = lib().sg_ed25519_layout(k_scalar, msg_len, ctypes.byref(w), ctypes.byref(h), ctypes.byref(k), rows)
    if rc != SG_OK:
        raise StarkGpuError(rc, "sg_ed25519_layout failed")
    names = ("k_hash", "reduce_row", "decompress_R_row", "decompress_A_row", "sB_first_row", "kA_first_row",
             "residual_row", "dbl_1_row", "dbl_2_row", "dbl_3_row", "result_row")
    return w.value, h.value, k.value, dict(zip(names, list(rows)))


def ed25519_program(pub: bytes, sig: bytes, msg: bytes, k_scalar: int = ED25519_K):
    """The row's constraint program -> ((n_blocks, 16) uint64 records, (n_pairs, 2) uint64 pairs)."""
    pub, sig, msg = _ed_args(pub, sig, msg)
    L = lib()
    nr, npr = ctypes.c_size_t(), ctypes.c_size_t()
    rc = L.sg_ed25519_program(pub, sig, msg, len(msg), k_scalar, None, 0, ctypes.byref(nr), None, 0,
                              ctypes.byref(npr))
    if rc != SG_OK:
        raise StarkGpuError(rc, "sg_ed25519_program failed")
    recs = np.zeros((nr.value, 16), dtype=np.uint64)
    pairs = np.zeros((npr.value, 2), dtype=np.uint64)
    rc = L.sg_ed25519_program(pub, sig, msg, len(msg), k_scalar, recs.ctypes.data, nr.value, ctypes.byref(nr),
                              pairs.ctypes.data, npr.value, ctypes.byref(npr))
    if rc != SG_OK:
        raise StarkGpuError(rc, "sg_ed25519_program failed")
    return recs, pairs


def ed25519_trace(pub: bytes, sig: bytes, msg: bytes, k_scalar: int = ED25519_K) -> np.ndarray:
    """fill_verify_air_v16 on the host -> (width, height) uint64."""
    pub, sig, msg = _ed_args(pub, sig, msg)
    w, h, _k, _r = ed25519_layout(len(msg), k_scalar)
    out = np.empty(w * h, dtype=np.uint64)
    rc = lib().sg_ed25519_trace(pub, sig, msg, len(msg), k_scalar, out.ctypes.data, out.size)
    if rc != SG_OK:
        raise StarkGpuError(rc, "sg_ed25519_trace failed")
    return out.reshape(w, h)


def ed25519_verify(pub: bytes, sig: bytes, msg: bytes) -> bool:
    """RFC 8032 cofactored verification (ed25519_verify.rs:54-117)."""
    pub, sig, msg = _ed_args(pub, sig, msg)
    rc = lib().sg_ed25519_verify(pub, sig, msg, len(msg))
    if rc < 0:
        raise StarkGpuError(rc, "sg_ed25519_verify failed")
    return rc == 1


def ed25519_pi_hash(pub: bytes, sig: bytes, msg: bytes, fs_binding: bytes, merkle_root: bytes,
                    root_f0: bytes) -> bytes:
    """zsk_ksk_pi_hash_v2_stark (swarm-dns/src/prover.rs:763-780)."""
    pub, sig, msg = _ed_args(pub, sig, msg)
    if len(fs_binding) != 32 or len(merkle_root) != 32 or len(root_f0) != 32:
        raise ValueError("fs_binding, merkle_root and root_f0 are 32 bytes")
    out = ctypes.create_string_buffer(32)
    rc = lib().sg_ed25519_pi_hash(pub, sig, msg, len(msg), fs_binding, merkle_root, root_f0, out)
    if rc != SG_OK:
        raise StarkGpuError(rc, "sg_ed25519_pi_hash failed")
    return out.raw


def _records(records):
    """canonical record byte strings -> (concatenated bytes, offsets[n+1])"""
    recs = [bytes(r) for r in records]
    offs = (ctypes.c_size_t * (len(recs) + 1))()
    o = 0
    for i, r in enumerate(recs):
        offs[i] = o
        o += len(r)
    offs[len(recs)] = o
    return b"".join(recs), offs


def dns_record_leaves(records, salt: bytes):
    """DnsRecord::leaf_hash (swarm-dns/src/dns.rs:56-79) of canonical records -> list of 32-byte hashes."""
    if len(salt) != 16:
        raise ValueError("salt must be 16 bytes")
    canon, offs = _records(records)
    out = ctypes.create_string_buffer(32 * max(1, len(records)))
    rc = lib().sg_dns_record_leaves(canon, offs, len(records), salt, out)
    if rc != SG_OK:
        raise StarkGpuError(rc, "sg_dns_record_leaves failed")
    return [out.raw[32 * i: 32 * i + 32] for i in range(len(records))]


def dns_merkle_root(leaves) -> bytes:
    """merkle_build + merkle_root (swarm-dns/src/dns.rs:85-102)."""
    root = ctypes.create_string_buffer(32)
    rc = lib().sg_dns_merkle_root(b"".join(leaves), len(leaves), root)
    if rc != SG_OK:
        raise StarkGpuError(rc, "sg_dns_merkle_root failed")
    return root.raw


def dns_merkle_path(leaves, index: int):
    """merkle_path (swarm-dns/src/dns.rs:104-114) -> list of 32-byte siblings."""
    cap = 32 * 64
    path = ctypes.create_string_buffer(cap)
    depth = ctypes.c_size_t()
    rc = lib().sg_dns_merkle_path(b"".join(leaves), len(leaves), index, path, cap, ctypes.byref(depth))
    if rc != SG_OK:
        raise StarkGpuError(rc, "sg_dns_merkle_path failed")
    return [path.raw[32 * i: 32 * i + 32] for i in range(depth.value)]


def dns_merkle_verify(leaf: bytes, index: int, path, root: bytes) -> bool:
    """merkle_verify (swarm-dns/src/dns.rs:116-131)."""
    return lib().sg_dns_merkle_verify(leaf, index, b"".join(path), len(path), root) == 1


def shard_pi_hash(salt: bytes, record_count: int, merkle_root: bytes, root_f0: bytes, fs_binding: bytes) -> bytes:
    """Inner-shard pi_hash (swarm-dns/src/prover.rs:207-214)."""
    out = ctypes.create_string_buffer(32)
    lib().sg_shard_pi_hash(salt, record_count, merkle_root, root_f0, fs_binding, out)
    return out.raw


def deep_fri_verify(params: FriParams, proof: bytes) -> bool:
    """STIR verifier on serialized proof bytes (host code; needs no GPU)."""
    return lib().sg_stir_verify(proof, len(proof), ctypes.byref(params)) == 1


class FriDomain:
    """fri.rs:161-169: the radix-2 domain of size n with ark-poly's generator."""

    def __init__(self, size: int):
        if size <= 0 or size & (size - 1):
            raise ValueError("radix-2 domain size must be a power of 2")
        self.size = size
        lg = size.bit_length() - 1
        r = pow(7, (P - 1) >> 32, P)
        for _ in range(32 - lg):
            r = r * r % P
        self.omega = r

    @classmethod
    def new_radix2(cls, size: int):
        return cls(size)


class Context:
    """One CUDA device + stream + twiddle tables (sg_ctx)."""

    def __init__(self, device: int = 0):
        self._lib = lib()
        h = ctypes.c_void_p()
        rc = self._lib.sg_ctx_create(device, ctypes.byref(h))
        if rc != SG_OK:
            raise StarkGpuError(rc, f"sg_ctx_create(device={device}) failed")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.sg_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc):
        if rc != SG_OK:
            raise StarkGpuError(rc, self._lib.sg_last_error(self._h).decode())

    def set_stream(self, stream_ptr: int = 0):
        self._check(self._lib.sg_ctx_set_stream(self._h, stream_ptr or None))

    def set_option(self, option: int, value: int):
        self._check(self._lib.sg_ctx_set_option(self._h, option, value))

    def ntt_autotune(self, n_cols: int, log_n: int, inverse: bool = False, n_valid: int = 0) -> int:
        """sg_ntt_autotune: measure the four-step splits of a 2^13..2^24 transform
        (zero-padded beyond n_valid when given) and keep the fastest; returns its log N1."""
        best = ctypes.c_int()
        self._check(self._lib.sg_ntt_autotune(self._h, n_cols, log_n, int(inverse), n_valid, ctypes.byref(best)))
        return best.value

    def pool_reserve(self, nbytes: int):
        """sg_pool_reserve: grow the device memory pool to nbytes up front (best effort)."""
        self._check(self._lib.sg_pool_reserve(self._h, nbytes))

    @property
    def kernel_launches(self) -> int:
        return self._lib.sg_kernel_launches(self._h)

    # ---------------------------------------------------------------- NTT / LDE
    def ntt(self, data, log_n: int, inverse: bool = False, out=None):
        """Batched ark-poly fft/ifft over the columns of a (cols, 2^log_n) buffer."""
        ip, _ki, host = _addr(data)
        n = 1 << log_n
        if out is None:
            if not host:
                raise ValueError("device input needs an explicit out buffer")
            out = np.empty_like(data)
        op, _ko, _ = _addr(out)
        cols = (data.size if host else data.numel()) // n
        self._check(self._lib.sg_ntt(self._h, ip, op, cols, log_n, int(inverse)))
        return out

    def lde_commit(self, trace, blowup: int, shift: int, arities, tree_label: int, keep_cols: int = 0, out=None,
                   keep=False):
        """lde_trace_columns then the Merkle commitment to the LDE's rows, in one call
        (sg_lde_commit): returns the root, plus the first keep_cols LDE columns (a new
        (keep_cols, n0) array unless `out` is given) and the tree handle if keep."""
        ip, _ki, host = _addr(trace)
        w, n = trace.shape
        n0 = n * blowup
        if keep_cols and out is None:
            out = np.empty((keep_cols, n0), dtype=np.uint64)
        op = _addr(out)[0] if keep_cols else None
        ar = np.ascontiguousarray(arities, dtype=np.uint64)
        root = ctypes.create_string_buffer(HASH_BYTES)
        t = ctypes.c_void_p()
        self._check(self._lib.sg_lde_commit(self._h, ip, w, n, blowup, shift, ar.ctypes.data, ar.size, tree_label, root,
                                            op, keep_cols, ctypes.byref(t) if keep else None))
        res = [root.raw]
        if keep_cols:
            res.append(out)
        if keep:
            res.append(MerkleTree(self, t))
        return res[0] if len(res) == 1 else tuple(res)

    def lde(self, trace, blowup: int, shift: int = 1, out=None):
        """lde_trace_columns on a (w, n_trace) column-major buffer -> (w, n_trace*blowup)."""
        ip, _ki, host = _addr(trace)
        w, n = trace.shape
        if out is None:
            if not host:
                raise ValueError("device input needs an explicit out buffer")
            out = np.empty((w, n * blowup), dtype=np.uint64)
        op, _ko, _ = _addr(out)
        self._check(self._lib.sg_lde(self._h, ip, w, n, blowup, shift, op))
        return out

    def lde_trace_columns(self, columns, trace_len: int, blowup: int):
        """Reference signature: list of columns -> list of LDE columns (raises ValueError like Err(String))."""
        if len(columns) == 0:
            raise ValueError("no columns provided")
        for i, col in enumerate(columns):
            if len(col) != trace_len:
                raise ValueError(f"column {i}: expected {trace_len} rows, got {len(col)}")
        if trace_len & (trace_len - 1) or trace_len == 0:
            raise ValueError(f"trace_len {trace_len} must be a power of 2")
        if blowup < 2 or blowup & (blowup - 1):
            raise ValueError(f"blowup {blowup} must be a power-of-2 >= 2")
        tr = np.ascontiguousarray(np.array(columns, dtype=np.uint64) % np.uint64(P))
        return list(self.lde(tr, blowup))

    # ---------------------------------------------------------------- merge
    def merge(self, air: int, lde, n_trace: int, blowup: int, lambdas, phi_mode=PHI_PARALLEL_GATE, out=None):
        ip, _ki, host = _addr(lde)
        w = lde.shape[0]
        lam = np.ascontiguousarray(lambdas, dtype=np.uint64)
        n = n_trace * blowup
        if out is None:
            if not host:
                raise ValueError("device input needs an explicit out buffer")
            out = np.empty(n, dtype=np.uint64)
        op, _ko, _ = _addr(out)
        self._check(self._lib.sg_merge(self._h, air, ip, w, n_trace, blowup, lam.ctypes.data, lam.size, phi_mode,
                                       op))
        return out

    def _hash_trace(self, hash_name: str, message: bytes, out=None):
        width, _, dbytes, _, _ = _HASH[hash_name]
        height = _trace_height(hash_name, message)
        if out is None:
            out = np.empty((width, height), dtype=np.uint64)
        op, _ko, _ = _addr(out)
        h, n = ctypes.c_size_t(), ctypes.c_size_t()
        dg = ctypes.create_string_buffer(dbytes)
        fn = getattr(self._lib, f"sg_{hash_name}_trace_gpu")
        self._check(fn(self._h, message, len(message), op, width * height, ctypes.byref(h), ctypes.byref(n), dg))
        return out, n.value, dg.raw

    def _merge_hash(self, hash_name, lde, n_trace, blowup, lambdas, n_blocks, phi_mode, out):
        _, k, _, _, _ = _HASH[hash_name]
        ip, _ki, host = _addr(lde)
        lam = np.ascontiguousarray(lambdas, dtype=np.uint64)
        if lam.size != k:
            raise ValueError(f"need one combination coefficient per constraint ({k})")
        n = n_trace * blowup
        if out is None:
            if not host:
                raise ValueError("device input needs an explicit out buffer")
            out = np.empty(n, dtype=np.uint64)
        op, _ko, _ = _addr(out)
        fn = getattr(self._lib, f"sg_merge_{hash_name}")
        self._check(fn(self._h, ip, n_trace, blowup, lam.ctypes.data, n_blocks, phi_mode, op))
        return out

    def _prove_hash(self, hash_name, message, fs_binding, phi_mode):
        if len(fs_binding) != 32:
            raise ValueError("fs_binding must be 32 bytes")
        dbytes = _HASH[hash_name][2]
        fn = getattr(self._lib, f"sg_prove_{hash_name}")
        cap = _PROOF_CAP
        while True:
            arr, buf = _out_buffer(cap)
            ln = ctypes.c_size_t()
            dg = ctypes.create_string_buffer(dbytes)
            rc = fn(self._h, message, len(message), fs_binding, phi_mode, buf, cap, ctypes.byref(ln), dg)
            if rc == SG_ESPACE:
                cap = ln.value
                continue
            self._check(rc)
            return arr[:ln.value].tobytes(), dg.raw

    def sha256_trace(self, message: bytes, out=None):
        """build_sha256_trace_multi with the column expansion on the GPU ->
        ((756, height) trace, n_blocks, asserted digest). `out`, if given, is a
        device tensor of at least 756 * height elements and receives the trace."""
        return self._hash_trace("sha256", message, out)

    def sha512_trace(self, message: bytes, out=None):
        """build_sha512_trace_multi with the column expansion on the GPU ->
        ((1510, height) trace, n_blocks, 64-byte digest)."""
        return self._hash_trace("sha512", message, out)

    def merge_sha256(self, lde, n_trace: int, blowup: int, lambdas, n_blocks: int, phi_mode=PHI_PARALLEL_GATE,
                     out=None):
        """deep_ali_merge_sha256 on a (756, n_trace*blowup) LDE."""
        return self._merge_hash("sha256", lde, n_trace, blowup, lambdas, n_blocks, phi_mode, out)

    def merge_sha512(self, lde, n_trace: int, blowup: int, lambdas, n_blocks: int, phi_mode=PHI_PARALLEL_GATE,
                     out=None):
        """deep_ali_merge_sha512 on a (1510, n_trace*blowup) LDE."""
        return self._merge_hash("sha512", lde, n_trace, blowup, lambdas, n_blocks, phi_mode, out)

    def prove_sha256(self, message: bytes, fs_binding: bytes, phi_mode=PHI_PARALLEL_GATE):
        """prove_ds_ksk_binding core -> (proof bytes, asserted SHA-256 digest); self-verified."""
        return self._prove_hash("sha256", message, fs_binding, phi_mode)

    def prove_sha512(self, message: bytes, fs_binding: bytes, phi_mode=PHI_PARALLEL_GATE):
        """SHA-512 AIR proof (LDE x32, lambda_j = j+1, STIR) -> (proof bytes, 64-byte digest); self-verified."""
        return self._prove_hash("sha512", message, fs_binding, phi_mode)

    def rsa2048_trace(self, records, out=None):
        """The RSA trace with the cells expanded on the GPU -> (len(records) * 11041, 32);
        `out`, if given, is a device tensor of at least that many elements."""
        ns, ss, es = _rsa_records(records)
        cells = len(records) * RSA_WIDTH * RSA_N_TRACE
        host = out is None
        if host:
            out = np.empty(cells, dtype=np.uint64)
        op, _k, _ = _addr(out)
        self._check(self._lib.sg_rsa2048_trace_gpu(self._h, ns, ss, es, len(records), op, cells))
        return out.reshape(len(records) * RSA_WIDTH, RSA_N_TRACE) if host else out

    def merge_rsa2048(self, lde, n_records: int, n_trace: int = RSA_N_TRACE, blowup: int = RSA_BLOWUP, out=None):
        """deep_ali_merge_rsa_exp_multirow / _stacked on a (n_records * 11041, n_trace * blowup) LDE -> c_eval."""
        n = n_trace * blowup
        ip, _ki, is_np = _addr(lde)
        if out is None:
            if not is_np:
                raise ValueError("device input needs an explicit out buffer")
            out = np.empty(n, dtype=np.uint64)
        op, _ko, _ = _addr(out)
        self._check(self._lib.sg_merge_rsa2048(self._h, ip, n_records, n_trace, blowup, op))
        return out

    def prove_rsa2048(self, records, pi: bytes) -> bytes:
        """RSA-2048 signature-check proof of [(n, s, em)] records (one record:
        prove_rsa2048_record_v1.rs; several: stacked_rsa_zone_prover.rs) -> proof bytes; self-verified."""
        if len(pi) != 32:
            raise ValueError("pi must be 32 bytes")
        ns, ss, es = _rsa_records(records)
        cap = _PROOF_CAP
        while True:
            arr, buf = _out_buffer(cap)
            ln = ctypes.c_size_t()
            rc = self._lib.sg_prove_rsa2048(self._h, ns, ss, es, len(records), pi, buf, cap, ctypes.byref(ln))
            if rc == SG_ESPACE:
                cap = ln.value
                continue
            self._check(rc)
            return arr[:ln.value].tobytes()

    def p256_chain_trace(self, a_point, a_bits, b_point, b_bits, out=None):
        """The double-chain trace with the cells expanded on the GPU -> (151334, len(bits))."""
        k = len(a_bits)
        width = p256_layout()[0]
        host = out is None
        if host:
            out = np.empty(width * k, dtype=np.uint64)
        op, _k, _ = _addr(out)
        self._check(self._lib.sg_p256_chain_trace_gpu(self._h, _be32(a_point[0]), _be32(a_point[1]), _bits(a_bits),
                                                      _be32(b_point[0]), _be32(b_point[1]), _bits(b_bits), k, op,
                                                      width * k))
        return out.reshape(width, k) if host else out

    def merge_p256_ecdsa(self, lde, n_trace: int, blowup: int = P256_BLOWUP, out=None):
        """deep_ali_merge_ecdsa_double_multirow_streaming on a (151334, n_trace * blowup) LDE -> c_eval."""
        ip, _ki, is_np = _addr(lde)
        if out is None:
            if not is_np:
                raise ValueError("device input needs an explicit out buffer")
            out = np.empty(n_trace * blowup, dtype=np.uint64)
        op, _ko, _ = _addr(out)
        self._check(self._lib.sg_merge_p256_ecdsa(self._h, ip, n_trace, blowup, op))
        return out

    def prove_p256_chains(self, a_point, a_bits, b_point, b_bits, pi: bytes) -> bytes:
        """Proof of two chains of len(bits) rows (LDE x32, STIR); self-verified."""
        cap = _PROOF_CAP
        while True:
            arr, buf = _out_buffer(cap)
            ln = ctypes.c_size_t()
            rc = self._lib.sg_prove_p256_chains(self._h, _be32(a_point[0]), _be32(a_point[1]), _bits(a_bits),
                                                _be32(b_point[0]), _be32(b_point[1]), _bits(b_bits), len(a_bits),
                                                pi, buf, cap, ctypes.byref(ln))
            if rc == SG_ESPACE:
                cap = ln.value
                continue
            self._check(rc)
            return arr[:ln.value].tobytes()

    def prove_p256_ecdsa(self, q, r, s, digest: bytes, pi: bytes) -> bytes:
        """ECDSA-P256 signature-check proof (prove_ecdsa_record_v1.rs: K = 256, n0 = 8192); self-verified."""
        cap = _PROOF_CAP
        while True:
            arr, buf = _out_buffer(cap)
            ln = ctypes.c_size_t()
            rc = self._lib.sg_prove_p256_ecdsa(self._h, _be32(q[0]), _be32(q[1]), _be32(r), _be32(s), _be32(digest),
                                               pi, buf, cap, ctypes.byref(ln))
            if rc == SG_ESPACE:
                cap = ln.value
                continue
            self._check(rc)
            return arr[:ln.value].tobytes()

    def ed25519_trace(self, pub: bytes, sig: bytes, msg: bytes, k_scalar: int = ED25519_K, out=None):
        """The verify AIR trace with the cells expanded on the GPU -> (width, height)."""
        pub, sig, msg = _ed_args(pub, sig, msg)
        w, h, _k, _r = ed25519_layout(len(msg), k_scalar)
        host = out is None
        if host:
            out = np.empty(w * h, dtype=np.uint64)
        op, _ko, _ = _addr(out)
        self._check(self._lib.sg_ed25519_trace_gpu(self._h, pub, sig, msg, len(msg), k_scalar, op, w * h))
        return out.reshape(w, h) if host else out

    def merge_ed25519(self, pub: bytes, sig: bytes, msg: bytes, lde, blowup: int = ED25519_BLOWUP,
                      k_scalar: int = ED25519_K, out=None):
        """deep_ali_merge_ed25519_verify on a (width, height * blowup) LDE -> c_eval."""
        pub, sig, msg = _ed_args(pub, sig, msg)
        ip, _ki, is_np = _addr(lde)
        if out is None:
            if not is_np:
                raise ValueError("device input needs an explicit out buffer")
            out = np.empty(ed25519_layout(len(msg), k_scalar)[1] * blowup, dtype=np.uint64)
        op, _ko, _ = _addr(out)
        self._check(self._lib.sg_merge_ed25519(self._h, pub, sig, msg, len(msg), k_scalar, ip, blowup, op))
        return out

    def prove_ed25519(self, pub: bytes, sig: bytes, msg: bytes, fs_binding: bytes, k_scalar: int = ED25519_K,
                      blowup: int = ED25519_BLOWUP) -> bytes:
        """Ed25519 verify AIR proof (LDE x blowup, STIR with build_params(height * blowup, fs_binding));
        self-verified."""
        pub, sig, msg = _ed_args(pub, sig, msg)
        if len(fs_binding) != 32:
            raise ValueError("fs_binding must be 32 bytes")
        cap = _PROOF_CAP
        while True:
            arr, buf = _out_buffer(cap)
            ln = ctypes.c_size_t()
            rc = self._lib.sg_prove_ed25519(self._h, pub, sig, msg, len(msg), fs_binding, k_scalar, blowup, buf, cap,
                                            ctypes.byref(ln))
            if rc == SG_ESPACE:
                cap = ln.value
                continue
            self._check(rc)
            return arr[:ln.value].tobytes()

    def prove_zsk_ksk_binding_v2(self, pub: bytes, sig: bytes, msg: bytes, fs_binding: bytes, merkle_root: bytes,
                                 k_scalar: int = ED25519_K):
        """prove_zsk_ksk_binding_v2 (swarm-dns/src/prover.rs:856-951) -> (proof bytes, pi_hash); the
        signature is verified natively first (SG_EVERIFY if it does not verify)."""
        pub, sig, msg = _ed_args(pub, sig, msg)
        if len(fs_binding) != 32 or len(merkle_root) != 32:
            raise ValueError("fs_binding and merkle_root must be 32 bytes")
        cap = _PROOF_CAP
        while True:
            arr, buf = _out_buffer(cap)
            ln = ctypes.c_size_t()
            pi = ctypes.create_string_buffer(32)
            rc = self._lib.sg_prove_zsk_ksk_binding_v2(self._h, pub, sig, msg, len(msg), fs_binding, merkle_root,
                                                       k_scalar, buf, cap, ctypes.byref(ln), pi)
            if rc == SG_ESPACE:
                cap = ln.value
                continue
            self._check(rc)
            return arr[:ln.value].tobytes(), pi.raw

    def prove_inner_shard(self, records, salt: bytes, fs_binding: bytes, stir: bool = True):
        """prove_inner_shard (swarm-dns/src/prover.rs:148-225) on canonical records ->
        (proof bytes, pi_hash, DNS merkle root); self-verified."""
        if len(salt) != 16 or len(fs_binding) != 32:
            raise ValueError("salt must be 16 bytes and fs_binding 32 bytes")
        canon, offs = _records(records)
        cap = _PROOF_CAP
        while True:
            arr, buf = _out_buffer(cap)
            ln = ctypes.c_size_t()
            pi, root = ctypes.create_string_buffer(32), ctypes.create_string_buffer(32)
            rc = self._lib.sg_prove_inner_shard(self._h, canon, offs, len(records), salt, fs_binding, int(stir), buf,
                                                cap, ctypes.byref(ln), pi, root)
            if rc == SG_ESPACE:
                cap = ln.value
                continue
            self._check(rc)
            return arr[:ln.value].tobytes(), pi.raw, root.raw

    def prove_outer_rollup(self, pi_hashes, pk_hash: bytes, stir: bool = True) -> bytes:
        """prove_outer_rollup (swarm-dns/src/prover.rs:250-304) -> proof bytes; self-verified."""
        if len(pk_hash) != 32 or not pi_hashes:
            raise ValueError("need pi hashes and a 32-byte pk_hash")
        cap = _PROOF_CAP
        while True:
            arr, buf = _out_buffer(cap)
            ln = ctypes.c_size_t()
            rc = self._lib.sg_prove_outer_rollup(self._h, b"".join(pi_hashes), len(pi_hashes), pk_hash, int(stir),
                                                 buf, cap, ctypes.byref(ln))
            if rc == SG_ESPACE:
                cap = ln.value
                continue
            self._check(rc)
            return arr[:ln.value].tobytes()

    def prove_batch(self, jobs, n_streams: int = 8, hbm_budget_bytes: int = 0, cap_per_job: int = 1 << 20):
        """jobs: list of (kind, data, pi[, phi_mode[, blowup[, flags]]]) -> list of (proof bytes, JobResult).
        blowup 0 (the default) is the reference prover's own, 32."""
        made = [make_job(*j) for j in jobs]
        arr = (Job * len(made))(*[m[0] for m in made])
        res = (JobResult * len(made))()
        # uninitialised result slots: only each proof's own bytes are touched and copied out
        buf = np.empty(cap_per_job * max(1, len(made)), dtype=np.uint8)
        rc = self._lib.sg_prove_batch(self._h, arr, len(made), n_streams, hbm_budget_bytes,
                                      ctypes.cast(buf.ctypes.data, ctypes.c_char_p), cap_per_job, res)
        if rc != SG_OK:
            raise StarkGpuError(rc, "sg_prove_batch failed")
        return [(buf[i * cap_per_job: i * cap_per_job + res[i].proof_len].tobytes(), res[i]) for i in range(len(made))]

    def deep_ali_merge_general(self, trace_evals_on_lde, combination_coeffs, air, omega, n_trace, blowup,
                               phi_mode=PHI_PARALLEL_GATE):
        del omega  # the domain generator is implied by n = n_trace * blowup
        lde = np.ascontiguousarray(np.array(trace_evals_on_lde, dtype=np.uint64))
        return self.merge(air, lde, n_trace, blowup, combination_coeffs, phi_mode)

    # ---------------------------------------------------------------- Merkle
    def merkle_commit(self, cols, arities, tree_label: int, n_leaves=None, col_stride=None, keep=False):
        """Commit to the rows of a column-major (width, n) buffer; returns root (and a tree handle if keep)."""
        ip, _ki, host = _addr(cols)
        width = cols.shape[0]
        n = cols.shape[1] if n_leaves is None else n_leaves
        cs = cols.shape[1] if col_stride is None else col_stride
        ar = np.ascontiguousarray(arities, dtype=np.uint64)
        root = ctypes.create_string_buffer(HASH_BYTES)
        t = ctypes.c_void_p()
        self._check(self._lib.sg_merkle_commit(self._h, ip, n, width, cs, ar.ctypes.data, ar.size, tree_label, root,
                                               ctypes.byref(t) if keep else None))
        return (root.raw, MerkleTree(self, t)) if keep else root.raw

    # ---------------------------------------------------------------- STIR
    def deep_fri_prove_group(self, f0s, params_list, cap_per_proof: int = 1 << 21):
        """n STIR proofs of one shape in lockstep (sg_stir_prove_group): f0s is an (n, n0)
        buffer, params_list n FriParams that differ only in their public-input hash.
        Returns the n proofs' bytes, each equal to deep_fri_prove's."""
        ip, _ki, host = _addr(f0s)
        n, n0 = f0s.shape
        if len(params_list) != n:
            raise ValueError("one FriParams per proof")
        ps = (FriParams * n)(*params_list)
        while True:
            buf = np.empty(cap_per_proof * n, dtype=np.uint8)
            lens = (ctypes.c_size_t * n)()
            rc = self._lib.sg_stir_prove_group(self._h, ip, n0, n, ps, ctypes.cast(buf.ctypes.data, ctypes.c_char_p),
                                               cap_per_proof, lens)
            if rc == SG_ESPACE:
                cap_per_proof = max(lens)
                continue
            self._check(rc)
            return [buf[g * cap_per_proof: g * cap_per_proof + lens[g]].tobytes() for g in range(n)]

    def deep_fri_prove(self, f0, domain0, params: FriParams) -> bytes:
        """deep_fri_prove (STIR or classic DEEP-FRI, per params.stir); returns the
        ark-serialize (Compress::Yes) bytes of the DeepFriProof."""
        ip, _ki, host = _addr(f0)
        n0 = domain0.size if isinstance(domain0, FriDomain) else int(domain0)
        cap = _PROOF_CAP
        while True:
            arr, buf = _out_buffer(cap)
            ln = ctypes.c_size_t()
            rc = self._lib.sg_stir_prove(self._h, ip, n0, ctypes.byref(params), buf, cap, ctypes.byref(ln))
            if rc == SG_ESPACE:
                cap = ln.value
                continue
            self._check(rc)
            return arr[:ln.value].tobytes()

    def prove_hash_rollup(self, leaves, pi: bytes, phi_mode=PHI_PARALLEL_GATE) -> bytes:
        """prove_inner_shard / prove_outer_rollup core on u64 rollup leaves; self-verified."""
        lv = np.ascontiguousarray(leaves, dtype=np.uint64)
        if len(pi) != 32:
            raise ValueError("pi must be 32 bytes")
        cap = _PROOF_CAP
        while True:
            arr, buf = _out_buffer(cap)
            ln = ctypes.c_size_t()
            rc = self._lib.sg_prove_hash_rollup(self._h, lv.ctypes.data if lv.size else None, lv.size, pi, phi_mode,
                                                buf, cap, ctypes.byref(ln))
            if rc == SG_ESPACE:
                cap = ln.value
                continue
            self._check(rc)
            return arr[:ln.value].tobytes()


def make_job(kind: int, data, pi: bytes, phi_mode: int = PHI_PARALLEL_GATE, blowup: int = 0, flags: int = 0):
    """A sg_job plus the buffer it points to (keep both alive until submitted)."""
    if len(pi) != 32:
        raise ValueError("pi must be 32 bytes")
    if kind == JOB_RSA2048:
        # data: [(n, s, em)] records (ints or 256-byte big-endian strings)
        data = b"".join(_be256(r[0]) + _be256(r[1]) + _be256(r[2]) for r in data)
        if not data:
            raise ValueError("an RSA job needs at least one record")
    if kind == JOB_P256_ECDSA and not isinstance(data, (bytes, bytearray)):
        # data: (q, r, s, digest) with q = (x, y), or the 160 packed bytes
        q, r, s_, dg = data
        data = _be32(q[0]) + _be32(q[1]) + _be32(r) + _be32(s_) + _be32(dg)
    if kind == JOB_ED25519 and not isinstance(data, (bytes, bytearray)):
        # data: (pub, sig, msg), or the packed pub || sig || msg
        pub, sig, msg = _ed_args(*data)
        data = pub + sig + msg
    if kind in (JOB_SHA256, JOB_SHA512, JOB_RSA2048, JOB_P256_ECDSA, JOB_ED25519):
        buf = ctypes.create_string_buffer(bytes(data), max(1, len(data)))
        n = len(data)
    elif kind == JOB_HASH_ROLLUP:
        buf = np.ascontiguousarray(data, dtype=np.uint64)
        n = buf.size
    else:
        raise ValueError("unknown job kind")
    j = Job()
    j.kind, j.phi_mode, j.blowup, j.flags = kind, phi_mode, blowup, flags
    j.input = ctypes.addressof(buf) if kind != JOB_HASH_ROLLUP else (buf.ctypes.data if n else None)
    j.input_len = n
    ctypes.memmove(j.pi, pi, 32)
    return j, buf


class Server:
    """Continuous-batching proof server (sg_server): submit() any time, wait() per ticket."""

    def __init__(self, ctx: "Context", n_streams: int = 8, hbm_budget_bytes: int = 0):
        self._ctx = ctx
        h = ctypes.c_void_p()
        rc = ctx._lib.sg_server_create(ctx._h, n_streams, hbm_budget_bytes, ctypes.byref(h))
        if rc != SG_OK:
            raise StarkGpuError(rc, "sg_server_create failed")
        self._h = h

    def submit(self, kind: int, data, pi: bytes, phi_mode: int = PHI_PARALLEL_GATE, blowup: int = 0,
               flags: int = 0) -> int:
        j, _keep = make_job(kind, data, pi, phi_mode, blowup, flags)
        t = ctypes.c_uint64()
        rc = self._ctx._lib.sg_server_submit(self._h, ctypes.byref(j), ctypes.byref(t))
        if rc != SG_OK:
            raise StarkGpuError(rc, "sg_server_submit failed")
        return t.value

    def poll(self, ticket: int) -> bool:
        return self._ctx._lib.sg_server_poll(self._h, ticket) == 1

    def wait(self, ticket: int, timeout_ms: int = None):
        """-> (proof bytes, JobResult). With timeout_ms, raises StarkGpuError with code
        SG_ETIMEDOUT (the ticket stays valid) when the job is not done in time."""
        cap = _PROOF_CAP
        while True:
            res = JobResult()
            arr, buf = _out_buffer(cap)
            if timeout_ms is None:
                rc = self._ctx._lib.sg_server_wait(self._h, ticket, ctypes.byref(res), buf, cap)
            else:
                rc = self._ctx._lib.sg_server_wait_for(self._h, ticket, int(timeout_ms), ctypes.byref(res), buf, cap)
            if rc == SG_ESPACE:
                cap = res.proof_len
                continue
            if rc != SG_OK:
                raise StarkGpuError(rc, f"job {ticket} failed")
            return arr[:res.proof_len].tobytes(), res

    def cancel(self, ticket: int) -> int:
        """0: dropped from the queue; 1: running, its result will be discarded; 2: already done."""
        rc = self._ctx._lib.sg_server_cancel(self._h, ticket)
        if rc < 0:
            raise StarkGpuError(rc, f"sg_server_cancel({ticket}) failed")
        return rc

    def set_retries(self, max_retries: int):
        """re-run a job whose attempt failed with SG_ENOMEM / SG_ECUDA up to max_retries times"""
        rc = self._ctx._lib.sg_server_set_retries(self._h, max_retries)
        if rc != SG_OK:
            raise StarkGpuError(rc, "sg_server_set_retries failed")

    def close(self):
        if getattr(self, "_h", None):
            self._ctx._lib.sg_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MerkleTree:
    """Device-resident tree kept by Context.merkle_commit(keep=True)."""

    def __init__(self, ctx: Context, handle):
        self._ctx, self._h = ctx, handle

    def open(self, index: int) -> bytes:
        cap = 1 << 16
        buf = ctypes.create_string_buffer(cap)
        ln = ctypes.c_size_t()
        self._ctx._check(self._ctx._lib.sg_merkle_open(self._ctx._h, self._h, index, buf, cap, ctypes.byref(ln)))
        return buf.raw[:ln.value]

    def free(self):
        if self._h:
            self._ctx._lib.sg_merkle_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

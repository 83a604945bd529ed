"""Checks of one hash profile (the reference's compile-time sha3-256 / sha3-384 /
sha3-512 feature, hash/src/selected.rs:8-48), run in a process of its own with
STARK_GPU_HASH set, since the oracle and the library each load the build of that
profile. `python tests/hash_profile_checks.py oracle|gpu`; exits non-zero on a
failure. The tests in test_hash_profiles*.py launch it.

What changes with the profile: every Merkle leaf and node digest and the
Fiat-Shamir transcript (transcript/src/lib.rs:162-212: same FSv1 framing, the
profile's SHA3, challenges of HASH_BYTES bytes folded 7 bytes at a time from the
end), so every root in a proof is HASH_BYTES long. DNS record hashing and the
pi_hash recipes stay SHA3-256 (swarm-dns/src/dns.rs:17, prover.rs:207).
"""
import hashlib
import os
import struct
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import oracle_lib as O  # noqa: E402

P = O.P
H = {"sha3-256": hashlib.sha3_256, "sha3-384": hashlib.sha3_384, "sha3-512": hashlib.sha3_512}[O.HASH_PROFILE]


def py_merkle(rows, arities, label):
    """merkle/src/lib.rs:95-238,423-476 restated with hashlib and the profile's SHA3."""
    def ds(ar, lvl, pos):
        return struct.pack("<4Q", ar, lvl, pos, label)
    lvl = [H(ds(arities[0], 0xFFFFFFFF, i) + struct.pack(f"<{len(r)}Q", *map(int, r))).digest()
           for i, r in enumerate(rows)]
    li = 0
    while len(lvl) > 1:
        a = arities[li]
        while len(lvl) % a:
            lvl.append(lvl[-1])
        lvl = [H(ds(a, li + 1, j) + b"".join(lvl[j * a:(j + 1) * a])).digest() for j in range(len(lvl) // a)]
        li += 1
    return lvl[0]


def pick_arity(n, m):
    """fri.rs:1094-1103"""
    for c in (128, 64, 32, 16, 8, 4):
        if m >= c and n % c == 0:
            return c
    return 2 if n % 2 == 0 else 1


def merkle_depth(leaves, arity):
    """fri.rs:950-959"""
    depth, cur = 1, leaves
    while cur > arity:
        cur = (cur + arity - 1) // arity
        depth += 1
    return depth


def f0_root(f0, m0):
    """The packed-f0 tree (fri.rs:1420-1431): leaf b = {f0[b + j n0/m0]}_j, label 0xFF."""
    nn = f0.size // m0
    rows = f0.reshape(m0, nn).T
    a = pick_arity(nn, 16)
    return py_merkle(rows, [a] * merkle_depth(nn, a), 0xFF)


def low_degree(n0, seed):
    rng = np.random.default_rng(seed)
    c = np.zeros(n0, dtype=np.uint64)
    k = max(1, n0 // 32)
    c[:k] = rng.integers(0, P, k, dtype=np.uint64)
    return O.ntt(c)


def oracle_checks():
    import ctypes
    L = O.lib()
    hb = O.HASH_BYTES
    assert L.orc_hash_bytes() == hb == H().digest_size
    for n in list(range(0, 260)) + [1000, 4096]:
        m = bytes((i * 7 + 3) % 256 for i in range(n))
        out = ctypes.create_string_buffer(hb)
        L.orc_sha3_selected(m, n, out)
        assert out.raw == H(m).digest(), n
    assert O.sha3_256(b"abc") == hashlib.sha3_256(b"abc").digest()  # SHA3-256 stays for DNS / pi
    for n, width, arities, label in ((1, 6, [2], 0xFE), (5, 3, [2, 2, 2], 7), (16, 8, [16], 0xFF),
                                     (100, 4, [8, 8, 8], 1), (37, 2, [4, 4, 4], 0)):
        rows = np.random.default_rng(n).integers(0, P, (n, width), dtype=np.uint64)
        assert O.merkle_root(rows, arities, label) == py_merkle(rows, arities, label)
    for lg in (4, 9, 12):
        n0 = 1 << lg
        f0 = low_degree(n0, lg)
        for stir in (True, False):
            params = O.build_params(n0, hashlib.sha3_256(b"profile %d" % lg).digest(), stir=stir)
            proof = O.stir_prove(f0, params)
            assert O.stir_verify(proof, params), (lg, stir)
            m0 = params.sched[0]
            if stir:
                assert proof[:hb] == f0_root(f0, m0), "root_f0"
            # (the classic branch's f0_openings and omega0 are not read by the verifier,
            # in the reference either, so its flips stay in the checked fields)
            for pos in ((3, hb + 5, len(proof) // 2, len(proof) - 40) if stir else (3, 40, 300)):
                bad = bytearray(proof)
                bad[pos] ^= 0x20
                assert not O.stir_verify(bytes(bad), params), (lg, stir, pos)
    print(f"oracle {O.HASH_PROFILE}: ok")


def _sg():
    import importlib
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    sg = importlib.import_module("stark-swarm_b200")
    assert sg.HASH_PROFILE == O.HASH_PROFILE and sg.lib().sg_hash_bytes() == O.HASH_BYTES
    return sg


def library_cpu_checks():
    """The library's host verifier against the oracle's proofs of the same profile."""
    sg = _sg()
    for lg in (4, 9, 12):
        n0 = 1 << lg
        f0 = low_degree(n0, lg)
        for stir in (True, False):
            pi = hashlib.sha3_256(b"profile %d" % lg).digest()
            proof = O.stir_prove(f0, O.build_params(n0, pi, stir=stir))
            params = sg.build_params(n0, pi, stir=stir)
            assert sg.deep_fri_verify(params, proof), (lg, stir)
            for pos in ((3, O.HASH_BYTES + 5, len(proof) // 2) if stir else (3, 40, 300)):
                bad = bytearray(proof)
                bad[pos] ^= 0x20
                assert not sg.deep_fri_verify(params, bytes(bad)), (lg, stir, pos)
    print(f"library (host) {O.HASH_PROFILE}: ok")


def gpu_checks():
    """GPU proofs and roots byte-identical to the oracle's in this profile."""
    sg = _sg()
    with sg.Context(0) as ctx:
        for n, width, arities, label in ((16, 8, [16], 0xFF), (100, 4, [8, 8, 8], 1), (37, 2, [4, 4, 4], 0),
                                         (4096, 64, [16, 16, 16], 0)):
            rows = np.random.default_rng(n).integers(0, P, (n, width), dtype=np.uint64)
            got = ctx.merkle_commit(np.ascontiguousarray(rows.T), arities, label)
            assert got == O.merkle_root(rows, arities, label), n
            if n <= 100:
                assert got == py_merkle(rows, arities, label), n
        # LDE + row commitment in one call (the fused last pass hashes with this profile's SHA3)
        tr = np.random.default_rng(9).integers(0, P, (32, 1 << 9), dtype=np.uint64)
        lde = O.lde(tr, 8, 7)
        assert ctx.lde_commit(tr, 8, 7, [16, 16, 16, 16], 3) == \
            O.merkle_root(np.ascontiguousarray(lde.T), [16, 16, 16, 16], 3)
        for lg in (3, 8, 12, 16):
            n0 = 1 << lg
            f0 = low_degree(n0, lg)
            for stir in (True, False):
                pi = hashlib.sha3_256(b"gpu profile %d" % lg).digest()
                want = O.stir_prove(f0, O.build_params(n0, pi, stir=stir))
                got = ctx.deep_fri_prove(f0, n0, sg.build_params(n0, pi, stir=stir))
                assert got == want, (lg, stir)
                assert sg.deep_fri_verify(sg.build_params(n0, pi, stir=stir), got)
        for m in (b"", b"abc", bytes(range(200))):
            fsb = hashlib.sha3_256(m).digest()
            proof, dg = ctx.prove_sha256(m, fsb)
            wproof, wdg = O.prove_sha256(m, fsb)
            assert proof == wproof and dg[:32] == wdg == hashlib.sha256(m).digest()
    print(f"gpu {O.HASH_PROFILE}: ok")


if __name__ == "__main__":
    {"oracle": oracle_checks, "library": library_cpu_checks, "gpu": gpu_checks}[sys.argv[1]]()

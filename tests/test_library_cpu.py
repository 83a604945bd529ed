"""CPU-side checks of the GPU library: it loads, exports the declared C ABI,
and its host-only parts (parameter builder, STIR verifier) agree with the
oracle. No kernel is launched here."""
import ctypes
import hashlib
import os
import random
import re
import subprocess

import numpy as np
import pytest

import dnszone
import oracle_lib as O
from conftest import ROOT, load_sgpu

HEADER = os.path.join(ROOT, "include", "stark_gpu.h")


def _declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sg_[a-z0-9_]+)\s*\(", src)))


def test_library_builds_and_exports_every_declared_symbol():
    sg = load_sgpu()
    if not os.path.exists(sg.LIB_PATH):
        subprocess.run(["make", "-s", "-C", os.path.dirname(sg.LIB_PATH)], check=True)
    L = sg.lib()
    declared = _declared_functions()
    assert declared, "no declarations parsed"
    assert sorted(sg.EXPORTS) == declared
    for name in declared:
        assert getattr(L, name) is not None
    nm = subprocess.run(["nm", "-D", "--defined-only", sg.LIB_PATH], capture_output=True, text=True).stdout
    for name in declared:
        assert re.search(rf"\bT {name}\b", nm), name


@pytest.mark.parametrize("n0", [8, 16, 512, 4096, 1 << 17, 1 << 23])
def test_build_params_matches_reference_recipe(n0):
    sg = load_sgpu()
    pi = bytes(range(32))
    a = sg.build_params(n0, pi)
    b = O.build_params(n0, pi)
    assert a.schedule_list == b.sched == sg.make_schedule(n0)
    for f in ("r", "s0", "seed_z", "d_final", "coeff_commit_final", "stir", "has_pi"):
        assert getattr(a, f) == getattr(b, f), f
    assert bytes(a.pi_hash) == pi


def test_verifier_accepts_golden_outer_and_rejects_tampering(golden):
    sg = load_sgpu()
    leaves, pk = dnszone.outer_rollup_inputs(golden)
    proof = O.prove_hash_rollup(leaves, pk)
    params = sg.build_params(512, pk)
    assert sg.deep_fri_verify(params, proof)
    rng = random.Random(11)
    for _ in range(30):
        i = rng.randrange(len(proof))
        bad = bytearray(proof)
        bad[i] ^= 1 << rng.randrange(8)
        assert not sg.deep_fri_verify(params, bytes(bad)), i
    assert not sg.deep_fri_verify(sg.build_params(512, bytes(32)), proof)
    assert not sg.deep_fri_verify(params, proof[:-1])
    assert not sg.deep_fri_verify(params, proof + b"\0")


def test_verifier_accepts_golden_inner_shard(golden):
    sg = load_sgpu()
    sh = golden["shards"][0]
    leaves, fsb, _root, _count = dnszone.inner_shard_inputs(golden, sh)
    proof = O.prove_hash_rollup(leaves, fsb)
    assert sg.deep_fri_verify(sg.build_params(sh["n0"], fsb), proof)


@pytest.mark.parametrize("sched,cc", [([4, 2, 8], True), ([2, 2, 2, 2, 2, 2], False), ([16, 4], True)])
def test_verifier_agrees_with_oracle_on_other_schedules(sched, cc):
    sg = load_sgpu()
    n0 = 1
    for m in sched:
        n0 *= m
    n0 *= 4
    pi = os.urandom(32)
    p_o = O.build_params(n0, pi)
    p_o.schedule_len = len(sched)
    for i, m in enumerate(sched):
        p_o.schedule[i] = m
    p_o.coeff_commit_final = int(cc)
    p_o.d_final = 4
    p_s = sg.FriParams.new(sched, coeff_commit_final=cc, d_final=4, public_inputs_hash=pi)
    # f0 of degree < 4 so the final-polynomial check holds for these schedules
    xs = [pow(int(sg.FriDomain(n0).omega), i, O.P) for i in range(n0)]
    c = [random.randrange(O.P) for _ in range(4)]
    f0 = np.array([sum(ci * pow(x, k, O.P) for k, ci in enumerate(c)) % O.P for x in xs], dtype=np.uint64)
    proof = O.stir_prove(f0, p_o)
    assert O.stir_verify(proof, p_o)
    assert sg.deep_fri_verify(p_s, proof)


@pytest.mark.parametrize("msg", [b"abc", b"", bytes(range(64)), b"c" * 120, bytes(range(200))])
def test_sha256_trace_builder_matches_oracle(msg):
    # host-side trace builder (build_sha256_trace_multi) of the library vs the oracle
    import hashlib
    sg = load_sgpu()
    tr, nb, digest = sg.build_sha256_trace_multi(msg)
    otr, onb = O.sha256_trace(msg)
    assert nb == onb
    assert np.array_equal(tr, otr)
    assert digest == hashlib.sha256(msg).digest()


@pytest.mark.parametrize("msg", [b"abc", b"", b"a" * 111, b"b" * 112, bytes(range(256)) + b"z" * 50])
def test_sha512_trace_builder_matches_oracle(msg):
    # host-side trace builder (build_sha512_trace_multi) of the library vs the oracle
    import hashlib
    sg = load_sgpu()
    tr, nb, digest = sg.build_sha512_trace_multi(msg)
    otr, onb = O.sha512_trace(msg)
    assert nb == onb
    assert np.array_equal(tr, otr)
    assert digest == hashlib.sha512(msg).digest()


@pytest.mark.parametrize("log_n0", [3, 6, 9])
def test_product_verifier_accepts_oracle_classic_fri(log_n0):
    import hashlib
    sg = load_sgpu()
    n0 = 1 << log_n0
    rng = np.random.default_rng(log_n0)
    c = np.zeros(n0, dtype=np.uint64)
    c[: max(1, n0 // 32)] = rng.integers(0, O.P, max(1, n0 // 32), dtype=np.uint64)
    f0 = O.ntt(c)
    pi = hashlib.sha3_256(b"cls").digest()
    proof = O.stir_prove(f0, O.build_params(n0, pi, stir=False))
    ps = sg.build_params(n0, pi, stir=False)
    assert sg.deep_fri_verify(ps, proof)
    bad = bytearray(proof)
    bad[100] ^= 1
    assert not sg.deep_fri_verify(ps, bytes(bad))


def test_dns_shard_helpers_match_golden_bundle(golden):
    # record leaf hashes, the DNS Merkle root and the shard pi_hash of every golden
    # shard (merkle_root_hex, pi_hash_hex come from the reference's zone bundle)
    sg = load_sgpu()
    salt = bytes.fromhex(golden["zone_salt_hex"])
    shards = dnszone.split_evenly(dnszone.synthetic_zone(golden["record_count"]), golden["shard_count"])
    for sh in golden["shards"]:
        recs = [dnszone.canonical_bytes(*r) for r in shards[sh["shard_id"] - 1]]
        leaves = sg.dns_record_leaves(recs, salt)
        assert leaves[:5] == [dnszone.record_leaf_hash(r, salt) for r in shards[sh["shard_id"] - 1][:5]]
        root = sg.dns_merkle_root(leaves)
        assert root.hex() == sh["merkle_root_hex"]
        _, fsb, _, count = dnszone.inner_shard_inputs(golden, sh)
        pi = sg.shard_pi_hash(salt, count, root, bytes.fromhex(sh["root_f0_hex"]), fsb)
        assert pi.hex() == sh["pi_hash_hex"]
        for idx in (0, 1, len(leaves) // 2, len(leaves) - 1):
            path = sg.dns_merkle_path(leaves, idx)
            assert sg.dns_merkle_verify(leaves[idx], idx, path, root)
            assert not sg.dns_merkle_verify(leaves[idx], idx ^ 1, path, root)


@pytest.mark.parametrize("n", [1, 2, 3, 7, 8, 33])
def test_dns_merkle_root_small_trees(n):
    sg = load_sgpu()
    leaves = [hashlib.sha3_256(bytes([i])).digest() for i in range(n)]
    assert sg.dns_merkle_root(leaves) == dnszone.dns_merkle_root(leaves)
    for idx in range(n):
        assert sg.dns_merkle_verify(leaves[idx], idx, sg.dns_merkle_path(leaves, idx), dnszone.dns_merkle_root(leaves))


def test_ntt_split_setter_bounds():
    # the split table is host state: valid splits are accepted and reset, others refused
    sg = load_sgpu()
    sg.ntt_set_split(20, False, 12)
    sg.ntt_set_split(20, False, 0)
    for log_n, l1 in ((12, 6), (25, 12), (20, 7), (20, 13), (13, -1)):
        with pytest.raises(sg.StarkGpuError):
            sg.ntt_set_split(log_n, False, l1)
    assert sg.lib().sg_hash_bytes() == sg.HASH_BYTES == 32


def test_ntt_noalloc_wrapper_refuses_bad_buffers_before_the_call():
    # the no-alloc NTT cannot see buffer lengths on the device, so its Python
    # wrapper checks them first; every case below raises before the library is called
    torch = pytest.importorskip("torch")
    sg = load_sgpu()
    n = 1 << 10
    good = torch.zeros(2 * n, dtype=torch.int64)
    with pytest.raises(ValueError):  # not a whole number of columns
        sg.ntt_noalloc(torch.zeros(2 * n + 1, dtype=torch.int64), good, 10)
    with pytest.raises(ValueError):  # shorter than one column
        sg.ntt_noalloc(torch.zeros(n // 2, dtype=torch.int64), good, 10)
    with pytest.raises(ValueError):  # output shorter than the input
        sg.ntt_noalloc(good, torch.zeros(n, dtype=torch.int64), 10)
    with pytest.raises(ValueError):  # raw pointers without a column count
        sg.ntt_noalloc(good.data_ptr(), good.data_ptr(), 10)
    with pytest.raises(ValueError):  # a raw output pointer cannot hold the tensor's 2 columns when n_cols says 3
        sg.ntt_noalloc(good, good.data_ptr(), 10, n_cols=3)
    with pytest.raises(ValueError):  # host arrays are refused
        sg.ntt_noalloc(np.zeros(n, dtype=np.uint64), np.zeros(n, dtype=np.uint64), 10)
    with pytest.raises(ValueError):
        sg.ntt_noalloc(good, good, 29)

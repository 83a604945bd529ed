"""GPU path vs the CPU oracle, through the C ABI (libstarkgpu.so).

Bit-exact equality everywhere: every value is an exact Goldilocks / Fp6
element and every proof byte must match. Sizes the oracle finishes in
seconds are compared directly; the full 2^23 domain is checked through
size-independent properties (inverse round trip, linearity, agreement with the
oracle at sampled points) and by full-proof self-verification.
"""
import hashlib
import struct

import numpy as np
import pytest

import dnszone
import oracle_lib as O

pytestmark = pytest.mark.gpu
P = O.P


def rand_field(rng, shape):
    return rng.integers(0, P, size=shape, dtype=np.uint64)


@pytest.mark.parametrize("log_n", list(range(0, 17)))
@pytest.mark.parametrize("inverse", [False, True])
def test_ntt_matches_oracle(ctx, log_n, inverse):
    rng = np.random.default_rng(100 + log_n)
    cols = 3 if log_n <= 14 else 1
    x = rand_field(rng, (cols, 1 << log_n))
    got = ctx.ntt(x, log_n, inverse)
    for c in range(cols):
        assert np.array_equal(got[c], O.ntt(x[c], inverse)), c


@pytest.mark.parametrize("log_n", [17, 20, 23, 24, 25, 26])
def test_ntt_large_round_trip_and_oracle(ctx, log_n):
    rng = np.random.default_rng(log_n)
    x = rand_field(rng, (1, 1 << log_n))
    y = ctx.ntt(x, log_n, False)
    if log_n <= 20:
        assert np.array_equal(y[0], O.ntt(x[0]))
    assert np.array_equal(ctx.ntt(y, log_n, True), x)
    # a sparse input (first 512 entries) makes the defining sum cheap on the CPU
    sp = np.zeros_like(x)
    sp[0, :512] = x[0, :512]
    ys = ctx.ntt(sp, log_n, False)
    w = int(O.lib().orc_root_of_unity(log_n))
    xs = [int(v) for v in sp[0, :512]]
    for i in (0, 1, 3, 4097, (1 << log_n) - 1):
        wi = pow(w, i, P)
        acc, p = 0, 1
        for v in xs:
            acc = (acc + v * p) % P
            p = p * wi % P
        assert int(ys[0, i]) == acc, i


def test_ntt_linearity_at_2p23(ctx):
    rng = np.random.default_rng(7)
    n = 1 << 23
    a, b = rand_field(rng, (1, n)), rand_field(rng, (1, n))
    s = ((a.astype(object) + b.astype(object)) % P).astype(np.uint64)
    fa, fb, fs = ctx.ntt(a, 23), ctx.ntt(b, 23), ctx.ntt(s, 23)
    assert np.array_equal(fs, ((fa.astype(object) + fb.astype(object)) % P).astype(np.uint64))


@pytest.mark.parametrize("w,log_n,blowup,shift", [
    (3, 3, 4, 1), (4, 7, 32, 1), (4, 12, 32, 1), (5, 10, 8, 7), (2, 16, 8, 7), (1, 1, 2, 1), (3, 13, 2, 3),
    # domains above 2^12 from at most 2^12 rows: one pass per coset
    (3, 8, 32, 1), (2, 9, 16, 5), (3, 11, 4, 3), (2, 6, 128, 1), (1, 12, 1024, 3), (2, 8, 8, 1),
    # above 2^14 points the coset twist comes from a per-size table (up to 2^20)
    (2, 10, 32, 1), (2, 11, 32, 7), (1, 10, 1024, 3),
])
def test_lde_matches_oracle(ctx, w, log_n, blowup, shift):
    rng = np.random.default_rng(w * 100 + log_n)
    tr = rand_field(rng, (w, 1 << log_n))
    assert np.array_equal(ctx.lde(tr, blowup, shift), O.lde(tr, blowup, shift))


def test_lde_reference_signature_and_errors(ctx):
    cols = [[i * 3 + c for i in range(8)] for c in range(2)]
    got = ctx.lde_trace_columns(cols, 8, 4)
    assert len(got) == 2 and len(got[0]) == 32
    assert np.array_equal(np.array(got), O.lde(np.array(cols, dtype=np.uint64), 4))
    with pytest.raises(ValueError):
        ctx.lde_trace_columns([], 8, 4)
    with pytest.raises(ValueError):
        ctx.lde_trace_columns(cols, 8, 3)
    with pytest.raises(ValueError):
        ctx.lde_trace_columns([[1] * 6], 6, 4)


def test_lde_device_pointers(ctx):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(5)
    tr = rand_field(rng, (4, 1 << 14))
    d_in = torch.from_numpy(tr.view(np.int64)).cuda()
    d_out = torch.empty((4, 1 << 17), dtype=torch.int64, device="cuda")
    ctx.lde(d_in, 8, 1, out=d_out)
    torch.cuda.synchronize()
    got = d_out.cpu().numpy().view(np.uint64)
    assert np.array_equal(got, O.lde(tr, 8, 1))


@pytest.mark.parametrize("log_nt,blowup,mode", [
    (3, 32, O.PHI_PARALLEL_GATE), (4, 32, O.PHI_ALWAYS), (7, 32, O.PHI_PARALLEL_GATE), (12, 32, O.PHI_PARALLEL_GATE),
    (10, 4, O.PHI_ALWAYS), (9, 8, O.PHI_NEVER),
])
def test_merge_hash_rollup_matches_oracle(ctx, log_nt, blowup, mode):
    rng = np.random.default_rng(log_nt)
    n_trace = 1 << log_nt
    leaves = rand_field(rng, n_trace)
    tr = O.hash_rollup_trace(leaves, n_trace)
    lde = O.lde(tr, blowup)
    want = O.merge(O.AIR_HASH_ROLLUP, lde, n_trace, blowup, [1, 2, 3], mode)
    got = ctx.merge(4, lde, n_trace, blowup, [1, 2, 3], mode)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("n,width,arities,label", [
    (1, 6, [2], 0xFE), (5, 3, [2, 2, 2], 7), (16, 8, [16], 0xFF), (100, 4, [8, 8, 8], 1), (37, 2, [4, 4, 4], 0),
    (4096, 6, [8, 8, 8, 8], 2), (1 << 14, 64, [16, 16, 16, 16], 0), (1000, 12, [4] * 5, 9),
])
def test_merkle_commit_matches_oracle(ctx, n, width, arities, label):
    rng = np.random.default_rng(n + width)
    rows = rand_field(rng, (n, width))
    cols = np.ascontiguousarray(rows.T)
    assert ctx.merkle_commit(cols, arities, label) == O.merkle_root(rows, arities, label)


def test_merkle_open_verifies(ctx):
    rng = np.random.default_rng(3)
    n, width, ar = 1000, 6, [8, 8, 8, 8]
    cols = rand_field(rng, (width, n))
    root, tree = ctx.merkle_commit(cols, ar, 5, keep=True)
    for idx in (0, 1, 511, 999):
        blob = tree.open(idx)
        leaf = hashlib.sha3_256(struct.pack("<4Q", ar[0], 0xFFFFFFFF, idx, 5) +
                                struct.pack(f"<{width}Q", *map(int, cols[:, idx]))).digest()
        assert blob[:32] == leaf
        # decode: leaf, path, index
        off = 32
        nl = int.from_bytes(blob[off:off + 8], "little"); off += 8
        path = []
        for _ in range(nl):
            ns = int.from_bytes(blob[off:off + 8], "little"); off += 8
            path.append([blob[off + 32 * k: off + 32 * (k + 1)] for k in range(ns)]); off += 32 * ns
        assert int.from_bytes(blob[off:off + 8], "little") == idx
        # recompute the root from the opening
        cur, i = blob[:32], idx
        for lv, sib in enumerate(path):
            a = ar[lv]
            ch, k = [], 0
            for j in range(a):
                if j == i % a:
                    ch.append(cur)
                else:
                    ch.append(sib[k]); k += 1
            ds = (a).to_bytes(8, "little") + (lv + 1).to_bytes(8, "little") + (i // a).to_bytes(8, "little") + (5).to_bytes(8, "little")
            cur = hashlib.sha3_256(ds + b"".join(ch)).digest()
            i //= a
        assert cur == root
    tree.free()


def _rand_params(sg, n0, pi, sched=None, cc=True):
    if sched is None:
        return sg.build_params(n0, pi), O.build_params(n0, pi)
    po = O.build_params(n0, pi)
    po.schedule_len = len(sched)
    for i, m in enumerate(sched):
        po.schedule[i] = m
    po.coeff_commit_final = int(cc)
    ps = sg.FriParams.new(sched, coeff_commit_final=cc, public_inputs_hash=pi)
    return ps, po


@pytest.mark.parametrize("log_n0", [3, 4, 5, 6, 9, 12, 13, 15, 17])
def test_stir_prove_matches_oracle_bytes(sgpu, ctx, log_n0):
    rng = np.random.default_rng(log_n0)
    n0 = 1 << log_n0
    f0 = rand_field(rng, n0)
    pi = rng.bytes(32)
    ps, po = _rand_params(sgpu, n0, pi)
    got = ctx.deep_fri_prove(f0, sgpu.FriDomain(n0), ps)
    want = O.stir_prove(f0, po)
    assert got == want


@pytest.mark.parametrize("sched,cc", [([4, 2, 8], True), ([2, 2, 2, 2], False), ([16, 4], True), ([8], True),
                                      ([8], False), ([2], True)])
def test_stir_prove_other_schedules_match_oracle(sgpu, ctx, sched, cc):
    rng = np.random.default_rng(len(sched))
    n0 = 4
    for m in sched:
        n0 *= m
    f0 = rand_field(rng, n0)
    pi = rng.bytes(32)
    ps, po = _rand_params(sgpu, n0, pi, sched, cc)
    assert ctx.deep_fri_prove(f0, n0, ps) == O.stir_prove(f0, po)


def test_stir_prove_rejects_bad_arguments(sgpu, ctx):
    f0 = np.zeros(64, dtype=np.uint64)
    with pytest.raises(sgpu.StarkGpuError):
        ctx.deep_fri_prove(f0, 64, sgpu.FriParams.new([3, 2]))
    with pytest.raises(sgpu.StarkGpuError):
        ctx.deep_fri_prove(f0, 64, sgpu.FriParams.new([8, 8, 8]))
    with pytest.raises(sgpu.StarkGpuError):  # classic branch: query count beyond the 2^20 bound
        ctx.deep_fri_prove(f0, 64, sgpu.FriParams.new([8, 8], stir=False, r=1 << 21))
    with pytest.raises(sgpu.StarkGpuError):
        ctx.deep_fri_prove(f0[:48], 48, sgpu.FriParams.new([8, 2]))


def test_golden_outer_rollup_on_gpu(ctx, golden):
    leaves, pk = dnszone.outer_rollup_inputs(golden)
    proof = ctx.prove_hash_rollup(leaves, pk)
    e = golden["outer"]
    assert len(proof) == e["len"]
    assert hashlib.sha3_256(proof).hexdigest() == e["sha3_256"]


@pytest.mark.parametrize("idx", [0, 1, 2])
def test_golden_inner_shards_on_gpu(ctx, golden, idx):
    sh = golden["shards"][idx]
    leaves, fsb, root, count = dnszone.inner_shard_inputs(golden, sh)
    proof = ctx.prove_hash_rollup(leaves, fsb)
    assert len(proof) == sh["len"]
    assert hashlib.sha3_256(proof).hexdigest() == sh["sha3_256"]
    pi = dnszone.shard_pi_hash(bytes.fromhex(golden["zone_salt_hex"]), count, root, proof[:32], fsb)
    assert pi.hex() == sh["pi_hash_hex"]


@pytest.mark.parametrize("n_leaves,mode", [(0, 0), (1, 0), (12, 1), (100, 0), (5000, 0), (5000, 2)])
def test_prove_hash_rollup_edge_sizes(ctx, n_leaves, mode):
    rng = np.random.default_rng(n_leaves)
    leaves = rand_field(rng, n_leaves)
    pi = rng.bytes(32)
    assert ctx.prove_hash_rollup(leaves, pi, mode) == O.prove_hash_rollup(leaves, pi, mode)


def test_full_size_stir_self_verifies(sgpu, ctx):
    # the 2^23 domain of the benchmark workload: too slow for the scalar oracle,
    # so check acceptance by the verifier and the OOD values against Horner on
    # the CPU for a low-degree f0
    n0 = 1 << 23
    rng = np.random.default_rng(23)
    coeffs = rand_field(rng, 1)
    f0 = np.full(n0, coeffs[0], dtype=np.uint64)  # constant polynomial: degree 0 < d_final
    pi = rng.bytes(32)
    proof = ctx.deep_fri_prove(f0, n0, sgpu.build_params(n0, pi))
    assert sgpu.deep_fri_verify(sgpu.build_params(n0, pi), proof)
    assert O.stir_verify(proof, O.build_params(n0, pi))


def test_full_size_stir_random_f0_consistent(sgpu, ctx):
    # random f0 at 2^20: not low degree, so only the prover's own values can be
    # checked; compare bytes with the oracle (multi-threaded, a few seconds)
    n0 = 1 << 20
    rng = np.random.default_rng(20)
    f0 = rand_field(rng, n0)
    pi = rng.bytes(32)
    assert ctx.deep_fri_prove(f0, n0, sgpu.build_params(n0, pi)) == O.stir_prove(f0, O.build_params(n0, pi))


def test_lde_into_three_pass_domain(ctx):
    # 2 x 2^13 -> blowup 4096 = 2^25 points: zero-padded forward three-pass transform
    rng = np.random.default_rng(25)
    tr = rand_field(rng, (2, 1 << 13))
    out = ctx.lde(tr, 1 << 12, 1)
    L = O.lib()
    w = int(L.orc_root_of_unity(25))
    for c in range(2):
        coeffs = [int(v) for v in O.ntt(tr[c], inverse=True)]
        for i in (0, 1, 4095, 4096, (1 << 25) - 1):
            x, acc = pow(w, i, P), 0
            for cf in reversed(coeffs):
                acc = (acc * x + cf) % P
            assert int(out[c, i]) == acc, (c, i)
    assert np.array_equal(out[:, ::4096], tr)  # coset 0 of the LDE is the trace itself


def _classic_params(sg, n0, pi, sched=None, cc=True):
    po = O.build_params(n0, pi, stir=False)
    if sched is None:
        return sg.build_params(n0, pi, stir=False), po
    po.schedule_len = len(sched)
    for i, m in enumerate(sched):
        po.schedule[i] = m
    po.coeff_commit_final = int(cc)
    ps = sg.FriParams.new(sched, coeff_commit_final=cc, stir=False, public_inputs_hash=pi)
    return ps, po


@pytest.mark.parametrize("log_n0,sched,cc,low", [
    (1, None, True, True), (3, None, True, True), (6, None, True, True), (10, None, True, True),
    (13, None, True, True), (16, None, True, False), (8, [4, 2, 2, 2, 2], True, True),
    (9, [8, 2, 2, 2, 2, 2, 2], False, True), (10, [16, 4, 2, 2, 2], True, True),
])
def test_classic_fri_matches_oracle(sgpu, ctx, log_n0, sched, cc, low):
    # classic DEEP-FRI branch (params.stir = false): byte-identical to the oracle; a
    # low-degree f0 also passes the library's verifier
    rng = np.random.default_rng(1000 + log_n0)
    n0 = 1 << log_n0
    if low:
        c = np.zeros(n0, dtype=np.uint64)
        c[: max(1, n0 // 32)] = rand_field(rng, max(1, n0 // 32))
        f0 = O.ntt(c)
    else:
        f0 = rand_field(rng, n0)
    pi = rng.bytes(32)
    ps, po = _classic_params(sgpu, n0, pi, sched, cc)
    got = ctx.deep_fri_prove(f0, sgpu.FriDomain(n0), ps)
    assert got == O.stir_prove(f0, po)
    if low:
        assert sgpu.deep_fri_verify(ps, got) and O.stir_verify(got, po)


@pytest.mark.parametrize("idx", [0, 1, 2])
def test_prove_inner_shard_reproduces_golden_bundle(sgpu, ctx, golden, idx):
    # prove_inner_shard from the zone's records: the proof file, pi_hash and DNS
    # merkle root of each golden shard, end to end
    sh = golden["shards"][idx]
    salt = bytes.fromhex(golden["zone_salt_hex"])
    recs = dnszone.split_evenly(dnszone.synthetic_zone(golden["record_count"]), golden["shard_count"])
    canon = [dnszone.canonical_bytes(*r) for r in recs[sh["shard_id"] - 1]]
    _, fsb, _, _ = dnszone.inner_shard_inputs(golden, sh)
    proof, pi, root = ctx.prove_inner_shard(canon, salt, fsb)
    assert len(proof) == sh["len"] and hashlib.sha3_256(proof).hexdigest() == sh["sha3_256"]
    assert pi.hex() == sh["pi_hash_hex"] and root.hex() == sh["merkle_root_hex"]


def test_prove_outer_rollup_reproduces_golden_bundle(sgpu, ctx, golden):
    pis = [bytes.fromhex(h) for h in golden["inner_pi_hashes_hex"]]
    proof = ctx.prove_outer_rollup(pis, bytes.fromhex(golden["authority_pk_hash_hex"]))
    assert hashlib.sha3_256(proof).hexdigest() == golden["outer"]["sha3_256"]


def test_prove_inner_shard_classic_fri(sgpu, ctx, golden):
    # the same shard with the classic DEEP-FRI low-degree test (LdtMode::Fri)
    sh = golden["shards"][0]
    salt = bytes.fromhex(golden["zone_salt_hex"])
    recs = dnszone.split_evenly(dnszone.synthetic_zone(golden["record_count"]), golden["shard_count"])
    canon = [dnszone.canonical_bytes(*r) for r in recs[0]]
    _, fsb, _, _ = dnszone.inner_shard_inputs(golden, sh)
    proof, pi, root = ctx.prove_inner_shard(canon, salt, fsb, stir=False)
    assert root.hex() == sh["merkle_root_hex"]
    params = sgpu.build_params(sh["n0"], fsb, stir=False)
    assert sgpu.deep_fri_verify(params, proof) and O.stir_verify(proof, O.build_params(sh["n0"], fsb, stir=False))
    assert pi == dnszone.shard_pi_hash(salt, len(canon), root, proof[:32], fsb)


def test_lde_host_input_pipelined_matches_device_input(ctx):
    # a host trace large enough to be copied in column chunks overlapped with the
    # transform (16-column chunks at 2^19 rows; 20 columns leave a partial chunk)
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(19)
    tr = rand_field(rng, (20, 1 << 19))
    pinned = torch.from_numpy(tr.view(np.int64)).pin_memory()
    d_out_host = torch.empty((20, 1 << 22), dtype=torch.int64, device="cuda")
    ctx.lde(pinned, 8, 7, out=d_out_host)
    d_out_dev = torch.empty_like(d_out_host)
    ctx.lde(pinned.cuda(), 8, 7, out=d_out_dev)
    torch.cuda.synchronize()
    assert torch.equal(d_out_host, d_out_dev)
    got = ctx.lde(tr, 8, 7)  # pageable numpy input, host output
    assert np.array_equal(got, d_out_dev.cpu().numpy().view(np.uint64))
    # spot values against the oracle's coset evaluation of column 19
    col = [int(v) for v in O.ntt(tr[19], inverse=True)]
    w = int(O.lib().orc_root_of_unity(22))
    for i in (0, 5, (1 << 22) - 1):
        x, acc = 7 * pow(w, i, P) % P, 0
        for cf in reversed(col):
            acc = (acc * x + cf) % P
        assert int(got[19, i]) == acc


@pytest.mark.parametrize("log_n", [13, 16, 20])
def test_ntt_every_four_step_split_matches_oracle(sgpu, ctx, log_n):
    # every split the autotuner may choose gives the oracle's transform, for dense
    # input and for a zero-padded LDE
    rng = np.random.default_rng(300 + log_n)
    x = rand_field(rng, (2, 1 << log_n))
    want = [O.ntt(x[c]) for c in range(2)]
    tr = rand_field(rng, (2, 1 << (log_n - 3)))
    want_lde = O.lde(tr, 8)
    try:
        for l1 in range(max(1, log_n - 12), min(12, log_n - 1) + 1):
            sgpu.ntt_set_split(log_n, False, l1)
            sgpu.ntt_set_split(log_n, True, l1)
            got = ctx.ntt(x, log_n, False)
            assert all(np.array_equal(got[c], want[c]) for c in range(2)), l1
            assert np.array_equal(ctx.lde(tr, 8, 1), want_lde), l1
    finally:
        sgpu.ntt_set_split(log_n, False, 0)
        sgpu.ntt_set_split(log_n, True, 0)
    with pytest.raises(sgpu.StarkGpuError):
        sgpu.ntt_set_split(log_n, False, 13)


def test_ntt_autotune_keeps_results(sgpu, ctx):
    rng = np.random.default_rng(9)
    x = rand_field(rng, (4, 1 << 18))
    want = ctx.ntt(x, 18, False)
    try:
        best = ctx.ntt_autotune(4, 18)
        assert 6 <= best <= 12
        assert np.array_equal(ctx.ntt(x, 18, False), want)
        best_pad = ctx.ntt_autotune(4, 21, False, 1 << 18)
        assert 9 <= best_pad <= 12
    finally:
        sgpu.ntt_set_split(18, False, 0)
        sgpu.ntt_set_split(21, True, 0)

#!/usr/bin/env python
"""Benchmark of the prover hot path on B200.

Workload (one step = one proof of the raw-kernel pipeline): 64 trace columns x
2^20 rows of uniform Goldilocks elements (seeded) -> coset LDE x8 (shift 7) to
2^23 rows -> SHA3-256 Merkle commitment over the 2^23 LDE rows (arity 16,
tree label 0) -> STIR proof of LDE column 0 with the reference's default
parameters (schedule [8]*7+[4], 54 queries, coefficient-committed final layer).
All inputs (512 MiB trace, 4 GiB LDE) exceed the 126 MB L2, so no flush is
needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0). `value` is whole-job proofs/s with the trace
resident in HBM; `e2e` is the same through the C ABI with the trace in pinned
host memory (H2D inside the timed region) and the root + proof bytes read
back. `--impl reference` times the CPU restatement of the reference prover
(the reference is Rust and cannot be built here) on a bounded sample.
"""
import argparse
import gc
import hashlib
import importlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
P = 0xFFFFFFFF00000001
W, LOG_N, BLOWUP, SHIFT = 64, 20, 8, 7
N, N0 = 1 << LOG_N, 1 << (LOG_N + 3)
ARITIES = [16] * 6          # pick_arity_for_layer(2^23, 16) / merkle_depth
TREE_LABEL = 0
PI_HASH = hashlib.sha3_256(b"stark-swarm-b200 bench seed 4").digest()
SEED = 3
METRIC = "proofs/s (64x2^20 trace -> LDE x8 -> Merkle 2^23 rows -> STIR, bit-exact)"
CONFIG = {
    "workload": "raw prover kernels: 64 cols x 2^20 rows, coset LDE blowup 8 (shift 7), "
                "SHA3-256 Merkle over 2^23 LDE rows (arity 16), STIR on LDE col 0 "
                "(schedule [8]*7+[4], s0=54, Fp6)",
    "columns": W, "rows": N, "blowup": BLOWUP, "lde_rows": N0, "hash": "SHA3-256", "field": "Goldilocks/Fp6",
    "l2": "inputs larger than L2 (512 MiB trace, 4 GiB LDE); no flush",
}


def make_trace(rank):
    rng = np.random.default_rng(SEED + 1000 * rank)
    return rng.integers(0, P, size=(W, N), dtype=np.uint64)


# ---------------------------------------------------------------- distributed
def dist_setup(ngpus):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def dist_max(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # nvidia-smi's start-up (its NVML initialisation) must not overlap the
            # timed steps: wait for its first sample, then keep sampling through them
            t0 = time.time()
            while not self.lines and self.proc.poll() is None and time.time() - t0 < 3.0:
                time.sleep(0.01)
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# Integer-pipe roofline and DRAM traffic of the dominant kernels, from ncu on the
# reduced case (4 columns, 2^20 -> 2^23; 256 MiB LDE, larger than L2), scaled to 64
# columns by the columns processed. int_frac = ALU-pipe instructions issued / peak
# over the kernel's active cycles (sm__inst_executed_pipe_alu.avg.pct_of_peak_
# sustained_active): these kernels are bound by integer issue, not by HBM.
#   ntt_pass <12,fwd> 500.6 us: ALU 64.2 %, DRAM 0.498 TB/s -> 249 MB per 4 columns
#   ntt_pass <11,fwd> 386.1 us: ALU 64.2 %, DRAM 1.275 TB/s -> 492 MB per 4 columns
#   ntt_pass <10,inv> x 2 (trace iNTT, 16-column capture): 471 MB per 16 columns
#   leaf_kernel_t<64> (2^20 rows of 64 columns) 1.489 ms: ALU 83.2 %
_LDE_TRAFFIC = (249e6 + 492e6) * 16 + 471e6 * 4  # bytes per 64-column LDE (4 launches)
MEASURED_NTT = {
    "ntt_pass": {"int_frac": 0.642, "int_metric": "ALU-pipe share of active cycles (ncu, 4-column case)",
                 "traffic_per_lde": _LDE_TRAFFIC},
    "merkle_leaves": {"int_frac": 0.832, "int_metric": "ALU-pipe share of active cycles (ncu, 2^20 x 64 leaves)"},
}
# DRAM bytes per step of the ntt_pass family: the LDE's (above) plus the STIR
# proof's transforms, taken at their algorithmic bytes times the LDE's
# measured/algorithmic ratio (their own traffic was not captured).
MEASURED_TRAFFIC_PER_STEP = {"ntt_pass": _LDE_TRAFFIC * (1 + 0.249e9 / 4.832e9)}


def run_config(ws):
    """The config dict of the JSON line, the same for both arms."""
    return dict(CONFIG, parallelism=f"{ws} independent proofs (one per GPU), no collective")


DTYPE = "u64 (Goldilocks) / Fp6"

# ---------------------------------------------------------------- CPU side
def load_oracle():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib
    return oracle_lib


def load_oracle_p256():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_p256
    return oracle_p256


def load_oracle_rsa():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_rsa
    return oracle_rsa


def cpu_sample_fraction(threads):
    """The share of one proof that a CPU sample computes: 16 of the 64 LDE columns
    (one per core on a 16-core host; 32 or all 64 on larger hosts, so that the
    column-parallel LDE keeps every core busy), and the same share of the Merkle
    rows and of the STIR domain."""
    cols = 16 if threads <= 16 else 32 if threads <= 32 else 64
    return cols / W if W == 64 else 1.0


class CpuSample:
    """A bounded sample of the step on the CPU oracle (the C++ restatement of the
    reference CPU prover, OpenMP on every host core): the LDE of `frac` of the
    trace columns, Merkle leaf + tree hashing of `frac` of the 2^23 LDE rows
    (64 columns, arity 16), and the STIR proof of a domain `frac` as large. Each
    part is `frac` of the work of the same part of the full step, so
    frac / (measured seconds) is the CPU's proofs/s, measured rather than scaled
    from a different shape."""

    def __init__(self, trace, threads):
        self.O = load_oracle()
        self.threads = threads
        self.frac = cpu_sample_fraction(threads)
        cols = max(1, int(round(W * self.frac)))
        self.lde_cols = trace[:cols]
        rows = int(N0 * self.frac)
        self.rows = np.random.default_rng(9).integers(0, P, size=(rows, W), dtype=np.uint64)
        self.f0 = np.random.default_rng(10).integers(0, P, size=rows, dtype=np.uint64)
        self.arities = [16] * max(1, (rows.bit_length() - 1 + 3) // 4)
        self.params = self.O.build_params(rows, PI_HASH)
        self.desc = (f"one {self.frac:g} share of the step per sample: oracle LDE of {cols}/{W} columns "
                     f"(2^{LOG_N} -> 2^{LOG_N + 3}), Merkle over {rows}/{N0} LDE rows of {W} columns, "
                     f"STIR at n0 {rows}")

    def run(self):
        """-> seconds for one sample"""
        O = self.O
        O.set_threads(self.threads)
        t0 = time.perf_counter()
        O.lde(self.lde_cols, BLOWUP, SHIFT)
        O.merkle_root(self.rows, self.arities, TREE_LABEL)
        O.stir_prove(self.f0, self.params)
        return time.perf_counter() - t0


def run_reference(args, ws, rank):
    """The CPU arm: rank 0 times the oracle on all host cores, one bounded sample
    per step; ms_per_step is the measured sample time and value = frac / time."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    cs = CpuSample(make_trace(0), threads)
    for _ in range(args.warmup):
        cs.run()
    t_start = time.perf_counter()
    times = [cs.run() for _ in range(args.steps)]
    wall = time.perf_counter() - t_start
    value = args.steps * cs.frac / wall
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "proofs/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * wall / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": DTYPE,
        "data": "synthetic (seeded uniform trace)", "config": run_config(ws),
        "cpu_baseline": {"value": value, "unit": "proofs/s", "cores": threads, "kind": "port",
                         "sample": cs.desc, "proofs_per_step": cs.frac},
        "e2e": {"value": value, "unit": "proofs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "sample_s": {"median": statistics.median(times), "min": min(times), "max": max(times)},
        "note": "the reference is Rust (no toolchain here); this is the C++ oracle restatement of its CPU "
                f"prover; each step proves a {cs.frac:g} share of one proof, and ms_per_step is that measured time",
    }
    print(json.dumps(line), flush=True)


def sha256_cpu_sample(threads, blocks=64):
    """Oracle time for a SHA-256 AIR proof of a `blocks`-block message (756 columns,
    blowup 32), the CPU side of the large-trace section."""
    O = load_oracle()
    O.set_threads(threads)
    msg = np.random.default_rng(blocks).integers(0, 256, blocks * 64 - 9, dtype=np.uint8).tobytes()
    t0 = time.perf_counter()
    O.prove_sha256(msg, hashlib.sha3_256(b"cpu-sample").digest())
    return time.perf_counter() - t0, 128 * blocks * 32


# ---------------------------------------------------------------- GPU side
def sha256_large(sg, ctx, blocks, reps, cpu_threads):
    """One SHA-256 AIR proof of a `blocks`-block message (8192 blocks = a 2^20-row
    trace, n0 = 2^25) through the public entry point: host message in, proof
    bytes and digest out (trace expansion, coset-sliced LDE + constraint merge,
    quotient, STIR and self-verification inside the timed call)."""
    msg = np.random.default_rng(5).integers(0, 256, blocks * 64 - 9, dtype=np.uint8).tobytes()
    fsb = hashlib.sha3_256(b"large-trace").digest()
    n_trace = 128
    while n_trace < 128 * blocks:
        n_trace *= 2
    n0 = 32 * n_trace
    ref = ctx.prove_sha256(msg, fsb)  # warm-up: memory-pool growth
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        out = ctx.prove_sha256(msg, fsb)
        times.append(time.perf_counter() - t0)
        assert out == ref, "non-deterministic proof"
    assert ref[1] == hashlib.sha256(msg).digest()
    assert sg.deep_fri_verify(sg.build_params(n0, fsb), ref[0]), "proof rejected by the verifier"
    sec = statistics.median(times)
    res = {"workload": f"SHA-256 AIR proof of a {len(msg)}-byte message ({blocks} blocks, n_trace 2^{n_trace.bit_length() - 1}, "
                       f"n0 2^{n0.bit_length() - 1}, 756 cols, 766 constraints, blowup 32), self-verified",
           "s_per_proof": sec, "proofs_per_s": 1.0 / sec, "proof_bytes": len(ref[0]), "reps": reps}
    if cpu_threads:
        t_cpu, n0_s = sha256_cpu_sample(cpu_threads)
        # prover work grows as n0 log n0 (LDE, quotient and STIR transforms dominate)
        scale = (n0 * (n0.bit_length() - 1)) / (n0_s * (n0_s.bit_length() - 1))
        est = t_cpu * scale
        res["cpu_baseline"] = {"s_per_proof": est, "cores": cpu_threads, "kind": "port", "extrapolated": True,
                               "sample": f"EXTRAPOLATED: oracle proof at n0 2^{n0_s.bit_length() - 1} took {t_cpu:.2f} s, "
                                         f"scaled by n0 log n0 (x{scale:.0f}); the full size needs "
                                         f"{756 * n0 * 8 / 2**30:.0f} GiB for the materialised LDE"}
        res["gpu_over_cpu"] = est / sec
    return res


def rsa_keys():
    """Seeded RSA-2048 test keys (n, d) shipped with the tests (tests/golden/rsa2048_keys.json)."""
    with open(os.path.join(ROOT, "tests", "golden", "rsa2048_keys.json")) as f:
        return [(int(k["n"], 16), int(k["d"], 16)) for k in json.load(f)["keys"]]


def rsa_record(sg, msg, key):
    """(n, s, em) of an RSASSA-PKCS1-v1_5 / SHA-256 signature of msg, and its pi_hash
    (prove_rsa2048_record_v1.rs recipe)."""
    n, d = key
    em = sg.rsa2048_em(msg)
    s = pow(int.from_bytes(em, "big"), d, n)
    assert sg.rsa2048_verify(n, s, em)
    return (n, s, int.from_bytes(em, "big")), sg.rsa2048_pi_record(n, s, msg, em)


def rsa2048(sg, ctx, n_jobs, stacked, cpu_threads):
    """RSA-2048 signature-check proofs (prove_rsa2048_record_v1.rs: n_trace 32,
    11041 columns, 11280 constraints, blowup 32, STIR [8,8,8,2]): one record per
    proof one at a time vs 16 in flight, and `stacked` records in one proof
    (stacked_rsa_zone_prover.rs). Inputs cross as bytes; proofs are self-verified."""
    keys = rsa_keys()
    recs = [rsa_record(sg, b"DNSSEC-RRSIG-V0|rec%05d.example.com.|A|10.0.%d.%d|epoch-0|alg-8" % (i, i // 256, i % 256),
                       keys[i % len(keys)]) for i in range(max(n_jobs, stacked))]
    jobs = [(sg.JOB_RSA2048, [r], pi) for r, pi in recs[:n_jobs]]
    ctx.prove_batch(jobs[:16], n_streams=16)
    out = {"workload": "RSA-2048 PKCS#1 v1.5 signature-check proof (e = 65537 chain, n_trace 32, 11041 cols, "
                       "11280 constraints, blowup 32, n0 1024), self-verified", "jobs": n_jobs}
    for label, streams in (("plain", 1), ("batched", 16)):
        t0 = time.perf_counter()
        res = ctx.prove_batch(jobs, n_streams=streams)
        dt = time.perf_counter() - t0
        assert all(r.status == 0 for _, r in res)
        lat = sorted(r.latency_ms for _, r in res)
        out[label] = {"streams": streams, "proofs_per_s": n_jobs / dt, "p50_ms": lat[len(lat) // 2],
                      "p99_ms": lat[min(len(lat) - 1, int(len(lat) * 0.99))]}
    out["batched_over_plain"] = out["batched"]["proofs_per_s"] / out["plain"]["proofs_per_s"]
    if stacked:
        zone = [r for r, _ in recs[:stacked]]
        pi = hashlib.sha3_256(b"stacked zone").digest()
        ctx.prove_rsa2048(zone, pi)
        t0 = time.perf_counter()
        ctx.prove_rsa2048(zone, pi)
        dt = time.perf_counter() - t0
        out["stacked"] = {"records": stacked, "ms_per_proof": dt * 1e3, "records_per_s": stacked / dt}
    if cpu_threads:
        R = load_oracle_rsa()
        O = load_oracle()
        O.set_threads(cpu_threads)
        (rec, pi) = recs[0]
        t0 = time.perf_counter()
        tr = R.trace([rec])
        cpu_proof = R.prove(tr, pi)
        dt = time.perf_counter() - t0
        assert cpu_proof == ctx.prove_rsa2048([rec], pi), "GPU and oracle RSA proofs differ"
        out["cpu_baseline"] = {"proofs_per_s": 1.0 / dt, "cores": cpu_threads, "kind": "port",
                               "sample": "one single-record proof by the oracle (trace, LDE, merge, STIR)"}
        out["plain_over_cpu"] = out["plain"]["proofs_per_s"] * dt
    return out


# P-256 test signatures (affine arithmetic over p; test data only)
P256_P = 0xFFFFFFFF00000001000000000000000000000000FFFFFFFFFFFFFFFFFFFFFFFF
P256_N = 0xFFFFFFFF00000000FFFFFFFFFFFFFFFFBCE6FAADA7179E84F3B9CAC2FC632551
P256_G = (0x6B17D1F2E12C4247F8BCE6E563A440F277037D812DEB33A0F4A13945D898C296,
          0x4FE342E2FE1A7F9B8EE7EB4A7C0F9E162BCE33576B315ECECBB6406837BF51F5)


def _p256_add(a, b):
    if a is None:
        return b
    if b is None:
        return a
    if a[0] == b[0] and (a[1] + b[1]) % P256_P == 0:
        return None
    if a == b:
        lam = (3 * a[0] * a[0] - 3) * pow(2 * a[1], -1, P256_P) % P256_P
    else:
        lam = (b[1] - a[1]) * pow(b[0] - a[0], -1, P256_P) % P256_P
    x = (lam * lam - a[0] - b[0]) % P256_P
    return x, (lam * (a[0] - x) - a[1]) % P256_P


def _p256_mul(k, pt):
    acc = None
    for bit in bin(k)[2:]:
        acc = _p256_add(acc, acc)
        if bit == "1":
            acc = _p256_add(acc, pt)
    return acc


def ecdsa_job(sg, i):
    """(q, r, s, digest) of a seeded ECDSA-P256 / SHA-256 signature, and its pi_hash."""
    rng = np.random.default_rng(1000 + i)
    d = int.from_bytes(rng.bytes(32), "big") % (P256_N - 1) + 1
    k = int.from_bytes(rng.bytes(32), "big") % (P256_N - 1) + 1
    q = _p256_mul(d, P256_G)
    digest = hashlib.sha256(b"DNSSEC-RRSIG-V0|rec%05d.example.com.|A|10.0.0.1|alg-13" % i).digest()
    e = int.from_bytes(digest, "big") % P256_N
    r = _p256_mul(k, P256_G)[0] % P256_N
    s = pow(k, -1, P256_N) * (e + r * d) % P256_N
    return (q, r, s, digest), sg.p256_ecdsa_pi(q[0], q[1], r, s, digest)


def p256_ecdsa(sg, ctx, n_jobs, cpu_threads):
    """ECDSA-P256 signature-check proofs (prove_ecdsa_record_v1.rs: the double-chain
    AIR, 256 rows of 151,334 cells and 155,774 constraints, blowup 32, n0 8192,
    STIR [8,8,8,8,2]) one at a time vs 8 in flight; each job is host signature in,
    proof bytes out, self-verified. A warm-up batch at the same concurrency grows
    the device memory pool first (it keeps freed memory), so the timed batches
    run in a server's steady state."""
    jobs = [(sg.JOB_P256_ECDSA,) + ecdsa_job(sg, i) for i in range(n_jobs)]
    ctx.prove_batch(jobs[:16], n_streams=8, hbm_budget_bytes=160 << 30)
    out = {"workload": "ECDSA-P256 signature-check proof (double-chain scalar-mult AIR, n_trace 256, 151334 cols, "
                       "155774 constraints, blowup 32, n0 8192), self-verified", "jobs": n_jobs}
    for label, streams in (("plain", 1), ("batched", 8)):
        t0 = time.perf_counter()
        res = ctx.prove_batch(jobs, n_streams=streams, hbm_budget_bytes=160 << 30)
        dt = time.perf_counter() - t0
        assert all(r.status == 0 for _, r in res)
        lat = sorted(r.latency_ms for _, r in res)
        out[label] = {"streams": streams, "proofs_per_s": n_jobs / dt, "p50_ms": lat[len(lat) // 2],
                      "p99_ms": lat[min(len(lat) - 1, int(len(lat) * 0.99))]}
    out["batched_over_plain"] = out["batched"]["proofs_per_s"] / out["plain"]["proofs_per_s"]
    if cpu_threads:
        E = load_oracle_p256()
        O = load_oracle()
        O.set_threads(cpu_threads)
        (q, r, s, digest), pi = jobs[0][1], jobs[0][2]
        u1, u2 = sg.p256_u_bits(digest, r, s)
        k = 64  # the bounded sample: the first 64 bits of each chain (n0 = 2048)
        t0 = time.perf_counter()
        tr, lay = E.trace(E.G, u1[:k], q, u2[:k])
        cpu_proof = E.prove(lay, tr, pi)
        dt = time.perf_counter() - t0
        assert cpu_proof == ctx.prove_p256_chains(E.G, u1[:k], q, u2[:k], pi), "GPU and oracle chain proofs differ"
        scale = 256 // k
        out["cpu_baseline"] = {"proofs_per_s": 1.0 / (dt * scale), "cores": cpu_threads, "kind": "port",
                               "extrapolated": True,
                               "sample": f"EXTRAPOLATED: oracle proof of the first {k} rows of both chains (n0 {k * 32}) took "
                                         f"{dt:.2f} s, scaled by n0 (x{scale}: the merge, linear in n0, dominates)"}
        out["plain_over_cpu"] = out["plain"]["proofs_per_s"] * dt * scale
    return out


# ---------------------------------------------------------------- Ed25519 inputs
# RFC 8032 section 5.1.5-5.1.6 signing, to make the benchmark's signatures (input
# generation only; the library proves and checks them).
ED_P = 2 ** 255 - 19
ED_L = 2 ** 252 + 27742317777372353535851937790883648493
ED_D = (-121665 * pow(121666, ED_P - 2, ED_P)) % ED_P


def _ed_add(p, q):
    (X1, Y1, Z1, T1), (X2, Y2, Z2, T2) = p, q
    a, b = (Y1 - X1) * (Y2 - X2) % ED_P, (Y1 + X1) * (Y2 + X2) % ED_P
    c, d = 2 * ED_D * T1 * T2 % ED_P, 2 * Z1 * Z2 % ED_P
    e, f, g, h = b - a, d - c, d + c, b + a
    return (e * f % ED_P, g * h % ED_P, f * g % ED_P, e * h % ED_P)


def _ed_mul(k, p):
    acc = (0, 1, 1, 0)
    for i in range(k.bit_length() - 1, -1, -1):
        acc = _ed_add(acc, acc)
        if (k >> i) & 1:
            acc = _ed_add(acc, p)
    return acc


def _ed_base():
    y = 4 * pow(5, ED_P - 2, ED_P) % ED_P
    x2 = (y * y - 1) * pow(ED_D * y * y + 1, ED_P - 2, ED_P) % ED_P
    x = pow(x2, (ED_P + 3) // 8, ED_P)
    if x * x % ED_P != x2:
        x = x * pow(2, (ED_P - 1) // 4, ED_P) % ED_P
    if x & 1:
        x = ED_P - x
    return (x, y, 1, x * y % ED_P)


ED_B = _ed_base()


def _ed_compress(p):
    zi = pow(p[2], ED_P - 2, ED_P)
    x, y = p[0] * zi % ED_P, p[1] * zi % ED_P
    return (y | (x & 1) << 255).to_bytes(32, "little")


def ed25519_signature(seed: bytes, msg: bytes):
    """(public key, signature R || S) of msg under the RFC 8032 key made from a 32-byte seed"""
    h = hashlib.sha512(seed).digest()
    a = (int.from_bytes(h[:32], "little") & ((1 << 254) - 8)) | (1 << 254)
    pub = _ed_compress(_ed_mul(a, ED_B))
    r = int.from_bytes(hashlib.sha512(h[32:] + msg).digest(), "little") % ED_L
    R = _ed_compress(_ed_mul(r, ED_B))
    k = int.from_bytes(hashlib.sha512(R + pub + msg).digest(), "little") % ED_L
    return pub, R + ((r + k * a) % ED_L).to_bytes(32, "little")


def ed25519_inputs(n, seed):
    """n (pub, sig, 32-byte message) with keys and messages from a seeded generator"""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        key, msg = rng.bytes(32), rng.bytes(32)
        pub, sig = ed25519_signature(key, msg)
        out.append((pub, sig, msg))
    return out


def load_oracle_ed25519():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_ed25519
    return oracle_ed25519


def ed25519(sg, ctx, n_jobs, cpu_threads):
    """Ed25519 signature-verification proofs (prove_zsk_ksk_binding_v2: the v16 verify
    AIR, k_scalar 256, 1024 rows of 41,519 cells and 70,606 constraints, blowup 32,
    n0 32768): n_jobs signatures of 32-byte messages (keys and messages from seed 5),
    one STARK per signature as in the reference, one at a time vs 8 in flight (and 8
    in flight with lockstep STIR groups of 8); each job is host signature in, proof
    bytes out, natively checked first and self-verified.
    Beside it: one proof's latency and kernel breakdown, and the CPU oracle's full-size
    proof of the same signature (measured, not scaled) next to the reference's published
    105.01 s per proof."""
    sigs = ed25519_inputs(n_jobs, 5)
    fs = hashlib.sha3_256(b"stark-swarm-b200 ed25519 fs binding").digest()
    jobs = [(sg.JOB_ED25519, s, fs) for s in sigs]
    ctx.prove_batch(jobs[:16], n_streams=8, hbm_budget_bytes=160 << 30)
    w, h, k, _rows = sg.ed25519_layout(32)
    out = {"workload": f"Ed25519 signature-verification proof (v16 verify AIR, k_scalar 256, n_trace {h}, {w} cols, "
                       f"{k} constraints, blowup 32, n0 {h * 32}), one proof per signature, self-verified",
           "jobs": n_jobs, "published_reference_s_per_proof": 105.01}
    pub, sig, msg = sigs[0]
    lat = []
    for _ in range(5):
        t0 = time.perf_counter()
        proof, _pi = ctx.prove_zsk_ksk_binding_v2(pub, sig, msg, fs, bytes(32))
        lat.append((time.perf_counter() - t0) * 1e3)
    out["single_ms"] = statistics.median(lat)
    out["proof_bytes"] = len(proof)
    sg.profile_enable(True)
    sg.profile_reset()
    ctx.prove_ed25519(pub, sig, msg, fs)
    prof = sg.profile_read()
    sg.profile_enable(False)
    out["kernels_ms"] = {kname: round(v[1], 3) for kname, v in sorted(prof.items(), key=lambda kv: -kv[1][1])[:10]}
    # grouped: 8 in flight, and each worker proves the STIR phases of up to 8 queued
    # proofs (all of n0 32768) in lockstep
    got = {}
    for label, streams, group in (("plain", 1, 1), ("batched", 8, 1), ("grouped", 8, 8)):
        ctx.set_option(sg.OPT_STIR_GROUP, group)
        try:
            t0 = time.perf_counter()
            res = ctx.prove_batch(jobs, n_streams=streams, hbm_budget_bytes=160 << 30)
            dt = time.perf_counter() - t0
        finally:
            ctx.set_option(sg.OPT_STIR_GROUP, 1)
        assert all(r.status == 0 for _, r in res)
        got[label] = [p for p, _ in res]
        ls = sorted(r.latency_ms for _, r in res)
        out[label] = {"streams": streams, "stir_group": group, "proofs_per_s": n_jobs / dt,
                      "p50_ms": ls[len(ls) // 2], "p99_ms": ls[min(len(ls) - 1, int(len(ls) * 0.99))]}
    assert got["plain"] == got["batched"] == got["grouped"], "a batched Ed25519 proof differs from the same proof alone"
    out["batched_over_plain"] = out["batched"]["proofs_per_s"] / out["plain"]["proofs_per_s"]
    out["grouped_over_plain"] = out["grouped"]["proofs_per_s"] / out["plain"]["proofs_per_s"]
    out["plain_over_published_reference"] = out["plain"]["proofs_per_s"] * 105.01
    if cpu_threads:
        E = load_oracle_ed25519()
        O = load_oracle()
        O.set_threads(cpu_threads)
        t0 = time.perf_counter()
        lay, pr, tr = E.build(pub, sig, msg, 256)
        cpu_proof = E.prove(lay, pr, tr, fs, 32)
        dt = time.perf_counter() - t0
        assert cpu_proof == proof, "GPU and oracle Ed25519 proofs differ"
        out["cpu_baseline"] = {"proofs_per_s": 1.0 / dt, "cores": cpu_threads, "kind": "port",
                               "sample": f"one full-size oracle proof of the first signature ({dt:.1f} s: trace, "
                                         f"LDE x32, merge, STIR), byte-identical to the GPU's"}
        out["plain_over_cpu"] = out["plain"]["proofs_per_s"] * dt
    return out


def serving(sg, ctx, rates, n_jobs, streams, seed=7, ed_max=32):
    """Poisson arrivals of proof requests admitted by the continuous-batching server
    under a 160 GB HBM budget: 35 % SHA-256 record proofs and 20 % SHA-512 over
    record-length messages (lognormal, median 120 B, clipped to 40-600 B), 21 %
    ECDSA-P256 and 14 % RSA-2048 signature checks (the record checks' 60/40
    signature split) and 10 % Ed25519 batches of 16-ed_max signatures (one proof
    per signature; a batch's latency is its slowest proof's); p50/p99 latency from
    submit to result, and throughput in requests and proofs against one proof at a
    time."""
    rng = np.random.default_rng(seed)
    lens = np.clip(np.round(rng.lognormal(np.log(120), 0.6, n_jobs)), 40, 600).astype(int)
    msgs = [rng.integers(0, 256, int(n), dtype=np.uint8).tobytes() for n in lens]
    u = rng.random(n_jobs)
    kinds = [sg.JOB_SHA512 if x < 0.2 else sg.JOB_ED25519 if x < 0.3 else sg.JOB_P256_ECDSA if x < 0.51
             else sg.JOB_RSA2048 if x < 0.65 else sg.JOB_SHA256 for x in u]
    pis = [hashlib.sha3_256(b"serve-%d" % i).digest() for i in range(n_jobs)]
    keys = rsa_keys()
    for i in range(n_jobs):
        if kinds[i] == sg.JOB_RSA2048:
            rec, pis[i] = rsa_record(sg, msgs[i], keys[i % len(keys)])
            msgs[i] = [rec]
        elif kinds[i] == sg.JOB_P256_ECDSA:
            msgs[i], pis[i] = ecdsa_job(sg, 50000 + i)
        elif kinds[i] == sg.JOB_ED25519:
            msgs[i] = ed25519_inputs(int(rng.integers(16, ed_max + 1)), 70000 + i)
    n_proofs = sum(len(m) if k == sg.JOB_ED25519 else 1 for k, m in zip(kinds, msgs))

    def prove_one(i):
        if kinds[i] == sg.JOB_ED25519:
            return [ctx.prove_ed25519(p, s, m, pis[i]) for p, s, m in msgs[i]]
        if kinds[i] == sg.JOB_RSA2048:
            return ctx.prove_rsa2048(msgs[i], pis[i])
        if kinds[i] == sg.JOB_P256_ECDSA:
            q, r, s, dg = msgs[i]
            return ctx.prove_p256_ecdsa(q, r, s, dg, pis[i])
        f = ctx.prove_sha512 if kinds[i] == sg.JOB_SHA512 else ctx.prove_sha256
        return f(msgs[i], pis[i])[0]

    def flat_jobs(i):
        if kinds[i] == sg.JOB_ED25519:
            return [(kinds[i], psm, pis[i]) for psm in msgs[i]]
        return [(kinds[i], msgs[i], pis[i])]

    alone = {i: prove_one(i) for i in range(12)}  # reference bytes, one at a time
    # one burst at the serving concurrency grows the device memory pool to its
    # steady-state size before anything is timed
    burst = [j for i in range(n_jobs) for j in flat_jobs(i)][:4 * streams]
    ctx.prove_batch(burst, n_streams=streams, hbm_budget_bytes=160 << 30)
    t0 = time.perf_counter()
    for i in range(n_jobs):
        prove_one(i)
    plain_s = time.perf_counter() - t0
    plain = n_jobs / plain_s
    out = {"workload": "35 % SHA-256 and 20 % SHA-512 AIR proofs of messages lognormal(median 120 B) clipped "
                       "40-600 B, 21 % ECDSA-P256 and 14 % RSA-2048 signature-check proofs, 10 % Ed25519 batches "
                       f"of 16-{ed_max} signatures (one proof each); Poisson arrivals",
           "jobs_per_rate": n_jobs, "proofs_per_rate": n_proofs, "streams": streams, "hbm_budget_gb": 160,
           "plain_proofs_per_s": n_proofs / plain_s, "plain_requests_per_s": plain, "rates": []}
    for lam in rates:
        gaps = rng.exponential(1.0 / lam, n_jobs)
        with sg.Server(ctx, n_streams=streams, hbm_budget_bytes=160 << 30) as srv:
            tickets = []
            start = time.perf_counter()
            due = start
            for i in range(n_jobs):
                due += gaps[i]
                wait = due - time.perf_counter()
                if wait > 0:
                    time.sleep(wait)
                tickets.append([(time.perf_counter(), srv.submit(*j)) for j in flat_jobs(i)])
            res, lat = [], []
            for group in tickets:
                got = [srv.wait(t) for _, t in group]
                res.append([p for p, _ in got])
                # a batch request ends with its last proof: its latency is its slowest job's
                lat.append(max((ts - group[0][0]) * 1e3 + r.latency_ms for (ts, _), (_, r) in zip(group, got)))
            wall = time.perf_counter() - start
        for i, want in alone.items():
            got = res[i] if kinds[i] == sg.JOB_ED25519 else res[i][0]
            assert got == want, "a proof in the mix differs from the same proof alone"
        lat = np.array(lat)
        out["rates"].append({"offered_per_s": lam, "requests_per_s": n_jobs / wall, "proofs_per_s": n_proofs / wall,
                             "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                             "over_plain": (n_jobs / wall) / plain})
    return out


def record_check_jobs(sg, n_jobs, seed=6, blowup=4):
    """The batched mixed-proving workload: n_jobs synthetic DNS-zone record checks
    (seeded). Each record is random bytes of lognormal length (median 120 B,
    sigma 0.6, clipped to 40-600 B) and gets two independent proofs at LDE
    blowup `blowup`: a SHA-256 AIR proof over the record bytes (1-10 blocks,
    n_trace 128-2048, with the reference's parallel-build Phi gate: Phi = 0
    below n0 = 4096) and a signature-check proof over SHA-256(record): ECDSA-P256
    (60 %, K = 256 rows) or RSA-2048 PKCS#1 v1.5 (40 %, n_trace 32)."""
    rng = np.random.default_rng(seed)
    lens = np.clip(np.round(rng.lognormal(np.log(120), 0.6, n_jobs)), 40, 600).astype(int)
    recs = [rng.integers(0, 256, int(n), dtype=np.uint8).tobytes() for n in lens]
    alg = rng.random(n_jobs)
    keys = rsa_keys()
    ecdsa_keys = []
    for i in range(16):
        d = int.from_bytes(np.random.default_rng(7000 + i).bytes(32), "big") % (P256_N - 1) + 1
        ecdsa_keys.append((d, _p256_mul(d, P256_G)))
    jobs, kinds = [], []
    for i in range(n_jobs):
        jobs.append((sg.JOB_SHA256, recs[i], hashlib.sha3_256(b"record-check-%d" % i).digest(), 0, blowup))
        kinds.append("sha256")
        digest = hashlib.sha256(recs[i]).digest()
        if alg[i] < 0.6:
            d, q = ecdsa_keys[i % 16]
            k = int.from_bytes(rng.bytes(32), "big") % (P256_N - 1) + 1
            e = int.from_bytes(digest, "big") % P256_N
            r = _p256_mul(k, P256_G)[0] % P256_N
            s_ = pow(k, -1, P256_N) * (e + r * d) % P256_N
            jobs.append((sg.JOB_P256_ECDSA, (q, r, s_, digest), sg.p256_ecdsa_pi(q[0], q[1], r, s_, digest), 0, blowup))
            kinds.append("p256_ecdsa")
        else:
            rec, pi = rsa_record(sg, recs[i], keys[i % len(keys)])
            jobs.append((sg.JOB_RSA2048, [rec], pi, 0, blowup))
            kinds.append("rsa2048")
    return jobs, kinds, lens


def record_checks(sg, ctx, n_jobs, streams):
    """Batched mixed proving: the record-check workload (2 proofs per record, blowup
    4) proved one proof at a time on one stream (the plain GPU loop) and with
    `streams` proofs in flight under a 160 GB HBM budget. Every proof of the
    batched run must equal the same proof made alone."""
    jobs, kinds, lens = record_check_jobs(sg, n_jobs)
    ctx.prove_batch(jobs[:4 * streams], n_streams=streams, hbm_budget_bytes=160 << 30)  # pool warm-up
    out = {"workload": f"{n_jobs} DNS-zone record checks (seed 6): SHA-256 AIR proof over lognormal(median 120 B, "
                       "sigma 0.6, 40-600 B) record bytes + ECDSA-P256 (60 %) or RSA-2048 (40 %) signature-check "
                       "proof, blowup 4, s0 = 54, STIR make_schedule(n0); every proof self-verified",
           "records": n_jobs, "proofs": len(jobs),
           "mix": {k: kinds.count(k) for k in sorted(set(kinds))},
           "sha256_blocks": {"min": int((lens.min() + 9 + 63) // 64), "max": int((lens.max() + 9 + 63) // 64)}}
    proofs = {}
    # plain: one proof at a time; batched: `streams` proofs in flight; grouped: the
    # same, and each worker proves the STIR phases of up to 8 queued jobs of one n0
    # in lockstep (one launch per stage for the group)
    for label, st, group in (("plain", 1, 1), ("batched", streams, 1), ("grouped", streams, 8)):
        ctx.set_option(sg.OPT_STIR_GROUP, group)
        try:
            t0 = time.perf_counter()
            res = ctx.prove_batch(jobs, n_streams=st, hbm_budget_bytes=160 << 30)
            dt = time.perf_counter() - t0
        finally:
            ctx.set_option(sg.OPT_STIR_GROUP, 1)
        assert all(r.status == 0 for _, r in res), "a record-check proof failed"
        proofs[label] = [p for p, _ in res]
        lat = sorted(r.latency_ms for _, r in res)
        out[label] = {"streams": st, "stir_group": group, "proofs_per_s": len(jobs) / dt,
                      "records_per_s": n_jobs / dt, "s": dt,
                      "p50_ms": lat[len(lat) // 2], "p99_ms": lat[min(len(lat) - 1, int(len(lat) * 0.99))]}
    assert proofs["plain"] == proofs["batched"] == proofs["grouped"], \
        "a proof in the batch differs from the same proof alone"
    out["batched_over_plain"] = out["batched"]["proofs_per_s"] / out["plain"]["proofs_per_s"]
    out["grouped_over_plain"] = out["grouped"]["proofs_per_s"] / out["plain"]["proofs_per_s"]
    out["identical_alone_and_batched"] = True
    return out


def algorithmic_bytes():
    """Minimal HBM bytes per step for each kernel family (read inputs once, write outputs once)."""
    lde = (W * N + W * N0) * 8                       # read trace, write LDE
    sizes = [N0 >> (3 * i) for i in range(8)] + [4]  # STIR layer sizes
    stir_ntt = 2 * N0 * 8 + sum(2 * 6 * s * 8 for s in sizes[1:8])
    return {
        "ntt_pass": lde + stir_ntt,
        "merkle_leaves": W * N0 * 8 + N0 * 32 + N0 * 8 + N0 * 32 + (N0 // 8) * (8 * 8 + 32),
        "stir_ood": sum((1 if i == 0 else 6) * s * 8 for i, s in enumerate(sizes[:8])),
        "stir_fold": sum((1 if i == 0 else 6) * s * 8 + 6 * (s // 8) * 8 + (s // 8) * 32 for i, s in enumerate(sizes[:7])),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sha256-jobs", type=int, default=256,
                    help="SHA-256 AIR proofs for the plain-vs-batched section (0 skips it)")
    ap.add_argument("--sha256-large-blocks", type=int, default=8192,
                    help="blocks of the large SHA-256 trace proof (8192 = 2^20 rows; 0 skips it)")
    ap.add_argument("--serve-jobs", type=int, default=200, help="jobs per arrival rate in the serving sweep (0 skips)")
    ap.add_argument("--rsa-jobs", type=int, default=256,
                    help="single-record RSA-2048 proofs for the plain-vs-batched section (0 skips it)")
    ap.add_argument("--rsa-stacked", type=int, default=64, help="records in the stacked RSA-2048 proof (0 skips)")
    ap.add_argument("--record-checks", type=int, default=1024,
                    help="records of the batched mixed-proving section (2 proofs each, blowup 4; 0 skips it)")
    ap.add_argument("--ecdsa-jobs", type=int, default=32,
                    help="ECDSA-P256 proofs for the plain-vs-batched section (0 skips it)")
    ap.add_argument("--ed25519-jobs", type=int, default=256,
                    help="Ed25519 signature proofs (config 3: 256 signatures, one proof each; 0 skips)")
    ap.add_argument("--serve-ed25519-max", type=int, default=32,
                    help="largest Ed25519 batch (signatures) in the serving mix; the full mix uses 256")
    ap.add_argument("--serve-rates", default="50,200,500,1000,2000", help="Poisson arrival rates (req/s)")
    ap.add_argument("--no-classic-fri", dest="classic_fri", action="store_false",
                    help="skip the classic DEEP-FRI timing")
    ap.add_argument("--pipeline", choices=["fused", "split"], default="split",
                    help="split: LDE, then Merkle and STIR concurrently; fused: the LDE's last pass hashes the rows "
                         "(sg_lde_commit) while column 0's LDE and its STIR proof run beside it (both are timed; "
                         "this one is the headline)")
    ap.add_argument("--columns", type=int, default=64,
                    help="trace columns (64 = the benchmark workload; fewer for small profiling captures)")
    args = ap.parse_args()
    global W
    W = args.columns
    if W != 64:
        CONFIG["workload"] = CONFIG["workload"].replace("64 cols", f"{W} cols") + " [reduced profiling case]"
        CONFIG["columns"] = W
    if args.impl == "reference":
        # CPU arm: rank 0 alone works; no process group is needed
        run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")))
        return
    ws, rank, local = dist_setup(args.gpus)

    import torch
    torch.cuda.set_device(local)
    sys.path.insert(0, ROOT)
    sg = importlib.import_module("stark-swarm_b200")
    ctx = sg.Context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    # The Merkle commitment over the LDE rows and the STIR proof of column 0 are
    # independent once the LDE exists: they run concurrently from two host
    # threads, each on its own context/stream (ctypes releases the GIL).
    ctx2 = sg.Context(local)
    from concurrent.futures import ThreadPoolExecutor
    pool = ThreadPoolExecutor(max_workers=1)

    trace = make_trace(rank)
    h_trace = torch.from_numpy(trace.view(np.int64)).pin_memory()
    d_trace = h_trace.cuda()
    d_lde = torch.empty((W, N0), dtype=torch.int64, device="cuda")
    params = sg.build_params(N0, PI_HASH)

    def commit_and_prove():
        fut = pool.submit(ctx2.deep_fri_prove, d_lde[0], N0, params)
        root = ctx.merkle_commit(d_lde, ARITIES, TREE_LABEL)
        return root, fut.result()

    def split_device():
        ctx.lde(d_trace, BLOWUP, SHIFT, out=d_lde)  # returns once the LDE is complete
        return commit_and_prove()

    def split_e2e():
        ctx.lde(h_trace, BLOWUP, SHIFT, out=d_lde)  # host (pinned) input: H2D inside the call
        return commit_and_prove()

    # fused: column 0's LDE and its STIR proof on the second context, beside the
    # LDE + row commitment of all columns whose last pass hashes the rows
    d_col0 = torch.empty((1, N0), dtype=torch.int64, device="cuda")

    def stir_col0(src):
        ctx2.lde(src, BLOWUP, SHIFT, out=d_col0)
        return ctx2.deep_fri_prove(d_col0[0], N0, params)

    def fused_device():
        fut = pool.submit(stir_col0, d_trace[0:1])
        root = ctx.lde_commit(d_trace, BLOWUP, SHIFT, ARITIES, TREE_LABEL)
        return root, fut.result()

    def fused_e2e():
        fut = pool.submit(stir_col0, h_trace[0:1])  # host (pinned) input: H2D inside the calls
        root = ctx.lde_commit(h_trace, BLOWUP, SHIFT, ARITIES, TREE_LABEL)
        return root, fut.result()

    fused = args.pipeline == "fused"
    step_device = fused_device if fused else split_device
    step_e2e = fused_e2e if fused else split_e2e

    # warm-up, and a determinism check: every step must give the same bytes, and
    # the two pipelines the same root and proof
    ref = None
    for _ in range(max(1, args.warmup)):
        out = step_device()
        assert ref is None or out == ref, "non-deterministic proof"
        ref = out
    other = split_device() if fused else fused_device()
    assert other == ref, "the fused and split pipelines disagree"
    assert sg.deep_fri_verify(params, ref[1]), "proof rejected by the verifier"
    torch.cuda.synchronize()

    # timed region (device-resident inputs); the STIR transcript's host round trips
    # sit inside each step, so no garbage-collector pause may land there
    gc.collect()
    gc.disable()
    barrier(ws)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    sg.profile_reset()
    sg.profile_enable(True)
    launches0 = ctx.kernel_launches
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    evs[0].record(stream)
    for k in range(args.steps):
        out = step_device()
        evs[k + 1].record(stream)
        assert out == ref
    torch.cuda.synchronize()
    launches_total = ctx.kernel_launches - launches0
    launches = launches_total // args.steps
    sg.profile_enable(False)
    prof = sg.profile_read()
    clk = clocks.stop()
    barrier(ws)
    step_ms = [evs[k].elapsed_time(evs[k + 1]) for k in range(args.steps)]
    total_ms = dist_max(evs[0].elapsed_time(evs[-1]), ws)
    value = ws * args.steps / (total_ms / 1000.0)

    # e2e through the C ABI with host buffers
    for _ in range(2):
        assert step_e2e() == ref
    torch.cuda.synchronize()
    barrier(ws)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        out = step_e2e()
    e1.record(stream)
    torch.cuda.synchronize()
    assert out == ref
    e2e_ms = dist_max(e0.elapsed_time(e1), ws)
    e2e_value = ws * args.steps / (e2e_ms / 1000.0)

    # the other pipeline, timed the same way, for comparison
    other_step = split_device if fused else fused_device
    e0.record(stream)
    for _ in range(args.steps):
        out = other_step()
    e1.record(stream)
    torch.cuda.synchronize()
    assert out == ref
    other_ms = dist_max(e0.elapsed_time(e1), ws) / args.steps
    other_e2e = split_e2e if fused else fused_e2e
    e0.record(stream)
    for _ in range(args.steps):
        out = other_e2e()
    e1.record(stream)
    torch.cuda.synchronize()
    assert out == ref
    other_e2e_value = ws * args.steps / (dist_max(e0.elapsed_time(e1), ws) / 1000.0)

    # LDE stage alone (trace and LDE in HBM): the NTT/LDE GB/s of the metric,
    # algorithmic bytes = read the trace once + write the LDE once; the profiler
    # gives ntt_pass's launches inside it
    sg.profile_reset()
    sg.profile_enable(True)
    e0.record(stream)
    for _ in range(args.steps):
        ctx.lde(d_trace, BLOWUP, SHIFT, out=d_lde)
    e1.record(stream)
    torch.cuda.synchronize()
    sg.profile_enable(False)
    prof_lde = sg.profile_read()
    lde_ms = dist_max(e0.elapsed_time(e1), ws) / args.steps

    # Merkle commitment of the LDE rows alone (the leaf kernel without the STIR
    # proof beside it): algorithmic bytes = read the LDE once + write the digests
    sg.profile_reset()
    sg.profile_enable(True)
    e0.record(stream)
    for _ in range(args.steps):
        ctx.merkle_commit(d_lde, ARITIES, TREE_LABEL)
    e1.record(stream)
    torch.cuda.synchronize()
    sg.profile_enable(False)
    prof_commit = sg.profile_read()
    commit_ms = dist_max(e0.elapsed_time(e1), ws) / args.steps
    gc.enable()

    # roofline of the dominant kernel family (CUDA events recorded on the launching stream)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"

    def roof(fam, profile, runs, alg_bytes_per_run, extra=None):
        """roofline entry of one kernel family from its event-timed launches"""
        if fam not in profile:
            return None
        n_l, ms = profile[fam]
        per_launch_ms = ms / n_l
        per_run = n_l / runs
        bytes_per_launch = alg_bytes_per_run / per_run
        achieved = bytes_per_launch / (per_launch_ms / 1e3) / 1e9
        r = {"bound": "hbm", "kernel": fam, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
             "frac": achieved / hbm_peak, "traffic": None, "peak_source": peak_src,
             "alg_bytes_per_launch": bytes_per_launch, "avg_launch_ms": per_launch_ms, "launches_per_step": per_run}
        r.update(extra or {})
        return r

    # ntt_pass inside the LDE alone: 4 launches per LDE (inverse 2^20: 2 passes, forward
    # 2^23: 2 passes); algorithmic bytes of the LDE = read the trace + write the LDE
    ntt_extra = {}
    if W == 64 and "ntt_pass" in MEASURED_NTT:
        ntt_extra = dict(MEASURED_NTT["ntt_pass"])
    roofline_ntt = roof("ntt_pass", prof_lde, args.steps, (W * N + W * N0) * 8, ntt_extra)
    if roofline_ntt and W == 64 and "traffic_per_lde" in ntt_extra:
        roofline_ntt["traffic"] = ntt_extra["traffic_per_lde"] / roofline_ntt["launches_per_step"]
    leaf_perms = N0 * ((4 + W) // 17 + 1)  # Keccak-f per commitment: 4 + W lanes at 17 per block, then the pad
    roofline_leaves = None
    if "merkle_leaves" in prof_commit:
        n_l, ms = prof_commit["merkle_leaves"]
        roofline_leaves = roof("merkle_leaves", prof_commit, args.steps, W * N0 * 8 + N0 * 32,
                               {"keccak_f_per_s": leaf_perms * n_l / (ms / 1e3)})
        if W == 64:
            roofline_leaves.update(MEASURED_NTT["merkle_leaves"])
    # the dominant family of the timed step
    roofline = None
    if fused and "lde_leaf" in prof:
        # reads the last pass's input once, writes one digest per row; 5 Keccak-f per
        # 64-column row (4 + 64 lanes absorbed at 17 per block, then the pad block)
        n_l, ms = prof["lde_leaf"]
        roofline = roof("lde_leaf", prof, args.steps, W * N0 * 8 + N0 * 32,
                        {"keccak_f_per_s": leaf_perms * n_l / (ms / 1e3)})
        if W == 64 and "lde_leaf" in MEASURED_NTT:
            roofline.update(MEASURED_NTT["lde_leaf"])
    elif prof:
        alg = algorithmic_bytes()
        fam = "ntt_pass" if "ntt_pass" in prof else max(prof, key=lambda k: prof[k][1])
        roofline = roof(fam, prof, args.steps, alg.get(fam, 0))
        if roofline and fam in MEASURED_TRAFFIC_PER_STEP and W == 64:
            roofline["traffic"] = MEASURED_TRAFFIC_PER_STEP[fam] / roofline["launches_per_step"]
        if roofline and fam in MEASURED_NTT and W == 64:
            roofline.update({k: v for k, v in MEASURED_NTT[fam].items() if k.startswith("int_")})
    kernels = {k: {"launches_per_step": v[0] / args.steps, "ms_per_step": v[1] / args.steps} for k, v in prof.items()}

    # The sections below characterise one GPU; with N > 1 ranks (the weak-scaling
    # run, one independent proof per GPU per step) only the main metric is taken.
    single = ws == 1

    # SHA-256 AIR proofs of seeded 64-byte messages (prove_ds_ksk_binding shape:
    # 2 blocks, n_trace 256, n0 8192): one proof at a time vs 16 in flight
    cfg1 = None
    if single and args.sha256_jobs > 0:
        rng = np.random.default_rng(1)
        jobs = [(sg.JOB_SHA256, rng.integers(0, 256, 64, dtype=np.uint8).tobytes(),
                 hashlib.sha3_256(b"cfg1-%d" % i).digest()) for i in range(args.sha256_jobs)]
        ctx.prove_batch(jobs[:16], n_streams=16)
        cfg1 = {"workload": "SHA-256 AIR proof of a 64-byte message (2 blocks, n_trace 256, n0 8192, 756 cols, "
                            "766 constraints), self-verified", "jobs": len(jobs)}
        for label, streams in (("plain", 1), ("batched", 16)):
            t0 = time.perf_counter()
            out = ctx.prove_batch(jobs, n_streams=streams)
            dt = time.perf_counter() - t0
            lat = sorted(r.latency_ms for _, r in out)
            assert all(r.status == 0 for _, r in out)
            cfg1[label] = {"streams": streams, "proofs_per_s": len(jobs) / dt,
                           "p50_ms": lat[len(lat) // 2], "p99_ms": lat[min(len(lat) - 1, int(len(lat) * 0.99))]}
        cfg1["batched_over_plain"] = cfg1["batched"]["proofs_per_s"] / cfg1["plain"]["proofs_per_s"]

    # classic DEEP-FRI (params.stir = false, the branch of the reference's published
    # scaling numbers) on the same 2^23 column, beside the STIR proof of the step
    classic = None
    if single and args.classic_fri:
        pc = sg.build_params(N0, PI_HASH, stir=False)
        ref_c = ctx.deep_fri_prove(d_lde[0], N0, pc)
        assert sg.deep_fri_verify(pc, ref_c), "classic proof rejected"
        tc = []
        for _ in range(3):
            e0.record(stream)
            out_c = ctx.deep_fri_prove(d_lde[0], N0, pc)
            e1.record(stream)
            torch.cuda.synchronize()
            tc.append(e0.elapsed_time(e1))
            assert out_c == ref_c
        ts = []
        for _ in range(3):
            e0.record(stream)
            ctx.deep_fri_prove(d_lde[0], N0, params)
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        classic = {"workload": f"deep_fri_prove of LDE column 0 (n0 = 2^{N0.bit_length() - 1}), schedule [2]*"
                               f"{N0.bit_length() - 1}, r = 54, coefficient-committed final layer",
                   "classic_ms": statistics.median(tc), "stir_ms": statistics.median(ts),
                   "classic_proof_bytes": len(ref_c)}

    cpu_threads = (os.cpu_count() or 1) if (rank == 0 and ws == 1 and not args.no_cpu_baseline) else 0
    large = sha256_large(sg, ctx, args.sha256_large_blocks, 3, cpu_threads) if single and args.sha256_large_blocks > 0 \
        else None
    rsa = rsa2048(sg, ctx, args.rsa_jobs, args.rsa_stacked, cpu_threads) if single and args.rsa_jobs > 0 else None
    ecdsa = p256_ecdsa(sg, ctx, args.ecdsa_jobs, cpu_threads) if single and args.ecdsa_jobs > 0 else None
    ed = ed25519(sg, ctx, args.ed25519_jobs, cpu_threads) if single and args.ed25519_jobs > 0 else None
    checks = record_checks(sg, ctx, args.record_checks, 16) if single and args.record_checks > 0 else None
    serve = None
    if single and args.serve_jobs > 0:
        serve = serving(sg, ctx, [float(r) for r in args.serve_rates.split(",")], args.serve_jobs, 16,
                        ed_max=args.serve_ed25519_max)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        cs = CpuSample(trace, threads)
        t_cpu = min(cs.run() for _ in range(2))
        cpu = {"value": cs.frac / t_cpu, "unit": "proofs/s", "cores": threads, "kind": "port",
               "sample": cs.desc + f"; {t_cpu:.2f} s per sample", "proofs_per_sample": cs.frac}

    if rank == 0:
        ms_step = total_ms / args.steps
        line = {
            "metric": METRIC, "value": value, "unit": "proofs/s", "n_gpus": ws, "steps": args.steps,
            "warmup": max(1, args.warmup), "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": DTYPE, "data": "synthetic (seeded uniform trace)",
            "config": run_config(ws),
            "p50_ms": statistics.median(step_ms), "p99_ms": float(np.percentile(step_ms, 99)),
            "lde_ms": lde_ms, "lde_gbs": (W * N + W * N0) * 8 / 1e9 / (lde_ms / 1e3),
            "pipeline": args.pipeline,
            "pipelines_ms_per_step": {args.pipeline: ms_step, ("split" if fused else "fused"): other_ms},
            "pipelines_e2e_proofs_per_s": {args.pipeline: e2e_value, ("split" if fused else "fused"): other_e2e_value},
            "roofline_ntt_pass": roofline_ntt,
            "commit_ms": commit_ms,
            "roofline_merkle_leaves": roofline_leaves,
            "e2e": {"value": e2e_value, "unit": "proofs/s", "h2d_bytes_per_step": W * N * 8 + (N * 8 if fused else 0),
                    "d2h_bytes_per_step": 32 + len(ref[1])},
            "gpu_launches": launches_total,  # this library's kernels in the timed region
            "gpu_launches_per_step": launches,
            "roofline": roofline,
            "kernels": kernels,
            "clocks": clk,
            "cpu_baseline": cpu,
            "sha256_proofs": cfg1,
            "sha256_large_trace": large,
            "rsa2048": rsa,
            "p256_ecdsa": ecdsa,
            "ed25519": ed,
            "record_checks": checks,
            "serving": serve,
            "classic_fri": classic,
            "proof_bytes": len(ref[1]),
            "root": ref[0].hex(),
        }
        print(json.dumps(line), flush=True)
    pool.shutdown()
    ctx2.close()
    ctx.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

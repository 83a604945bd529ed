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


# ---------------------------------------------------------------- CPU side
def load_oracle():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib
    return oracle_lib


def cpu_sample(trace, threads):
    """Time the oracle (C++ restatement of the reference CPU prover, OpenMP) on a
    bounded sample and scale to one full step: LDE of 8 of the 64 columns (x8),
    Merkle leaf+tree hashing of 2^20 of the 2^23 rows of 64 columns (x8), and
    STIR on a 2^21 domain (x4; STIR work is linear in the domain)."""
    O = load_oracle()
    O.set_threads(threads)
    t0 = time.perf_counter()
    O.lde(trace[:8], BLOWUP, SHIFT)
    t_lde = time.perf_counter() - t0
    rows = np.random.default_rng(9).integers(0, P, size=(1 << 20, W), dtype=np.uint64)
    t0 = time.perf_counter()
    O.merkle_root(rows, [16] * 5, TREE_LABEL)
    t_mk = time.perf_counter() - t0
    f0 = np.random.default_rng(10).integers(0, P, size=1 << 21, dtype=np.uint64)
    t0 = time.perf_counter()
    O.stir_prove(f0, O.build_params(1 << 21, PI_HASH))
    t_stir = time.perf_counter() - t0
    full = 8 * t_lde + 8 * t_mk + 4 * t_stir
    sample = ("oracle on 8/64 LDE columns (x8), Merkle over 2^20/2^23 rows of 64 cols (x8), STIR at 2^21 (x4); "
              f"measured {t_lde:.2f}+{t_mk:.2f}+{t_stir:.2f} s")
    return 1.0 / full, sample, t_lde + t_mk + t_stir


def run_reference(args, ws, rank):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    trace = make_trace(0)
    for _ in range(args.warmup):
        cpu_sample(trace, threads)
    vals = []
    t_start = time.perf_counter()
    for _ in range(args.steps):
        v, sample, _ = cpu_sample(trace, threads)
        vals.append(v)
    wall = time.perf_counter() - t_start
    value = statistics.median(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "proofs/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64 (Goldilocks)", "data": "synthetic (seeded uniform)",
        "config": dict(CONFIG, parallelism="rank 0 only, CPU"),
        "cpu_baseline": {"value": value, "unit": "proofs/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "proofs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "sample_wall_s": wall,
        "note": "the reference is Rust (no toolchain here); this is the C++ oracle restatement of its CPU prover",
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU side
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

    def step_device():
        ctx.lde(d_trace, BLOWUP, SHIFT, out=d_lde)  # returns once the LDE is complete
        return commit_and_prove()

    def step_e2e():
        ctx.lde(h_trace, BLOWUP, SHIFT, out=d_lde)  # host (pinned) input: H2D inside the call
        return commit_and_prove()

    # warm-up, and a determinism check: every step must give the same bytes
    ref = None
    for _ in range(max(1, args.warmup)):
        out = step_device()
        assert ref is None or out == ref, "non-deterministic proof"
        ref = out
    assert sg.deep_fri_verify(params, ref[1]), "proof rejected by the verifier"
    torch.cuda.synchronize()

    # timed region (device-resident inputs)
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
    launches = (ctx.kernel_launches - launches0) // args.steps
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

    # LDE stage alone (trace and LDE in HBM): the NTT/LDE GB/s of the metric,
    # algorithmic bytes = read the trace once + write the LDE once
    e0.record(stream)
    for _ in range(args.steps):
        ctx.lde(d_trace, BLOWUP, SHIFT, out=d_lde)
    e1.record(stream)
    torch.cuda.synchronize()
    lde_ms = dist_max(e0.elapsed_time(e1), ws) / args.steps

    # roofline of the dominant kernel family (CUDA events recorded on the launching stream)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    alg = algorithmic_bytes()
    fam = max(prof, key=lambda k: prof[k][1]) if prof else None
    roofline = None
    if fam:
        n_l, ms = prof[fam]
        per_launch_ms = ms / n_l
        launches_per_step = n_l / args.steps
        if fam in alg:
            bytes_per_launch = alg[fam] / launches_per_step
            achieved = bytes_per_launch / (per_launch_ms / 1e3) / 1e9
        else:
            bytes_per_launch, achieved = None, None
        roofline = {"bound": "hbm", "kernel": fam, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                    "frac": (achieved / hbm_peak) if achieved else None,
                    "traffic": None, "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                    "alg_bytes_per_launch": bytes_per_launch, "avg_launch_ms": per_launch_ms,
                    "launches_per_step": launches_per_step}
    kernels = {k: {"launches_per_step": v[0] / args.steps, "ms_per_step": v[1] / args.steps} for k, v in prof.items()}

    # SHA-256 AIR proofs of seeded 64-byte messages (prove_ds_ksk_binding shape:
    # 2 blocks, n_trace 256, n0 8192): one proof at a time vs 16 in flight
    cfg1 = None
    if args.sha256_jobs > 0:
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

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, sample, _ = cpu_sample(trace, threads)
        cpu = {"value": v, "unit": "proofs/s", "cores": threads, "kind": "port", "sample": sample}

    if rank == 0:
        ms_step = total_ms / args.steps
        line = {
            "metric": METRIC, "value": value, "unit": "proofs/s", "n_gpus": ws, "steps": args.steps,
            "warmup": max(1, args.warmup), "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64 (Goldilocks) / Fp6", "data": "synthetic (seeded uniform trace)",
            "config": dict(CONFIG, parallelism=f"{ws} independent proofs (one per GPU), no collective"),
            "p50_ms": statistics.median(step_ms), "p99_ms": float(np.percentile(step_ms, 99)),
            "lde_ms": lde_ms, "lde_gbs": (W * N + W * N0) * 8 / 1e9 / (lde_ms / 1e3),
            "e2e": {"value": e2e_value, "unit": "proofs/s", "h2d_bytes_per_step": W * N * 8,
                    "d2h_bytes_per_step": 32 + len(ref[1])},
            "gpu_launches": launches,
            "roofline": roofline,
            "kernels": kernels,
            "clocks": clk,
            "cpu_baseline": cpu,
            "sha256_proofs": cfg1,
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

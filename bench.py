"""Benchmark of the B200 RBF-PUM transfer (one JSON line on rank 0).

Workload (default): grid_blobs_1m -- 1,000,000 sources (500k jittered 100^3
grid cells + 500k from 64 Gaussian blobs, sigma 0.02) -> 1,000,000 uniform
targets in [0,1]^3, Wendland C4, 50 nodes per cluster, Franke 3D field,
seeded synthetic data.  One step = one full transfer (patch radius, centre
cover, membership lists, patch solves, partition-of-unity evaluation).

value: target points/s of the batched mixed-precision path with inputs
resident in HBM; e2e: the same through the host API with pinned host inputs
and the host copy of the result inside the timed region.  Inputs (56 MB) are
smaller than L2, so L2 is flushed (a 512 MB write) between timed steps,
outside the CUDA-event brackets.

N > 1 (torchrun): one transfer of the same workload sharded over the ranks
by target ranges (every rank builds the whole geometry and solves the patches
its targets need; one sum all-reduce assembles the result): strong scaling,
value = the transfer's targets / max-over-ranks time.

--impl reference times the CPU restatement of the reference algorithm (the
reference itself cannot be built here: it needs Kokkos, KokkosKernels and
ArborX) on all host threads; each step times a bounded, stratified sample of
the patch solves and estimates the whole transfer from it.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "target pts/s, 1M→1M RBF-PUM: batched FP32+refine vs plain FP64 GPU @1e-10 err"
UNIT = "target pts/s"
# int8 64x64x64 digit products per FP64-equivalent tile product of the mixed
# Cholesky: slice pairs (a, b) of 7 slices with a + b <= 9.
I8_DIGIT_PRODUCTS = sum(min(7, 9 - a) for a in range(1, 8))


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="grid_blobs_1m")
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--no-fp64-compare", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the many-uneven-transfers measurement (256 problems per call)")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--kernels-only", action="store_true",
                    help="run warmup + steps transfers and exit (for ncu launch lists)")
    ap.add_argument("--with-adjoint", action="store_true",
                    help="with --kernels-only: each step also runs the adjoint (values and "
                         "target coordinates) of a saved execute")
    ap.add_argument("--with-fe", action="store_true",
                    help="with --kernels-only: each step also runs the NEAREST_NEAREST "
                         "finite-element transfer of the same points")
    ap.add_argument("--with-mls", action="store_true",
                    help="with --kernels-only: each step also runs the moving least squares "
                         "transfer of the same points")
    ap.add_argument("--mls-only", action="store_true",
                    help="with --kernels-only: run only the moving least squares transfers")
    ap.add_argument("--configs", action="store_true",
                    help="one line per configuration of the baseline table (GPU in both "
                         "precisions, the CPU restatement in Serial and OpenMP, errors)")
    return ap.parse_args()


def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (CPU restatement), bounded sample
# ---------------------------------------------------------------------------

def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(w, seconds_budget: float, threads: int | None = None):
    """Times the CPU restatement on a bounded sample: the full geometry phase,
    then the patch solves of a stratified random sample (by patch size), whose
    time is scaled by the inverse sampling fraction of each stratum, plus one
    partition-of-unity pass.  Returns (pts_per_s, description, threads,
    seconds spent, estimated seconds per transfer)."""
    import oracle
    threads = oracle.set_threads(threads or os.cpu_count() or 1)
    t_start = time.perf_counter()
    t0 = time.perf_counter()
    plan = oracle.build(3, w["src"], w["tgt"], w["nodes_per_cluster"])
    t_geom = time.perf_counter() - t0
    off, _ = plan.src_csr()
    toff, _ = plan.tgt_csr()
    n = np.diff(off)
    mt = np.diff(toff)
    live = mt > 0
    # Work proxy of a patch (factorisation ~n^3, evaluation ~m n): within a
    # stratum the sampled time is scaled by the proxy's sum rather than by
    # the patch count, which cuts the variance of small samples of large
    # patches (their time grows as n^3 across the stratum).
    cost = n.astype(np.float64) ** 3 + 3.0 * n.astype(np.float64) * mt
    K = int(live.sum())
    rng = np.random.default_rng(0)
    edges = [0, 64, 128, 256, 512, 1024, 2048, 1 << 30]
    total = 0.0
    sampled = 0
    budget_each = seconds_budget / (len(edges) - 1)
    vals = w["values"]
    # Every solve call also makes one partition-of-unity pass over all targets
    # (and zeroes the output): timed once with no patches, it is taken off
    # each sampled call and counted once per transfer below.
    calls0 = []
    for _ in range(3):
        t1 = time.perf_counter()
        plan.solve(w["basis"], vals, patch_list=np.zeros(0, dtype=np.int64))
        calls0.append(time.perf_counter() - t1)
    t_call = float(np.median(calls0))
    for lo, hi in zip(edges[:-1], edges[1:]):
        ids = np.where((n > lo) & (n <= hi) & live)[0]
        if len(ids) == 0:
            continue
        rng.shuffle(ids)
        # Grow the sample until the stratum's time budget is used; the calls'
        # fixed cost is taken off the stratum's sum (not per call, so that
        # its noise averages out).
        # At least one patch per thread per call: the restatement runs the
        # patches of a call in parallel, one per thread, as the full
        # transfer does.
        take = min(len(ids), max(threads, min(len(ids) // 64, 64) if lo < 512 else 1))
        raw = 0.0
        calls = 0
        done = 0
        while done < len(ids) and raw - calls * t_call < budget_each:
            chunk = ids[done:done + take]
            t1 = time.perf_counter()
            plan.solve(w["basis"], vals, patch_list=chunk)
            raw += time.perf_counter() - t1
            calls += 1
            done += len(chunk)
            take = min(take * 2, len(ids) - done) if done < len(ids) else take
        total += max(raw - calls * t_call, 0.0) * cost[ids].sum() / cost[ids[:done]].sum()
        sampled += done
    t_pu = t_call
    est = t_geom + total + t_pu
    m = w["tgt"].shape[0]
    desc = (f"CPU restatement of the reference algorithm (FP64, unpivoted LU; the reference "
            f"itself needs Kokkos/KokkosKernels/ArborX), {threads} thread(s) on {cpu_model()}: "
            f"full geometry ({t_geom:.2f}s) + patch solves of a stratified sample of "
            f"{sampled}/{K} patches ({100.0 * sampled / max(K, 1):.1f}%) scaled per size stratum "
            f"({total:.1f}s est.) + PU pass ({t_pu:.2f}s); estimated {est:.1f}s per transfer")
    return m / est, desc, threads, time.perf_counter() - t_start, est


def run_reference(args):
    """The reference arm: the CPU restatement on all host threads.  A warm-up
    step solves a small sample untimed; each timed step is one bounded
    estimator pass (a stratified sample of the patch solves, about
    min(30, 150 / steps) seconds), whose estimate of the whole transfer gives
    the step's throughput.  ms_per_step is the time a step actually took."""
    rank, world, _ = dist_info()
    if rank != 0:
        return
    args.world = world
    from pacman_b200 import workloads as W
    w = W.make(args.workload, args.scale)
    for _ in range(args.warmup):
        cpu_baseline(w, 0.5)
    budget = max(3.0, min(args.cpu_seconds, 30.0, 150.0 / max(args.steps, 1)))
    vals, spent, ests = [], [], []
    desc, threads = "", 1
    for _ in range(max(args.steps, 1)):
        v, desc, threads, sec, est = cpu_baseline(w, budget)
        vals.append(v)
        spent.append(sec)
        ests.append(est)
    value = statistics.median(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(spent) / len(spent),
        "estimated_ms_per_transfer": 1e3 * statistics.median(ests),
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded numpy generators)",
        "config": config_dict(args, w),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"each step: {desc}"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config_dict(args, w):
    return {"workload": f"{args.workload}: {w['src'].shape[0]} sources (jittered 100^3 grid + 64 "
                        f"Gaussian blobs) -> {w['tgt'].shape[0]} uniform targets, Wendland C4, "
                        f"{w['values'].shape[1]} field(s), 50 nodes/cluster, overlap 0.15, "
                        f"support 0.1" if args.workload == "grid_blobs_1m" else args.workload,
            "n_source": int(w["src"].shape[0]), "n_target": int(w["tgt"].shape[0]),
            "fields": int(w["values"].shape[1]), "basis": "WendlandC4" if w["basis"] == 0x12 else hex(w["basis"]),
            "precision": args.precision, "l2": "flushed between timed steps (512 MB write)",
            "parallelism": (f"targets sharded over {args.world} GPUs (global geometry per rank, "
                            "Morton ranges balanced by patch cost, sum all-reduce of the outputs)"
                            if getattr(args, "world", 1) > 1 else "one GPU")}


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi samples of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi's start-up (NVML initialisation) goes before the
            # timed region: wait for its first sample.
            t0 = time.perf_counter()
            while not self.lines and time.perf_counter() - t0 < 3.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            parts = [p.strip() for p in l.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def fp64_gemm_peak(torch, dev):
    """Measured FP64 denominator: cuBLAS DGEMM 8192^3 (2 N^3 flops), best of 5."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def measured_peaks():
    """HBM GB/s and dense bf16 TFLOP/s (burst, sustained) measured on this
    pool's B200s (MEASURED_PEAKS.json, written beside this file by the
    pipeline), else the pool's earlier measurement; with the source named."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))

        def pick(*keys):
            for k in keys:
                v = d.get(k)
                if isinstance(v, dict):
                    v = v.get("value")
                if isinstance(v, (int, float)) and v > 0:
                    return float(v)
            return None
        hbm = pick("hbm_gbs", "hbm_GBs", "hbm_copy_gbs")
        bf16 = pick("bf16_tflops", "bf16_dense_tflops")
        bf16s = pick("bf16_tflops_sustained") or bf16
        if hbm and bf16:
            return {"hbm_gbs": hbm, "bf16_tflops": bf16, "bf16_tflops_sustained": bf16s,
                    "source": "measured (MEASURED_PEAKS.json)"}
    except (OSError, ValueError):
        pass
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0,
            "source": "fallback (an earlier B200 measurement: 6.65 TB/s copy, 1.59 PFLOP/s "
                      "bf16 burst, ~1.4 sustained)"}


def read_profile_value(key: str):
    """A figure from the committed ncu summaries (a line '<key>: <number>'
    in profiles/*.txt), or None."""
    import glob
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.txt"))):
        for line in open(path):
            if line.startswith(key + ":"):
                try:
                    return float(line.split(":", 1)[1].strip().split()[0])
                except ValueError:
                    return None
    return None


def run_configs(args):
    """The five configurations of the baseline table, one JSON line each: GPU
    time per transfer in both precisions (device-resident inputs, CUDA events,
    median after warm-up), the CPU restatement of the reference algorithm with
    1 thread (Serial) and all host threads (OpenMP) -- in full where it runs in
    seconds, else estimated from a bounded stratified sample -- and relative L2
    errors (against the oracle in full where it runs, else mixed vs FP64)."""
    import torch
    import oracle
    import pacman_b200 as pacman
    from pacman_b200 import workloads as W
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    nthreads = os.cpu_count() or 1
    base = {"cpu_model": cpu_model(), "host_threads": nthreads}

    def gpu_ms(fn, reps, warm=3):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)

    def transfer_case(name, w, basis, reps, full_oracle):
        S = torch.tensor(w["src"], device=dev)
        T = torch.tensor(w["tgt"], device=dev)
        vals = w["values"][:, 0] if w["values"].shape[1] == 1 else w["values"]
        V = torch.tensor(vals, device=dev)
        npc = w["nodes_per_cluster"]
        line = dict(base, config=name, n_source=int(S.shape[0]), n_target=int(T.shape[0]),
                    fields=int(w["values"].shape[1]), basis=hex(basis))
        outs = {}
        for prec in ("mixed", "fp64"):
            f = lambda: pacman.rbf.interpolate(3, 3, basis, S, V, T, nodes_per_cluster=npc,
                                               precision=prec)
            line[f"gpu_{prec}_ms"] = gpu_ms(f, reps)
            outs[prec] = f().cpu().numpy()
        m = w["tgt"].shape[0]
        line["gpu_mixed_pts_s"] = m / (line["gpu_mixed_ms"] * 1e-3)
        line["gpu_fp64_pts_s"] = m / (line["gpu_fp64_ms"] * 1e-3)
        line["mixed_over_fp64"] = line["gpu_fp64_ms"] / line["gpu_mixed_ms"]
        line["rel_l2_mixed_vs_fp64"] = float(np.linalg.norm(outs["mixed"] - outs["fp64"]) /
                                             np.linalg.norm(outs["fp64"]))
        ww = dict(w, basis=basis)
        if full_oracle:
            for label, th in (("serial", 1), ("openmp", nthreads)):
                oracle.set_threads(th)
                t0 = time.perf_counter()
                ref = oracle.interpolate(3, basis, w["src"], vals, w["tgt"], npc)
                line[f"oracle_{label}_s"] = time.perf_counter() - t0
            for prec in ("mixed", "fp64"):
                line[f"rel_l2_{prec}_vs_oracle"] = float(np.linalg.norm(outs[prec] - ref) /
                                                         np.linalg.norm(ref))
            line["oracle_kind"] = "full transfer"
        else:
            _, desc, _, _, est = cpu_baseline(ww, 20.0)
            _, desc1, _, _, est1 = cpu_baseline(ww, 10.0, threads=1)
            line["oracle_openmp_s"] = est
            line["oracle_serial_s"] = est1
            line["oracle_kind"] = "estimated: " + desc + " | " + desc1
        print(json.dumps(line), flush=True)
        return line

    transfer_case("1: 20k -> 20k uniform, C2", W.make("uniform_20k"), W.WENDLANDC2, 10, True)
    transfer_case("2: 1M -> 1M grid + blobs, C4", W.make("grid_blobs_1m"), W.WENDLANDC4, 5,
                  False)
    shell = W.make("shell_4m")
    for b in (W.WENDLANDC2, W.WENDLANDC4, W.WENDLANDC6):
        transfer_case(f"3: 4M -> 2M shell + cube, 8 fields, {hex(b)}", shell, b, 3, False)
    # 4: adjoint workload: forward (saved) + adjoint of values and target
    # coordinates; the oracle times the forward transfer.
    w = W.make("uniform_500k")
    S = torch.tensor(w["src"], device=dev)
    T = torch.tensor(w["tgt"], device=dev)
    V = torch.tensor(w["values"], device=dev)
    G = torch.randn(T.shape[0], V.shape[1], dtype=torch.float64, device=dev,
                    generator=torch.Generator(device=dev).manual_seed(7))
    line = dict(base, config="4: 500k -> 500k uniform, C4, 4 fields, adjoint")
    grads = {}
    for prec in ("mixed", "fp64"):
        plan = pacman.rbf.Plan(3, S, T, precision=prec)
        line[f"gpu_{prec}_forward_ms"] = gpu_ms(
            lambda: plan.execute(W.WENDLANDC4, V, save_for_adjoint=True), 5)
        line[f"gpu_{prec}_adjoint_ms"] = gpu_ms(lambda: plan.adjoint(G), 5)
        grads[prec] = [g.cpu().numpy() for g in plan.adjoint(G)]
        plan.close()
    line["rel_l2_grad_values_mixed_vs_fp64"] = float(
        np.linalg.norm(grads["mixed"][0] - grads["fp64"][0]) / np.linalg.norm(grads["fp64"][0]))
    line["rel_l2_grad_targets_mixed_vs_fp64"] = float(
        np.linalg.norm(grads["mixed"][1] - grads["fp64"][1]) / np.linalg.norm(grads["fp64"][1]))
    for label, th in (("serial", 1), ("openmp", nthreads)):
        oracle.set_threads(th)
        t0 = time.perf_counter()
        oracle.interpolate(3, W.WENDLANDC4, w["src"], w["values"], w["tgt"], 50)
        line[f"oracle_forward_{label}_s"] = time.perf_counter() - t0
    print(json.dumps(line), flush=True)
    # 5: many uneven problems in one batched call; the oracle runs a random
    # 32 of them in full, scaled by the targets of all.
    probs = W.many_problems(count=256)
    bP = [(3, q["basis"], torch.tensor(q["src"], device=dev),
           torch.tensor(q["values"] if q["values"].shape[1] > 1 else q["values"][:, 0],
                        device=dev), torch.tensor(q["tgt"], device=dev)) for q in probs]
    tot = sum(q["tgt"].shape[0] for q in probs)
    line = dict(base, config="5: 256 uneven problems, C0-C8, 1-4 fields", targets=int(tot))
    for prec in ("mixed", "fp64"):
        ms = gpu_ms(lambda: pacman.rbf.interpolate_batch(bP, precision=prec), 3, warm=1)
        line[f"gpu_{prec}_ms"] = ms
        line[f"gpu_{prec}_pts_s"] = tot / (ms * 1e-3)
    pick = np.random.default_rng(3).choice(len(probs), size=32, replace=False)
    sub = sum(probs[i]["tgt"].shape[0] for i in pick)
    for label, th in (("serial", 1), ("openmp", nthreads)):
        oracle.set_threads(th)
        t0 = time.perf_counter()
        for i in pick:
            q = probs[i]
            oracle.interpolate(3, q["basis"], q["src"], q["values"], q["tgt"], 50)
        line[f"oracle_{label}_s"] = (time.perf_counter() - t0) * tot / sub
    line["oracle_kind"] = f"32 of 256 problems in full, scaled by targets ({sub} of {tot})"
    print(json.dumps(line), flush=True)


def measure_mls(pacman, S, V0, T, timed, steps):
    """Moving least squares transfer of device-resident points and one field:
    one warm call, then the median of `steps` timed calls."""
    pacman.MLS.interpolate(3, pacman.execspaces.CUDA, S, V0, T)
    mt = timed(lambda: pacman.MLS.interpolate(3, pacman.execspaces.CUDA, S, V0, T), steps)
    mms = statistics.median(mt)
    return {"value": T.shape[0] / (mms * 1e-3), "unit": UNIT, "ms_per_call": mms,
            "what": "pacman.MLS.interpolate, same sources, targets and first field, "
                    "device-resident (k_mls: 10-nearest search, Jacobi pseudo-inverse of the "
                    "10 x 10 moment matrix)"}


def mls_cpu_baseline(w):
    """The CPU restatement of the moving least squares transfer (cell-grid
    neighbour search, the same fit per target) over the whole workload with
    every host thread."""
    import oracle
    threads = oracle.set_threads(os.cpu_count() or 1)
    t0 = time.perf_counter()
    oracle.mls_interpolate(3, w["src"], w["values"][:, 0], w["tgt"])
    sec = time.perf_counter() - t0
    return {"value": w["tgt"].shape[0] / sec, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"the whole transfer, {sec:.2f} s"}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.configs:
        return run_configs(args)
    import torch
    import torch.distributed as dist
    import pacman_b200 as pacman
    from pacman_b200 import workloads as W

    rank, world, local = dist_info()
    args.world = world
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=dev)
    w = W.make(args.workload, args.scale)
    m = w["tgt"].shape[0]
    F = w["values"].shape[1]
    vals_np = w["values"][:, 0] if F == 1 else w["values"]
    S = torch.tensor(w["src"], device=dev)
    T = torch.tensor(w["tgt"], device=dev)
    V = torch.tensor(vals_np, device=dev)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    kw = dict(nodes_per_cluster=w["nodes_per_cluster"])
    stream = torch.cuda.current_stream(dev)

    def step(precision, stats=None):
        if world > 1:  # one transfer, targets sharded over the ranks
            return pacman.distributed.interpolate_sharded(3, w["basis"], S, V, T,
                                                          precision=precision, stats=stats, **kw)
        return pacman.rbf.interpolate(3, pacman.execspaces.CUDA, w["basis"], S, V, T,
                                      precision=precision, stats=stats, **kw)

    def barrier():
        if world > 1:
            dist.barrier()

    def timed(fn, steps):
        times = []
        for _ in range(steps):
            flush.zero_()
            barrier()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            barrier()
            times.append(e0.elapsed_time(e1))
        return times

    for _ in range(args.warmup):
        step(args.precision)
    torch.cuda.synchronize()
    if args.kernels_only:
        st = {}
        plan = None
        if args.with_adjoint:
            plan = pacman.rbf.Plan(3, S, T, precision=args.precision, **kw)
            G = torch.ones_like(V)
        V0 = V if V.dim() == 1 else V[:, 0].contiguous()
        for _ in range(args.steps):
            if args.with_mls or args.mls_only:
                pacman.MLS.interpolate(3, pacman.execspaces.CUDA, S, V0, T)
            if args.mls_only:
                continue
            step(args.precision, st)
            if plan is not None:
                plan.execute(w["basis"], V, save_for_adjoint=True)
                plan.adjoint(G)
            if args.with_fe:
                pacman.fe.interpolate(3, pacman.execspaces.CUDA, 0xF0, S,
                                      V if V.dim() == 1 else V[:, 0].contiguous(), None, None,
                                      None, T)
        torch.cuda.synchronize()
        if rank == 0:
            print(json.dumps({"kernels_only": True, "steps": args.steps, "stats": st}), flush=True)
        return
    stats = {}
    with ClockSampler(local) as clk:
        times = timed(lambda: step(args.precision, stats), args.steps)
    total_ms = sum(times)
    if world > 1:
        t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = m * args.steps / (total_ms * 1e-3)  # one transfer, whatever the rank count
    ms_per_step = total_ms / args.steps

    # End to end through the host API: pinned host inputs, host result.
    hS = torch.from_numpy(w["src"]).pin_memory()
    hT = torch.from_numpy(w["tgt"]).pin_memory()
    hV = torch.from_numpy(np.ascontiguousarray(vals_np)).pin_memory()
    hO = torch.empty((m,) if F == 1 else (m, F), dtype=torch.float64).pin_memory()
    sp_np, tp_np, v_np, o_np = hS.numpy(), hT.numpy(), hV.numpy(), hO.numpy()

    def e2e_step():
        if world > 1:
            out = pacman.distributed.interpolate_sharded(3, w["basis"], sp_np, v_np, tp_np,
                                                         precision=args.precision, **kw)
        else:
            out = pacman.rbf.interpolate(3, pacman.execspaces.CUDA, w["basis"], sp_np, v_np,
                                         tp_np, precision=args.precision,
                                         stream=stream.cuda_stream, **kw)
        o_np[...] = out

    e2e_step()
    e2e_times = timed(e2e_step, args.steps)
    e2e_ms = sum(e2e_times) / len(e2e_times)
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    h2d = (w["src"].nbytes + w["tgt"].nbytes + np.ascontiguousarray(vals_np).nbytes)
    d2h = o_np.nbytes

    # Plain FP64 path (the reference's unpivoted-LU algorithm) over the same
    # number of timed steps, and the agreement of the two paths.
    extra = {"ms_per_step_median": statistics.median(times),
             "e2e_ms_per_step_median": statistics.median(e2e_times),
             "step_ms": [round(t, 3) for t in times],
             "e2e_step_ms": [round(t, 3) for t in e2e_times]}
    if not args.no_fp64_compare:
        out_mixed = step(args.precision).cpu().numpy()
        f64_stats = {}
        step("fp64")
        f64_times = timed(lambda: step("fp64", f64_stats), args.steps)
        out64 = step("fp64").cpu().numpy()
        f64_ms = sum(f64_times) / len(f64_times)
        if world > 1:
            t = torch.tensor([f64_ms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            f64_ms = float(t.item())
        extra["fp64_value"] = m / (f64_ms * 1e-3)
        extra["fp64_ms_per_step"] = f64_ms
        extra["fp64_ms_per_step_median"] = statistics.median(f64_times)
        extra["mixed_over_fp64"] = extra["fp64_value"] and value / extra["fp64_value"]
        extra["mixed_over_fp64_median"] = (statistics.median(f64_times) /
                                           statistics.median(times))
        extra["rel_l2_mixed_vs_fp64"] = float(np.linalg.norm(out_mixed - out64) / np.linalg.norm(out64))
        extra["fp64_ms_factor"] = f64_stats.get("ms_factor")

    # A coupling loop's repeated transfer over fixed points: a plan that keeps
    # its factorisations re-executes with only the polynomial block, the
    # triangular solves and the evaluation.
    if args.precision == "mixed":
        rplan = pacman.rbf.Plan(3, S, T, precision=args.precision, **kw)
        rplan.execute(w["basis"], V, keep_factors=True)
        rst = {}
        r_times = timed(lambda: rplan.execute(w["basis"], V, stats=rst, keep_factors=True),
                        max(1, args.steps))
        rplan.close()
        r_ms = sum(r_times) / len(r_times)
        extra["reexecute"] = {
            "value": m / (r_ms * 1e-3), "unit": UNIT, "ms_per_step": r_ms,
            "factors_reused": rst.get("factors_reused"),
            "what": "Plan.execute(keep_factors=True) after a factorising execute: geometry "
                    "and patch factorisations kept, values new each step"}

    # Many uneven transfers in one call: 256 independent problems (sources
    # log-uniform in [1000, 50000], uniform in boxes of side 0.5-2, bases
    # C0..C8, 1-4 fields), device-resident, through interpolate_batch.
    if world == 1 and not args.no_batch and args.scale == 1.0:
        probs = W.many_problems(count=256)
        bP = [(3, q["basis"], torch.tensor(q["src"], device=dev),
               torch.tensor(q["values"] if q["values"].shape[1] > 1 else q["values"][:, 0],
                            device=dev),
               torch.tensor(q["tgt"], device=dev)) for q in probs]
        btot = sum(q["tgt"].shape[0] for q in probs)
        batch = {"problems": len(probs), "targets": int(btot), "unit": UNIT}
        for prec in ("mixed", "fp64"):
            pacman.rbf.interpolate_batch(bP, precision=prec)
            bt = timed(lambda: pacman.rbf.interpolate_batch(bP, precision=prec), 2)
            bms = sum(bt) / len(bt)
            batch[prec] = {"value": btot / (bms * 1e-3), "ms_per_call": bms}
        extra["many_uneven_256"] = batch

    # Moving least squares (pacman.MLS.interpolate) over the same points and
    # the first field, device-resident: K = 10 nearest sources, a quadratic
    # weighted least-squares fit per target.
    if world == 1 and not args.no_batch and args.scale == 1.0:
        extra["mls"] = measure_mls(pacman, S, V if V.dim() == 1 else V[:, 0].contiguous(), T,
                                   timed, max(3, args.steps))

    # Roofline of the dominant kernel: the int8 step kernel of the large-patch
    # Cholesky (k_col_step_ws).  One extra transfer after the timed region,
    # in the timed configuration (all slot groups on their streams), with CUDA
    # events around every step launch on the stream it runs on; the span of
    # each kind is the union of its launch intervals.
    peaks = measured_peaks()
    dgemm = fp64_gemm_peak(torch, dev)
    kst = {}
    plan = pacman.rbf.Plan(3, S, T, precision=args.precision, **kw)
    plan.execute(w["basis"], V, stats=kst, time_kernels=True)
    plan.close()
    tile_flops = 2.0 * 64 ** 3
    ms_i8 = kst.get("ms_update_i8", 0.0)
    prod_i8 = kst.get("mma_products_i8", 0.0)
    ms_f64 = kst.get("ms_update_f64", 0.0)
    # Algorithmic work of one int8 tile product: 34 int8 digit products of
    # 64x64x64 (slice pairs a + b <= 9 of 7 slices) and the 7 int8 slices of
    # one 64x64 L tile read from HBM (the shared tile row comes from L2).
    i8_ops = prod_i8 * I8_DIGIT_PRODUCTS * tile_flops
    i8_bytes = prod_i8 * 7 * 64 * 64
    int8_peak = 2.0 * peaks["bf16_tflops"]
    nl = max(1, int(kst.get("update_launches_i8", 0)))
    ach = i8_ops / (ms_i8 * 1e-3) / 1e12 if ms_i8 else 0.0
    hbm_ach = i8_bytes / (ms_i8 * 1e-3) / 1e9 if ms_i8 else 0.0
    traffic_per_product = read_profile_value("dram_bytes_per_tile_product[k_col_step_ws]")
    roofline = {
        "bound": "tensor",
        "kernel": "k_col_step_ws (left-looking Cholesky step of the large patches: column "
                  "update on the int8 tensor cores, tcgen05.mma kind::i8, 7-slice split-integer "
                  "FP64 emulation, levels 2..9; triangular solve; next diagonal tile)",
        "achieved": ach, "peak": int8_peak, "unit": "TFLOP/s",
        "frac": ach / int8_peak if int8_peak else None,
        "peak_source": "int8 dense = 2 x bf16 dense, " + peaks["source"]
                       + " (derived: int8 throughput itself is not measured)",
        "traffic": (traffic_per_product * prod_i8 / nl) if traffic_per_product else None,
        "algorithmic_bytes_per_launch": i8_bytes / nl,
        "hbm": {"achieved_gbs": hbm_ach, "peak_gbs": peaks["hbm_gbs"],
                "frac": hbm_ach / peaks["hbm_gbs"]},
        "tile_products_per_launch": prod_i8 / nl,
        "ms_per_launch": ms_i8 / nl,
        "launches_per_step": nl,
        "ms_span_per_step": ms_i8,
        "share_of_step": ms_i8 / ms_per_step if ms_per_step else None,
        "fp64_steps": {
            "kernel": "k_col_step<1> (the tile columns below PACMAN_B200_INT8_FROM, none "
                      "with the tuned B200 setting: column update on the FP64 tensor cores, "
                      "mma.sync f64)",
            "achieved": kst.get("update_flops_f64", 0.0) / (ms_f64 * 1e-3) / 1e12 if ms_f64 else 0,
            "peak": dgemm, "unit": "TFLOP/s",
            "peak_source": "measured live: cuBLAS DGEMM 8192^3 on this GPU",
            "launches_per_step": int(kst.get("update_launches_f64", 0)),
            "ms_span_per_step": ms_f64},
    }
    if roofline["fp64_steps"]["peak"]:
        roofline["fp64_steps"]["frac"] = roofline["fp64_steps"]["achieved"] / dgemm

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None,
        "dtype": "f64/i8" if args.precision == "mixed" else "f64",
        "data": "synthetic (seeded numpy generators; no public data set)",
        "config": config_dict(args, w),
        "e2e": {"value": m / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(stats.get("kernel_launches", 0)) * args.steps,
        "host_syncs_per_step": int(stats.get("host_syncs", 0)),
        "clocks": clk.summary(),
        "roofline": roofline,
        "stats": {k: stats.get(k) for k in ("radius", "num_patches", "sum_n", "sum_m", "max_n",
                                            "patches_fp32", "patches_fp64", "patches_fallback",
                                            "ms_geometry", "ms_solve", "ms_factor")},
        **extra,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, desc, threads, _, _ = cpu_baseline(w, args.cpu_seconds)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": desc}
        v1, desc1, _, _, _ = cpu_baseline(w, args.cpu_seconds / 2, threads=1)
        line["cpu_baseline_serial"] = {"value": v1, "unit": UNIT, "cores": 1, "kind": "port",
                                       "sample": desc1}
        if "mls" in line:
            line["mls"]["cpu_baseline"] = mls_cpu_baseline(w)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

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

N > 1 (torchrun): every rank runs its own transfer of the same workload
(independent replicas, weak scaling); value = all ranks' targets / max time.

--impl reference times the CPU restatement of the reference algorithm (the
reference itself cannot be built here: it needs Kokkos, KokkosKernels and
ArborX) on all host threads, on a stratified sample of the patch solves.
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
    return ap.parse_args()


def dist_info():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (CPU restatement), bounded sample
# ---------------------------------------------------------------------------

def cpu_baseline(w, seconds_budget: float):
    """Times the CPU restatement on a bounded sample: the full geometry phase,
    then the patch solves of a stratified random sample (by patch size), whose
    time is scaled by the inverse sampling fraction of each stratum, plus one
    partition-of-unity pass.  Returns (pts_per_s, description, threads)."""
    import oracle
    threads = oracle.set_threads(os.cpu_count() or 1)
    t0 = time.perf_counter()
    plan = oracle.build(3, w["src"], w["tgt"], w["nodes_per_cluster"])
    t_geom = time.perf_counter() - t0
    off, _ = plan.src_csr()
    n = np.diff(off)
    K = len(n)
    rng = np.random.default_rng(0)
    edges = [0, 64, 128, 256, 512, 1024, 2048, 1 << 30]
    total = 0.0
    sampled = 0
    budget_each = seconds_budget / (len(edges) - 1)
    vals = w["values"]
    for lo, hi in zip(edges[:-1], edges[1:]):
        ids = np.where((n > lo) & (n <= hi))[0]
        if len(ids) == 0:
            continue
        rng.shuffle(ids)
        # Grow the sample until the stratum's time budget is used.
        take = 1
        spent = 0.0
        done = 0
        while done < len(ids) and spent < budget_each:
            chunk = ids[done:done + take]
            t1 = time.perf_counter()
            plan.solve(w["basis"], vals, patch_list=chunk)
            spent += time.perf_counter() - t1
            done += len(chunk)
            take = min(take * 2, len(ids) - done) if done < len(ids) else take
        total += spent * len(ids) / done
        sampled += done
    # One partition-of-unity pass over all targets (solve of a single patch).
    t1 = time.perf_counter()
    plan.solve(w["basis"], vals, patch_list=np.array([0]))
    t_pu = time.perf_counter() - t1
    est = t_geom + total + t_pu
    m = w["tgt"].shape[0]
    desc = (f"CPU restatement of the reference algorithm (FP64, unpivoted LU), {threads} threads: "
            f"full geometry ({t_geom:.2f}s) + patch solves of a stratified sample of {sampled}/{K} "
            f"patches scaled per size stratum ({total:.1f}s est.) + PU pass ({t_pu:.2f}s); "
            f"estimated {est:.1f}s per transfer")
    return m / est, desc, threads


def run_reference(args):
    rank, world, _ = dist_info()
    if rank != 0:
        return
    args.world = world
    from pacman_b200 import workloads as W
    w = W.make(args.workload, args.scale)
    vals = []
    for _ in range(args.warmup):
        pass  # the oracle has no warm state worth priming beyond the first build
    desc = ""
    threads = 1
    for _ in range(max(args.steps, 1)):
        v, desc, threads = cpu_baseline(w, min(args.cpu_seconds, 30.0))
        vals.append(v)
    value = statistics.median(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": w["tgt"].shape[0] / value * 1e3,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded numpy generators)",
        "config": config_dict(args, w),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": desc},
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


def read_traffic(kernel_key: str):
    """dram bytes per launch of the dominant kernel from the committed ncu
    summary (line 'dram_bytes_per_launch[<key>]: <bytes>'), or None."""
    import glob
    for path in glob.glob(os.path.join(ROOT, "profiles", "*.txt")):
        for line in open(path):
            if line.startswith(f"dram_bytes_per_launch[{kernel_key}]:"):
                try:
                    return float(line.split(":", 1)[1].strip().split()[0])
                except ValueError:
                    return None
    return None


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
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
        for _ in range(args.steps):
            step(args.precision, st)
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
    e2e_times = timed(e2e_step, max(1, min(args.steps, 3)))
    e2e_ms = sum(e2e_times) / len(e2e_times)
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    h2d = (w["src"].nbytes + w["tgt"].nbytes + np.ascontiguousarray(vals_np).nbytes)
    d2h = o_np.nbytes

    # Plain FP64 path and agreement with it.
    extra = {}
    if not args.no_fp64_compare:
        out_mixed = step(args.precision).cpu().numpy()
        f64_stats = {}
        f64_times = timed(lambda: step("fp64", f64_stats), 1)
        out64 = step("fp64").cpu().numpy()
        f64_ms = f64_times[0]
        if world > 1:
            t = torch.tensor([f64_ms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            f64_ms = float(t.item())
        extra["fp64_value"] = m / (f64_ms * 1e-3)
        extra["mixed_over_fp64"] = extra["fp64_value"] and value / extra["fp64_value"]
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

    # Roofline of the dominant kernel, the step kernel of the large-patch
    # Cholesky: one extra transfer after the timed region with CUDA events
    # around each of its launches, on the stream it runs on.
    peak = fp64_gemm_peak(torch, dev)
    kst = {}
    plan = pacman.rbf.Plan(3, S, T, precision=args.precision, **kw)
    plan.execute(w["basis"], V, stats=kst, time_kernels=True)
    plan.close()
    ms_upd = kst.get("ms_update", 0.0)
    achieved = kst.get("update_flops", 0.0) / (ms_upd * 1e-3) / 1e12 if ms_upd else 0.0
    nl = max(1, int(kst.get("update_launches", 0)))
    roofline = {"bound": "fp64", "kernel": "k_col_step / k_col_step_oz (left-looking Cholesky "
                                           "step: column update on the FP64 tensor cores, from "
                                           "step 4 on the int8 tensor cores; trsm; next diagonal)",
                "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak if peak else None,
                "peak_source": "measured live: cuBLAS DGEMM 8192^3 on this GPU (FP64 has no "
                               "faster path on B200; MEASURED_PEAKS.json holds no FP64 figure)",
                "traffic": read_traffic(args.workload),
                "flops_per_launch": kst.get("update_flops", 0.0) / nl,
                "ms_per_launch": ms_upd / nl,
                "launches_per_step": nl,
                "ms_update_per_step": ms_upd,
                "share_of_step": ms_upd / ms_per_step if ms_per_step else None}

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
        "clocks": clk.summary(),
        "roofline": roofline,
        "stats": {k: stats.get(k) for k in ("radius", "num_patches", "sum_n", "sum_m", "max_n",
                                            "patches_fp32", "patches_fp64", "patches_fallback",
                                            "ms_geometry", "ms_solve", "ms_factor")},
        **extra,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, desc, threads = cpu_baseline(w, args.cpu_seconds)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": desc}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

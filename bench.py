"""Benchmark: seconds to embed a 1,000,000 x 128 mixture with PaCMAP on B200 (one JSON line).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n ROWS] [--d COLS]

One step = one full fit_transform (preprocess -> exact kNN -> reselection -> MN/FP sampling -> CSR ->
450 fused gradient+Adam iterations in one CUDA graph) of the whole synthetic dataset:
  * value: inputs resident in HBM, C ABI `pacmap_fit_transform_device`, CUDA events around each step;
  * e2e:   the same through `pacmap_fit_transform` with pinned host input and host output (the host
           copies are inside the timed region).
With N GPUs (torchrun) every rank embeds its own dataset (replicas only: the path does not shard);
timing is the max over ranks and value is seconds per embedding for the whole job.
`--impl reference` times the CPU restatement of the reference (the reference's Rust crate cannot be
built here) on a bounded sample on rank 0 and projects it to the full size.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "pacmap-rs_b200"))

METRIC = "s to embed 1M×128 at matched 10-NN preservation, learned-init vs plain GPU"
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")


def _peaks():
    try:
        with open(MEASURED_PEAKS) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), float(p["bf16_tflops"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.rows = []
        self._stop = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.QUERY}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                for line in out.stdout.strip().splitlines():
                    self.rows.append([v.strip() for v in line.split(",")])
            except (OSError, subprocess.SubprocessError):
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def make_data(n, d, seed):
    from pacmap_b200 import datasets

    if d == 128:
        x, _ = datasets.anisotropic_mixture(n=n, d=d, k=50, seed=seed)
    else:
        x, _ = datasets.isotropic_mixture(n=n, d=d, k=50, seed=seed)
    return x


def config_for(pm, seed):
    return pm.Configuration(initialization=pm.Initialization.Random(7 + seed), seed=7 + seed)


def cpu_baseline(n_full, d, sample_n=12000, threads=None):
    """Time the oracle (C++/OpenMP restatement of the reference) on a sample and project to n_full.

    The exact kNN is O(n^2 d) and is scaled by (n_full / sample_n)^2; pair sampling, the CSR-free
    gradient and Adam are O(n) and scaled by n_full / sample_n.
    """
    import oracle

    cores = oracle.set_threads(threads or os.cpu_count() or 1)
    x = make_data(sample_n, d, seed=99)
    t0 = time.perf_counter()
    xp, *_ = oracle.preprocess(x)
    t1 = time.perf_counter()
    rc, (k, n_mn, n_fp) = oracle.decide_num_pairs(n_full)
    kp = min(k + 50, sample_n - 1)
    ki, kd = oracle.knn_exact(xp, kp)
    t2 = time.perf_counter()
    pnn = oracle.sample_neighbors_pair(oracle.scale_dist(kd, oracle.sigma(kd), ki), ki, k)
    pmn = oracle.sample_mn_pairs(xp, n_mn, 7)
    pfp = oracle.sample_fp_pairs(pnn, sample_n, k, n_fp, 7)
    y0 = oracle.init_random(sample_n, 2, 7)
    t3 = time.perf_counter()
    oracle.optimize(y0, pnn, pmn, pfp)
    t4 = time.perf_counter()
    lin = (t1 - t0) + (t3 - t2) + (t4 - t3)
    quad = t2 - t1
    s = n_full / sample_n
    projected = lin * s + quad * s * s
    return {"value": round(projected, 3), "unit": "s", "cores": cores, "kind": "port",
            "sample": (f"oracle fit_transform on {sample_n}x{d} of the same generator (k={k}, n_mn={n_mn}, "
                       f"n_fp={n_fp}, 450 iters): kNN {quad:.2f}s scaled x{s * s:.0f}, rest {lin:.2f}s scaled "
                       f"x{s:.0f}; reference Rust crate unavailable (no cargo in the image)"),
            "measured_s": round(t4 - t0, 3)}


def run_reference(args, rank, world):
    if rank != 0:
        return
    base = cpu_baseline(args.n, args.d)
    steps = []
    for _ in range(args.steps):
        steps.append(base["value"])
    v = float(np.mean(steps))
    line = {"metric": METRIC, "value": v, "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": v * 1000, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": f"plain PaCMAP {args.n}x{args.d} -> 2-D, 450 iterations, exact kNN", "n": args.n,
                       "d": args.d},
            "cpu_baseline": base, "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local_rank):
    import torch

    import pacmap_b200 as pm

    torch.cuda.set_device(local_rank)
    dist = world > 1
    if dist:
        import datetime

        import torch.distributed as tdist

        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    n, d = args.n, args.d
    x = make_data(n, d, seed=rank)
    cfg = config_for(pm, 0)
    cfg.device = local_rank
    dx = torch.from_numpy(x).to(f"cuda:{local_rank}")
    dy = torch.empty((n, 2), dtype=torch.float32, device=f"cuda:{local_rank}")
    hx = torch.from_numpy(x).pin_memory()
    hy = torch.empty((n, 2), dtype=torch.float32).pin_memory()

    def step_device():
        pm.fit_transform_device(dx.data_ptr(), n, d, dy.data_ptr(), cfg)

    def step_e2e():
        import ctypes as C

        from pacmap_b200 import _abi

        cc = pm._CConfig(cfg, n)
        rc = _abi.lib().pacmap_fit_transform(C.c_void_p(hx.data_ptr()), n, d, C.byref(cc.c),
                                             C.c_void_p(hy.data_ptr()), None)
        pm._check(rc)

    def barrier():
        if dist:
            tdist.barrier()
        torch.cuda.synchronize()

    def timed(fn, k):
        barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        for _ in range(k):
            fn()
        ev1.record()
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        barrier()
        if dist:
            t = torch.tensor([ms], device=f"cuda:{local_rank}")
            tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    for _ in range(args.warmup):
        step_device()
    stages = {}
    if not args.minimal:
        # stage breakdown of one untimed step (CUDA events inside the library, on its stream)
        pm.set_stage_timing(True)
        step_device()
        stages = pm.stage_times()
        pm.set_stage_timing(False)
    pm.last_launch_count()
    with ClockSampler(local_rank) as clk:
        ms = timed(step_device, args.steps)
    launches = pm.last_launch_count()
    if args.minimal:
        if rank == 0:
            print(json.dumps({"minimal": True, "ms_per_step": ms / args.steps, "gpu_launches": launches}), flush=True)
        if dist:
            tdist.destroy_process_group()
        return
    e2e_steps = max(1, args.steps // 2)
    ms_e2e = timed(step_e2e, e2e_steps)

    # quality of the embedding (outside the timed region)
    from pacmap_b200 import datasets

    sample, trip = datasets.quality_sample(n, 10000, 5)
    pres, tacc = pm.quality(x, dy.cpu().numpy(), sample, trip, 10, local_rank)

    if rank != 0:
        if dist:
            tdist.destroy_process_group()
        return
    hbm, bf16, src = _peaks()
    per_step = ms / args.steps
    knn_ms = stages.get("knn_filter") or stages.get("knn", 0.0)
    flops = 2.0 * n * n * d
    achieved_tf = flops / (knn_ms * 1e-3) / 1e12 if knn_ms > 0 else None
    line = {
        "metric": METRIC, "value": round(per_step / 1000.0 / world, 4), "unit": "s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(per_step, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"plain PaCMAP {n}x{d} -> 2-D, Random init, 450 iterations, exact kNN (k'={min(40 + 50, n - 1)})",
                   "n": n, "d": d, "generator": "anisotropic 50-Gaussian mixture" if d == 128 else "isotropic mixture",
                   "l2": "inputs larger than L2 (x = %.0f MB)" % (n * d * 4 / 1e6), "parallelism": f"replicas{world}",
                   "init": "Random(7)", "knn_mode": "auto"},
        "e2e": {"value": round(ms_e2e / e2e_steps / 1000.0 / world, 4), "unit": "s",
                "h2d_bytes_per_step": int(n * d * 4), "d2h_bytes_per_step": int(n * 2 * 4)},
        "gpu_launches": int(launches),
        "stages_ms": {k: round(v, 3) for k, v in stages.items()},
        "quality": {"knn10_preservation": round(pres, 4), "triplet_accuracy": round(tacc, 4)},
        "roofline": {"kernel": "knn_filter_kernel (tcgen05 distance GEMM + fused candidate filter)" if stages.get("knn_filter") else "knn_simt_kernel", "bound": "tensor",
                     "achieved": round(achieved_tf, 2) if achieved_tf else None, "peak": bf16, "unit": "TFLOP/s",
                     "frac": round(achieved_tf / bf16, 4) if achieved_tf else None, "traffic": None,
                     "peak_source": f"{src} bf16 dense", "algorithmic": "2*n^2*d flops per launch"},
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(n, d)
    print(json.dumps(line), flush=True)
    if dist:
        tdist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--d", type=int, default=128)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--minimal", action="store_true",
                    help="profiling runs: only warm-up + timed steps (no stage timing, e2e or quality passes)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus if args.gpus else 1)))
    if "RANK" not in os.environ:
        world = 1
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()

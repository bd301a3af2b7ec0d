"""Benchmark: seconds to embed a 1,000,000 x 128 mixture with PaCMAP on B200 (one JSON line).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload 1m-128|4m-256]
                    [--n ROWS] [--d COLS]

A learned initialiser (MLP 128-512-512-2) is first trained, outside the timed region, on the plain GPU
embedding of 200,000 draws of the generator. One step = one full learned-init fit_transform of a fresh
draw (preprocess -> exact kNN -> reselection -> MN/FP sampling -> MLP prediction as Value init -> CSR ->
the shortened schedule (0, 50, 150) of fused gradient+Adam iterations in one CUDA graph):
  * value: inputs resident in HBM, C ABI `pacmap_fit_transform_learned_device`, CUDA events around
           each step; the plain schedule (Random init, (100, 100, 250)) on the same draw is timed the
           same way (`plain_gpu_s`), and both embeddings are judged by 10-NN preservation and triplet
           accuracy; a learned run more than 0.005 below the plain preservation continues on the plain
           schedule, inside the timed step;
  * e2e:   the learned step through `pacmap_fit_transform_learned` with pinned host input and host
           output (the host copies are inside the timed region).
With N GPUs (torchrun) every rank embeds its own dataset (replicas only: the path does not shard);
timing is the max over ranks and value is seconds per embedding for the whole job.
`--impl reference` times the CPU restatement of the reference (the reference's Rust crate cannot be
built here) on a bounded sample on rank 0 and projects it to the full size.
`--workload 4m-256` runs the large configuration instead: 4,000,000 x 256 draws of a 200-Gaussian
mixture on a 32-dim subspace (noise 0.05 elsewhere) -> 3-D, MLP 256-512-512-3 trained on 300,000 draws.
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
WORKLOADS = {
    "1m-128": {"n": 1_000_000, "d": 128, "dim": 2, "n_train": 200_000, "generator": "anisotropic",
               "metric": METRIC,
               "generator_desc": "anisotropic 50-Gaussian mixture (seed 0; draw seed 1000+rank)"},
    "4m-256": {"n": 4_000_000, "d": 256, "dim": 3, "n_train": 300_000, "generator": "subspace",
               "metric": "s to embed 4M×256 -> 3-D at matched 10-NN preservation, learned-init vs plain GPU",
               "generator_desc": ("200 Gaussians on a random 32-dim subspace + N(0, 0.05^2) in the other dims "
                                  "(seed 0; draw seed 1000+rank)")},
}
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


def make_data(n, d, seed, draw_seed=None, generator="anisotropic"):
    """n draws of the workload's mixture fixed by `seed` (fresh points per `draw_seed`)."""
    from pacmap_b200 import datasets

    if generator == "subspace":
        x, _ = datasets.subspace_mixture(n=n, d=d, k=200, seed=seed, draw_seed=draw_seed)
    else:
        x, _ = datasets.anisotropic_mixture(n=n, d=d, k=50, seed=seed, draw_seed=draw_seed)
    return x


def config_for(pm, seed):
    return pm.Configuration(initialization=pm.Initialization.Random(7 + seed), seed=7 + seed)


def cpu_baseline(n_full, d, sample_n=12000, threads=None, dim=2, generator="anisotropic"):
    """Time the oracle (C++/OpenMP restatement of the reference) on a sample and project to n_full.

    The exact kNN is O(n^2 d) and is scaled by (n_full / sample_n)^2; pair sampling, the CSR-free
    gradient and Adam are O(n) and scaled by n_full / sample_n.
    """
    import oracle

    cores = oracle.set_threads(threads or os.cpu_count() or 1)
    x = make_data(sample_n, d, seed=99, generator=generator)
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
    y0 = oracle.init_random(sample_n, dim, 7)
    t3 = time.perf_counter()
    oracle.optimize(y0, pnn, pmn, pfp)
    t4 = time.perf_counter()
    lin = (t1 - t0) + (t3 - t2) + (t4 - t3)
    quad = t2 - t1
    s = n_full / sample_n
    projected = lin * s + quad * s * s
    return {"value": round(projected, 3), "unit": "s", "cores": cores, "kind": "port",
            "sample": (f"oracle fit_transform on {sample_n}x{d} -> {dim}-D of the same generator (k={k}, n_mn={n_mn}, "
                       f"n_fp={n_fp}, 450 iters): kNN {quad:.2f}s scaled x{s * s:.0f}, rest {lin:.2f}s scaled "
                       f"x{s:.0f}; reference Rust crate unavailable (no cargo in the image)"),
            "measured_s": round(t4 - t0, 3)}


def run_reference(args, rank, world):
    if rank != 0:
        return
    w = WORKLOADS[args.workload]
    base = cpu_baseline(args.n, args.d, dim=w["dim"], generator=w["generator"])
    steps = []
    for _ in range(args.steps):
        steps.append(base["value"])
    v = float(np.mean(steps))
    line = {"metric": w["metric"], "value": v, "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": v * 1000, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": f"plain PaCMAP {args.n}x{args.d} -> {w['dim']}-D, 450 iterations, exact kNN", "n": args.n,
                       "d": args.d},
            "cpu_baseline": base, "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _pair_counts(n, mid_near_ratio=0.5, far_pair_ratio=2.0):
    """decide_num_pairs (lib.rs:565-597) in f32: (k, n_mn, n_fp)."""
    rnd = lambda v: int(np.floor(np.float32(v) + np.float32(0.5)))  # noqa: E731  (f32::round: half away from 0)
    k = 10 if n <= 10000 else rnd(np.float32(10.0) + np.float32(15.0) * (np.log10(np.float32(n)) - np.float32(4.0)))
    return k, rnd(np.float32(k) * np.float32(mid_near_ratio)), rnd(np.float32(k) * np.float32(far_pair_ratio))


def _optimize_bytes(n, dim, iters):
    """Algorithmic HBM bytes of the gradient + Adam iterations: 8 B per active pair (its two u32
    endpoints, read once), 4*n*dim for y read by the gradient, 24*n*dim for Adam (y, m, v read+write);
    mid-near pairs are inactive in phase 3 (w_mn = 0)."""
    k, n_mn, n_fp = _pair_counts(n)
    p12 = n * (k + n_mn + n_fp)
    p3 = n * (k + n_fp)
    per = lambda pairs: 8 * pairs + 28 * n * dim  # noqa: E731
    return (iters[0] + iters[1]) * per(p12) + iters[2] * per(p3)


def run_ours(args, rank, world, local_rank):
    import ctypes as C

    import torch

    import pacmap_b200 as pm
    from pacmap_b200 import _abi, datasets, learned

    torch.cuda.set_device(local_rank)
    dist = world > 1
    if dist:
        import datetime

        import torch.distributed as tdist

        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    w = WORKLOADS[args.workload]
    n, d, dim, gen = args.n, args.d, w["dim"], w["generator"]
    n_train = min(w["n_train"], max(n // 5, 4096))
    # the learned initialiser is trained once per generator (outside the timed region): plain GPU PaCMAP
    # of n_train draws, then AdamW on (x', embedding)
    train_s, train_losses = None, None
    if args.minimal:
        params = learned.init_params(d, dim, seed=0)
    else:
        x_train = make_data(n_train, d, seed=0, draw_seed=10_000 + rank, generator=gen)
        y_train, _ = pm.fit_transform(x_train, pm.Configuration(initialization=pm.Initialization.Random(7), seed=7,
                                                                embedding_dimensions=dim, device=local_rank))
        xp_train, *_ = pm.stages.preprocess(x_train, local_rank)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        params, train_losses = learned.train(learned.init_params(d, dim, seed=0), xp_train, y_train, epochs=20,
                                             batch=4096, lr=1e-3, weight_decay=1e-4, seed=0, device=local_rank)
        train_s = time.perf_counter() - t0
        del x_train, y_train, xp_train
    # a fresh draw of the same generator
    x = make_data(n, d, seed=0, draw_seed=1000 + rank, generator=gen)
    cfg_plain = pm.Configuration(initialization=pm.Initialization.Random(7), seed=7, embedding_dimensions=dim,
                                 device=local_rank)
    cfg_short = pm.Configuration(seed=7, num_iters=learned.SHORT_SCHEDULE, embedding_dimensions=dim,
                                 device=local_rank)
    dev = f"cuda:{local_rank}"
    dx = torch.from_numpy(x).to(dev)
    dy_l = torch.empty((n, dim), dtype=torch.float32, device=dev)
    dy_p = torch.empty((n, dim), dtype=torch.float32, device=dev)
    dy_c = torch.empty((n, dim), dtype=torch.float32, device=dev)
    hx = torch.from_numpy(x).pin_memory()
    hy = torch.empty((n, dim), dtype=torch.float32).pin_memory()
    gate = {"continued": False}

    def step_learned():
        learned.fit_transform_learned_device(dx.data_ptr(), n, d, dy_l.data_ptr(), params, cfg_short)
        if gate["continued"]:
            # the run missed the plain run's 10-NN preservation by more than 0.005: continue it on the
            # plain schedule from where it stopped
            cont = pm.Configuration(initialization=pm.Initialization.Value(dy_l.cpu().numpy()), seed=7,
                                    embedding_dimensions=dim, device=local_rank)
            pm.fit_transform_device(dx.data_ptr(), n, d, dy_c.data_ptr(), cont)

    def step_plain():
        pm.fit_transform_device(dx.data_ptr(), n, d, dy_p.data_ptr(), cfg_plain)

    def step_e2e():
        cc = pm._CConfig(cfg_short, n)
        p = np.ascontiguousarray(params, dtype=np.float32)
        pm._check(_abi.lib().pacmap_fit_transform_learned(C.c_void_p(hx.data_ptr()), n, d, C.byref(cc.c),
                                                          C.c_void_p(p.ctypes.data), C.c_void_p(hy.data_ptr()),
                                                          None))

    def barrier():
        if dist:
            tdist.barrier()
        torch.cuda.synchronize()

    # every library call enqueues its kernels on the library's own stream: time on that stream
    lib_stream = torch.cuda.ExternalStream(_abi.lib().pacmap_device_stream(local_rank), device=dev)

    def timed(fn, k):
        barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(lib_stream)
        for _ in range(k):
            fn()
        ev1.record(lib_stream)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        barrier()
        if dist:
            t = torch.tensor([ms], device=dev)
            tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    for _ in range(args.warmup):
        step_learned()
    if args.minimal:
        pm.last_launch_count()
        ms = timed(step_learned, args.steps)
        launches = pm.last_launch_count()
        if rank == 0:
            print(json.dumps({"minimal": True, "ms_per_step": ms / args.steps, "gpu_launches": launches}), flush=True)
        if dist:
            tdist.destroy_process_group()
        return
    for _ in range(args.warmup):
        step_plain()
    # quality gate: learned (short schedule) against the plain schedule on the same draw
    sample, trip = datasets.quality_sample(n, 10000, 5)
    q_plain = pm.quality(x, dy_p.cpu().numpy(), sample, trip, 10, local_rank)
    q_learned = pm.quality(x, dy_l.cpu().numpy(), sample, trip, 10, local_rank)
    gate["continued"] = q_learned[0] < q_plain[0] - 0.005
    q_final = q_learned
    if gate["continued"]:
        step_learned()
        q_final = pm.quality(x, dy_c.cpu().numpy(), sample, trip, 10, local_rank)
    # stage breakdown of one untimed step of each (CUDA events inside the library, on its stream)
    pm.set_stage_timing(True)
    step_plain()
    stages_plain = pm.stage_times()
    learned.fit_transform_learned_device(dx.data_ptr(), n, d, dy_l.data_ptr(), params, cfg_short)
    stages_learned = pm.stage_times()
    pm.set_stage_timing(False)

    pm.last_launch_count()
    with ClockSampler(local_rank) as clk:
        ms = timed(step_learned, args.steps)
    launches = pm.last_launch_count()
    ms_plain = timed(step_plain, args.steps)
    e2e_steps = max(1, args.steps // 2)
    ms_e2e = timed(step_e2e, e2e_steps)

    if rank != 0:
        if dist:
            tdist.destroy_process_group()
        return
    hbm, bf16, src = _peaks()
    per_step = ms / args.steps
    per_plain = ms_plain / args.steps
    knn_ms = stages_learned.get("knn_filter") or stages_learned.get("knn", 0.0)
    flops = 2.0 * n * n * d
    achieved_tf = flops / (knn_ms * 1e-3) / 1e12 if knn_ms > 0 else None
    opt_ms = stages_learned.get("optimize", 0.0)
    opt_bytes = _optimize_bytes(n, dim, learned.SHORT_SCHEDULE)
    opt_gbs = opt_bytes / (opt_ms * 1e-3) / 1e9 if opt_ms > 0 else None
    rnd = lambda q: {"knn10_preservation": round(q[0], 5), "triplet_accuracy": round(q[1], 4)}  # noqa: E731
    line = {
        "metric": w["metric"], "value": round(per_step / 1000.0 / world, 4), "unit": "s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(per_step, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": (f"learned-init PaCMAP of a fresh {n}x{d} draw -> {dim}-D: MLP {d}-512-512-{dim} "
                                f"prediction as Value init + schedule {learned.SHORT_SCHEDULE}; vs plain Random(7) "
                                f"with {learned.PLAIN_SCHEDULE}; exact kNN (k'={min(_pair_counts(n)[0] + 50, n - 1)})"),
                   "n": n, "d": d, "dim": dim, "generator": w["generator_desc"],
                   "mlp_training": f"{n_train} draws (draw seed 10000+rank), plain GPU embedding, 20 epochs, batch "
                                   "4096, AdamW lr 1e-3 wd 1e-4 (outside the timed region)",
                   "l2": "inputs larger than L2 (x = %.0f MB)" % (n * d * 4 / 1e6), "parallelism": f"replicas{world}",
                   "knn_mode": "auto"},
        "plain_gpu_s": round(per_plain / 1000.0 / world, 4),
        "learned_over_plain": round(per_step / per_plain, 4),
        "gate": {"rule": "continue on the plain schedule if 10-NN preservation < plain - 0.005",
                 "continued": gate["continued"], "plain": rnd(q_plain), "learned_short": rnd(q_learned),
                 "final": rnd(q_final)},
        "mlp_train_s": round(train_s, 3) if train_s else None,
        "mlp_train_loss": [round(float(v), 4) for v in (train_losses[0], train_losses[-1])] if train_losses is not None else None,
        "e2e": {"value": round(ms_e2e / e2e_steps / 1000.0 / world, 4), "unit": "s",
                "h2d_bytes_per_step": int(n * d * 4 + np.asarray(params).nbytes), "d2h_bytes_per_step": int(n * dim * 4)},
        "gpu_launches": int(launches),
        "stages_ms": {"learned": {k: round(v, 3) for k, v in stages_learned.items()},
                      "plain": {k: round(v, 3) for k, v in stages_plain.items()}},
        "roofline": {"kernel": "knn_filter_kernel (tcgen05 distance GEMM + fused candidate filter)" if stages_learned.get("knn_filter") else "knn_simt_kernel", "bound": "tensor",
                     "achieved": round(achieved_tf, 2) if achieved_tf else None, "peak": bf16, "unit": "TFLOP/s",
                     "frac": round(achieved_tf / bf16, 4) if achieved_tf else None, "traffic": None,
                     "peak_source": f"{src} bf16 dense", "algorithmic": "2*n^2*d flops per launch",
                     "filter_rate_scores_per_s": round(n * n / (knn_ms * 1e-3), 1) if knn_ms > 0 else None},
        "roofline_optimizer": {"kernel": "grad_adam_kernel (CSR gradient + Adam, CUDA graph)", "bound": "hbm",
                               "achieved": round(opt_gbs, 1) if opt_gbs else None, "peak": hbm, "unit": "GB/s",
                               "frac": round(opt_gbs / hbm, 4) if opt_gbs else None,
                               "algorithmic": "8 B per active pair + 28*n*dim B per iteration (k, n_mn, n_fp = %d, %d, %d)" % _pair_counts(n),
                               "peak_source": f"{src} HBM copy"},
        "clocks": clk.summary(),
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(n, d, dim=dim, generator=gen)
    print(json.dumps(line), flush=True)
    if dist:
        tdist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="1m-128", choices=sorted(WORKLOADS))
    ap.add_argument("--n", type=int, default=None, help="rows (default: the workload's)")
    ap.add_argument("--d", type=int, default=None, help="columns (default: the workload's)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--minimal", action="store_true",
                    help="profiling runs: only warm-up + timed steps (no stage timing, e2e or quality passes)")
    args = ap.parse_args()
    if args.n is None:
        args.n = WORKLOADS[args.workload]["n"]
    if args.d is None:
        args.d = WORKLOADS[args.workload]["d"]
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

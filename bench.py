#!/usr/bin/env python
"""Benchmark of the variational fisheye stereo solve on B200.

One *step* is one solve of every pair in the rank's batch of seeded synthetic 848x800
fisheye pairs (5 pyramid levels x 3 warps x 50 primal-dual iterations, masked solve, the
reference's solver settings).  ``value`` is whole-job frames/s with inputs resident in HBM;
``e2e`` is the same metric through the public API with pinned host buffers (H2D of both
images and D2H of the disparity inside the timed region).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--path fused|plain] [--batch B]
    python bench.py --impl reference ...   # the CPU restatement of the reference on host cores

Under torchrun every rank runs its own replica (the solve has no cross-GPU exchange); the
job value is all frames over the slowest rank's time.
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

METRIC = "848×800 stereo frames/s + p99 latency, fused vs plain, at ≤0.05px mean err"
W0, H0 = 848, 800
B_ALG_FP32 = 116.0  # algorithmic bytes per pixel-iteration of the inner loop, FP32 storage
B_ALG_FP16 = 84.0   # with p, q, v in FP16


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--path", default="fused", choices=["fused", "plain"])
    ap.add_argument("--batch", type=int, default=0, help="pairs per rank (default: 8 fused, 1 plain)")
    ap.add_argument("--storage", default="fp16", choices=["fp16", "fp32"], help="fused path: p, q, v-bar and warped-image storage")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain drop-in comparison run")
    ap.add_argument("--seed", type=int, default=20260)
    ap.add_argument("--mode", default="frames", choices=["frames", "mixed", "serving"],
                    help="frames: 848x800 batch (headline); mixed: 8x848x800 + 4x640x480 + 4x424x400 in one "
                         "batch; serving: 6 camera streams with Poisson arrivals")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the mixed-size batch and serving runs that the default line carries")
    ap.add_argument("--fine", type=int, default=-1,
                    help="fused batches: pairs at full resolution at a time (-1 auto, 0 no limit)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def pair_cache(w, h, seed):
    """Synthetic pair (rendered on the GPU when there is one), cached under /tmp so repeated
    runs on one machine skip rendering."""
    from vfs_b200 import synth
    path = f"/tmp/vfs_b200_pair_{w}x{h}_{seed}.npz"
    if os.path.exists(path):
        try:
            d = np.load(path)
            return dict(i0=d["i0"], i1=d["i1"], mask=d["mask"], tv=d["tv"], cv=d["cv"])
        except Exception:
            pass
    try:
        import torch
        gpu = torch.cuda.is_available()
    except Exception:
        gpu = False
    p = synth.make_pair_gpu(w, h, seed) if gpu else synth.make_pair(w, h, seed)
    d = dict(i0=p.i0, i1=p.i1, mask=p.mask, tv=p.tv, cv=p.cv)
    try:
        np.savez(path, **d)
    except OSError:
        pass
    return d


class ClockSampler:
    """nvidia-smi clock / throttle samples while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.lines = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    for p in (os.path.join(ROOT, "MEASURED_PEAKS.json"),):
        try:
            d = json.load(open(p))
            return float(d["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def ncu_traffic(kernel_key):
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    try:
        d = json.load(open(p))
        return d.get(kernel_key)
    except Exception:
        return None


def union_ms(iv):
    """Total length of the union of [start, end] intervals."""
    iv = iv[np.argsort(iv[:, 0])]
    tot, cs, ce = 0.0, iv[0, 0], iv[0, 1]
    for a, b in iv[1:]:
        if a > ce:
            tot += ce - cs
            cs, ce = a, b
        else:
            ce = max(ce, b)
    return float(tot + ce - cs)


def make_solver(pair, path, stream, half=False):
    from vfs_b200 import synth
    from vfs_b200.stereotgv import StereoTgv
    sp = synth.SOLVER_PARAMS
    s = StereoTgv()
    s.set_solve_path(path == "fused", half)
    s.limitRange = synth.LIMIT_RANGE
    s.initialize(W0, H0, sp["beta"], sp["gamma"], sp["alpha0"], sp["alpha1"], sp["timestep_lambda"], sp["lambda_"],
                 synth.n_levels_for(W0), sp["fScale"], sp["nWarpIters"], sp["nSolverIters"])
    s.copyMaskToDevice(pair["mask"])
    s.loadVectorFields(pair["tv"], pair["cv"])
    s.set_stream(stream)
    return s


def cpu_baseline(pair, budget_s=12.0, precision=64):
    """Time the CPU oracle (all host threads) on the workload; returns (frames/s, threads, u of the last frame)."""
    from oracle.oracle import OracleStereoTgv
    from vfs_b200 import synth
    sp = synth.SOLVER_PARAMS
    o = OracleStereoTgv(precision)
    o.set_limit_range(synth.LIMIT_RANGE)
    o.initialize(W0, H0, sp["beta"], sp["gamma"], sp["alpha0"], sp["alpha1"], sp["timestep_lambda"], sp["lambda_"],
                 synth.n_levels_for(W0), sp["fScale"], sp["nWarpIters"], sp["nSolverIters"])
    o.copy_mask_to_device(pair["mask"])
    o.load_vector_fields(pair["tv"], pair["cv"])
    n, t0 = 0, time.perf_counter()
    while True:
        o.copy_images_to_device(pair["i0"], pair["i1"])
        o.solve_stereo_forward_masked()
        n += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    dt = time.perf_counter() - t0
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return n / dt, threads, o.get("u"), n, dt


def cpu_single_thread_s(pair, precision=64):
    """Seconds for one 848x800 frame of the CPU oracle on one host thread (the same solve as
    cpu_baseline, OpenMP limited to one thread, then restored)."""
    from oracle.oracle import OracleStereoTgv, set_threads
    from vfs_b200 import synth
    sp = synth.SOLVER_PARAMS
    o = OracleStereoTgv(precision)
    o.set_limit_range(synth.LIMIT_RANGE)
    o.initialize(W0, H0, sp["beta"], sp["gamma"], sp["alpha0"], sp["alpha1"], sp["timestep_lambda"], sp["lambda_"],
                 synth.n_levels_for(W0), sp["fScale"], sp["nWarpIters"], sp["nSolverIters"])
    o.copy_mask_to_device(pair["mask"])
    o.load_vector_fields(pair["tv"], pair["cv"])
    o.copy_images_to_device(pair["i0"], pair["i1"])
    prev = set_threads(1)
    try:
        t0 = time.perf_counter()
        o.solve_stereo_forward_masked()
        return time.perf_counter() - t0
    finally:
        set_threads(prev)


def run_reference(args, rank, world):
    """--impl reference: the reference's solver restated on the host cores, all host threads.
    The reference has no CPU path of its own; its CUDA sources, built here as a test oracle
    (oracle/_ref), run on the GPU and are compared with this library in the tests."""
    if rank != 0:
        return
    pair = pair_cache(W0, H0, args.seed)
    from oracle.oracle import OracleStereoTgv, build as build_oracle
    from vfs_b200 import synth
    build_oracle()
    sp = synth.SOLVER_PARAMS
    o = OracleStereoTgv(32)
    o.set_limit_range(synth.LIMIT_RANGE)
    o.initialize(W0, H0, sp["beta"], sp["gamma"], sp["alpha0"], sp["alpha1"], sp["timestep_lambda"], sp["lambda_"],
                 synth.n_levels_for(W0), sp["fScale"], sp["nWarpIters"], sp["nSolverIters"])
    o.copy_mask_to_device(pair["mask"])
    o.load_vector_fields(pair["tv"], pair["cv"])

    def step():
        o.copy_images_to_device(pair["i0"], pair["i1"])
        o.solve_stereo_forward_masked()

    t0 = time.perf_counter()
    step()
    t_frame = time.perf_counter() - t0
    budget = 150.0
    warm = max(0, min(args.warmup - 1, int(budget * 0.2 / max(t_frame, 1e-3))))
    steps = max(1, min(args.steps, int(budget * 0.8 / max(t_frame, 1e-3))))
    for _ in range(warm):
        step()
    times = []
    for _ in range(steps):
        t = time.perf_counter()
        step()
        times.append(time.perf_counter() - t)
    tot = sum(times)
    fps = steps / tot
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    line = {
        "impl": "reference", "metric": METRIC, "value": fps, "unit": "frames/s", "n_gpus": world, "steps": steps,
        "warmup": warm + 1, "ms_per_step": 1000 * tot / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "848x800 fisheye stereo pair, masked TGV-L1 solve, 5 levels x 3 warps x 50 iterations",
                   "batch": 1, "seed": args.seed},
        "latency_ms": {"p50": 1000 * float(np.percentile(times, 50)), "p99": 1000 * float(np.percentile(times, 99))},
        "cpu_baseline": {"value": fps, "unit": "frames/s", "cores": threads, "kind": "port",
                         "sample": f"{steps} full 848x800 frames, float32 restatement of the reference solver, "
                                   f"OpenMP over rows"},
        "e2e": {"value": fps, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def fp64_u(pair, w=W0, h=H0):
    """One float64 oracle solve of a w x h pair (all host threads)."""
    from oracle.oracle import OracleStereoTgv
    from vfs_b200 import synth
    sp = synth.SOLVER_PARAMS
    o = OracleStereoTgv(64)
    o.set_limit_range(synth.LIMIT_RANGE)
    o.initialize(w, h, sp["beta"], sp["gamma"], sp["alpha0"], sp["alpha1"], sp["timestep_lambda"], sp["lambda_"],
                 synth.n_levels_for(w), sp["fScale"], sp["nWarpIters"], sp["nSolverIters"])
    o.copy_mask_to_device(pair["mask"])
    o.load_vector_fields(pair["tv"], pair["cv"])
    o.copy_images_to_device(pair["i0"], pair["i1"])
    o.solve_stereo_forward_masked()
    return o.get("u")


def error_stats(us, refs, masks):
    """Disparity error of the solves `us` against float64 oracle solves `refs`, inside the masks."""
    d = np.concatenate([np.abs(np.asarray(u, np.float64) - r)[m > 0] for u, r, m in zip(us, refs, masks)])
    return {"mean_abs_px": float(d.mean()), "max_abs_px": float(d.max()), "bad_1px_rate": float((d > 1.0).mean()),
            "frames": len(us)}


def accuracy_report(pairs, u_timed, u64_first, half, dev):
    """Disparity error against the float64 oracle over every pair of the batch, inside the
    masks, for the timed form and the other two forms on the same inputs: the fused solve with
    the other storage, and the plain drop-in path (one kernel per reference kernel)."""
    import torch
    from vfs_b200.stereotgv import StereoBatch
    st = torch.cuda.Stream(device=dev)
    other = StereoBatch(half_storage=not half, stream=st)
    solvers = [make_solver(p, "fused", st, not half) for p in pairs]
    for s in solvers:
        other.add(s)
    u_other = other.solve_host([(p["i0"], p["i1"]) for p in pairs])
    u_plain = []
    for p in pairs:
        s = make_solver(p, "plain", st)
        s.copyImagesToDevice(p["i0"], p["i1"])
        s.solveStereoForwardMasked()
        u_plain.append(s.copy1DDisparityToHost())
    torch.cuda.synchronize()
    u64 = [u64_first] + [fp64_u(p) for p in pairs[1:]]

    def stats(us):
        d = np.concatenate([np.abs(np.asarray(u, np.float64) - r)[p["mask"] > 0] for u, r, p in zip(us, u64, pairs)])
        per_pair_max = [float(np.abs(np.asarray(u, np.float64) - r)[p["mask"] > 0].max())
                        for u, r, p in zip(us, u64, pairs)]
        return {"mean_abs_px": float(d.mean()), "max_abs_px": float(d.max()), "bad_1px_rate": float((d > 1.0).mean()),
                "max_abs_px_per_pair": per_pair_max}

    forms = {("fused_fp16" if half else "fused_fp32"): stats(u_timed),
             ("fused_fp32" if half else "fused_fp16"): stats(u_other),
             "plain_fp32": stats(u_plain)}
    fp32_key = "fused_fp32"
    fused32 = u_other if half else u_timed
    forms["fused_fp32_vs_plain_max_abs_px"] = float(max(np.abs(a - b).max() for a, b in zip(fused32, u_plain)))
    forms["pairs"] = len(pairs)
    forms["region"] = "pixels inside each pair's fisheye mask"
    return forms


def plain_reference_run(pair, dev, flush, steps=6):
    """The drop-in path (one kernel per reference kernel, FP32, one pair at a time) on the
    same GPU and inputs: frames/s with device-resident inputs, L2 flushed before each frame."""
    import torch
    st = torch.cuda.Stream(device=dev)
    s = make_solver(pair, "plain", st)
    a = torch.from_numpy(pair["i0"]).to(dev)
    b = torch.from_numpy(pair["i1"]).to(dev)
    for _ in range(2):
        s.copy_images_from_device(a, b)
        s.solveStereoForwardMasked()
    torch.cuda.synchronize()
    ms = []
    for _ in range(steps):
        with torch.cuda.stream(st):
            flush.fill_(3.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        s.copy_images_from_device(a, b)
        s.solveStereoForwardMasked()
        e1.record(st)
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    return {"value": 1000.0 / float(np.mean(ms)), "unit": "frames/s", "ms_per_frame": float(np.mean(ms)),
            "p99_ms": float(np.percentile(ms, 99)), "storage": "fp32", "batch": 1}


def run_ours(args, rank, world, local):
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    from vfs_b200.build import build
    if rank == 0:
        build()
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist.barrier()
        build()  # other ranks see the built library (no-op when current)
    from vfs_b200.stereotgv import StereoBatch, StereoTgv
    fused = args.path == "fused"
    half = fused and args.storage == "fp16"
    batch = args.batch or (8 if fused else 1)
    pairs = [pair_cache(W0, H0, args.seed + 1000 * rank + k) for k in range(batch)]
    stream = torch.cuda.Stream(device=dev)
    solvers = [make_solver(p, args.path, stream, half) for p in pairs]
    sbatch = None
    if fused:
        sbatch = StereoBatch(half_storage=half, stream=stream)
        sbatch.set_fine_concurrency(args.fine)
        for s in solvers:
            sbatch.add(s)
    d_imgs = [(torch.from_numpy(p["i0"]).to(dev), torch.from_numpy(p["i1"]).to(dev)) for p in pairs]
    d_out = [torch.empty((H0, W0), dtype=torch.float32, device=dev) for _ in pairs]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # 256 MiB > L2
    torch.cuda.synchronize()

    def device_step():
        if fused:
            # one call: per pair (on its own lane) the device copy in, solve, copy out
            sbatch.solve_device(d_imgs, d_out)
            return
        for s, (a, b), o in zip(solvers, d_imgs, d_out):
            s.copy_images_from_device(a, b)
            s.solveStereoForwardMasked()
            s.copy_1d_disparity_to_device(o)

    # The timed region runs without the per-level profiling records (CUDA events inside the
    # captured graphs, which cost about 3 % of a step); its graphs are captured in the warm-up.
    for _ in range(args.warmup):
        device_step()
        flush.fill_(1.0)
    torch.cuda.synchronize()

    # ---- timed region: device-resident inputs -----------------------------------------
    launches0 = StereoTgv.launch_count()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(float(k))  # evict the previous step's working set from L2
            ev[k][0].record(stream)
            device_step()
            ev[k][1].record(stream)
        torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    launches = StereoTgv.launch_count() - launches0
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = float(sum(step_ms))
    # ---- roofline pass (not timed into the value): the same steps with the per-level
    # profiling records, whose graphs are captured by two untimed steps first
    for s in solvers:
        s.profile(True)
    for _ in range(2):
        device_step()
        flush.fill_(1.0)
    torch.cuda.synchronize()
    for s in solvers:
        s.profile_reset()
    StereoTgv.profile_epoch(stream)
    n_prof = max(1, min(args.steps, 5))
    for k in range(n_prof):
        with torch.cuda.stream(stream):
            flush.fill_(float(k))
        device_step()
    torch.cuda.synchronize()
    # roofline of the inner primal-dual loop: kind 0 (drop-in, one record per iteration)
    # Pairs solved on concurrent streams overlap, so the time is the union of the records'
    # intervals (time during which at least one inner group ran), not their sum.
    kind = 1 if args.path == "fused" else 0
    iv = np.concatenate([s.profile_intervals(kind) for s in solvers])
    for s in solvers:
        s.profile(False)
    # all levels, and the dominant kernel alone: the iteration kernel at full resolution (the
    # records with the largest pixel count)
    pi_all = float(iv[:, 2].sum()) if len(iv) else 0.0
    ms_all = union_ms(iv[:, :2]) if len(iv) else 0.0
    top = iv[iv[:, 2] == iv[:, 2].max()] if len(iv) else iv
    pi_l = float(top[:, 2].sum()) if len(top) else 0.0
    n_launch = int(top[:, 3].sum()) if len(top) else 0
    ms_l = union_ms(top[:, :2]) if len(top) else 0.0
    ms_sum = float((top[:, 1] - top[:, 0]).sum()) if len(top) else 0.0
    variants = solvers[0].iteration_variants() if fused else []
    n_variant_sets = len({tuple(s.iteration_variants()) for s in solvers}) if fused else 0
    # job-wide: frames of all replicas over the slowest replica's time
    from vfs_b200.replicas import job_rate
    frames, total_ms, value = job_rate(batch * args.steps, total_ms, device=dev)

    # ---- e2e: the public API with pinned host buffers -----------------------------------
    pinned = []  # page-locked host buffers (kept alive for the numpy views)
    h_in, h_out = [], []
    for p in pairs:
        ta = torch.from_numpy(p["i0"]).pin_memory()
        tb = torch.from_numpy(p["i1"]).pin_memory()
        to = torch.empty((H0, W0), dtype=torch.float32).pin_memory()
        pinned += [ta, tb, to]
        h_in.append((ta.numpy(), tb.numpy()))
        h_out.append(to.numpy())
    for s in solvers:
        s.set_stream(stream)
    e2e_steps = max(3, min(args.steps, 10))

    def host_step():
        outs = []
        if fused:
            # one call: per pair H2D of both images, solve, D2H of the disparity
            return sbatch.solve_host(h_in, h_out)
        for s, (a, b) in zip(solvers, h_in):
            s.copyImagesToDevice(a, b)
            s.solveStereoForwardMasked()
            outs.append(s.copy1DDisparityToHost())
        return outs

    # two warm calls: a solve alternates between two pointer states, each with its own graph
    host_step()
    host_step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    e2e_ms = []
    for _ in range(e2e_steps):
        with torch.cuda.stream(stream):
            flush.fill_(2.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        outs = host_step()
        e2e_ms.append(1000 * (time.perf_counter() - t0))
    _, e2e_total, e2e_value = job_rate(batch * e2e_steps, float(sum(e2e_ms)), device=dev)
    gpu_u = np.array(outs[0])

    result = None
    if rank == 0:
        peak, peak_kind = measured_peak()
        b_alg = B_ALG_FP16 if half else B_ALG_FP32
        achieved = (pi_l * b_alg / (ms_l / 1000.0) / 1e9) if ms_l > 0 else None
        achieved_all = (pi_all * b_alg / (ms_all / 1000.0) / 1e9) if ms_all > 0 else None
        storage = "fp16" if half else "fp32"
        kernel_key = f"fused_inner_{storage}" if args.path == "fused" else "plain_inner_iteration"
        px_per_launch = pi_l / n_launch if n_launch else 0.0
        tr = ncu_traffic(kernel_key)
        traffic = None
        if tr and n_launch > 0:
            traffic = tr["dram_bytes_per_pixel_iteration"] * px_per_launch
        per_frame = np.array(step_ms) / (1 if fused else batch)
        in_mask_frac = float(np.mean([(p["mask"] > 0).mean() for p in pairs]))
        result = {
            "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "848x800 fisheye stereo pairs, masked TGV-L1 solve, 5 levels x 3 warps x 50 iterations",
                       "path": args.path, "batch_per_gpu": batch, "storage": "fp16" if half else "fp32",
                       "full_resolution_pairs_at_once": "auto" if args.fine < 0 else args.fine,
                       "l2": "flushed (256 MiB write) before every step",
                       "seed": args.seed, "parallelism": f"replicas x{world}"},
            "latency_ms": {"p50": float(np.percentile(per_frame, 50)), "p99": float(np.percentile(per_frame, 99)),
                           "note": "per frame; a batched step completes all its frames together"},
            "roofline": {"bound": "latency", "peak_basis": "hbm (measured copy bandwidth)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                         "limiter": "instruction issue and short dependencies with the working sets of the pairs "
                                    "at full resolution resident in L2 (ncu, one cold launch: DRAM 24 %, issue 53 %, "
                                    "228 warp instructions per 32 pixels; stalls per issued instruction: long "
                                    "scoreboard 8.4, short scoreboard 3.1, not selected 2.1); frac > 1 is an "
                                    "algorithmic-bytes rate, not DRAM traffic",
                         "frac_in_mask": (achieved * in_mask_frac / peak) if achieved else None,
                         "frac_per_launch": (pi_l * b_alg / (ms_sum / 1000.0) / 1e9 / peak) if ms_sum > 0 else None,
                         "dram_gbs_per_launch_cold": (traffic / (ms_l / 1000.0 / n_launch) / 1e9)
                         if (traffic and n_launch and ms_l > 0) else None,
                         "kernel": ("full-resolution fused iteration (variant %s)" % (variants[0] if variants else "?"))
                         if fused else "drop-in inner iteration at full resolution",
                         "launches_measured": int(n_launch),
                         "algorithmic_bytes_per_launch": b_alg * px_per_launch,
                         "bytes_per_pixel_iteration": b_alg, "peak_kind": peak_kind,
                         "time_basis": "union of the full-resolution inner-loop event intervals of all pairs "
                                       "in the last step of a profiled pass run after the timed region on the "
                                       "same inputs (concurrent pairs overlap)",
                         "busy_ms": ms_l, "sum_of_interval_ms": ms_sum,
                         "all_levels": {"achieved": achieved_all, "frac": (achieved_all / peak) if achieved_all else None,
                                        "busy_ms": ms_all},
                         "iteration_variants_by_level": variants,
                         "distinct_variant_choices_over_pairs": n_variant_sets,
                         "traffic_source": "profiles/roofline_traffic.json (ncu) x pixels per launch"
                         if traffic is not None else None},
            "e2e": {"value": e2e_value, "unit": "frames/s", "h2d_bytes_per_step": batch * 2 * W0 * H0,
                    "d2h_bytes_per_step": batch * W0 * H0 * 4},
            "gpu_launches": int(launches),
            "clocks": clocks.summary(),
        }
        if fused and not args.no_plain:
            result["plain_dropin"] = plain_reference_run(pairs[0], dev, flush)
            result["speedup_vs_plain"] = value / result["plain_dropin"]["value"] / world
        if world == 1 and not args.no_cpu_baseline:
            fps, threads, u_cpu, n, dt = cpu_baseline(pairs[0])
            result["cpu_baseline"] = {"value": fps, "unit": "frames/s", "cores": threads, "kind": "port",
                                      "sample": f"{n} full 848x800 frame(s) in {dt:.1f} s, float64 oracle "
                                                f"(CPU restatement of the reference solver), OpenMP over rows"}
            result["cpu_baseline"]["single_thread_s_per_frame"] = cpu_single_thread_s(pairs[0])
            if fused:
                result["accuracy_vs_fp64_oracle"] = accuracy_report(pairs, outs, u_cpu, half, dev)
        if fused and world == 1 and not args.no_extras:
            # the metric's other configurations, run after the timed region on the same GPU
            mixed = run_mixed(args, emit=False)
            result["mixed_batch"] = {k: mixed[k] for k in ("value", "unit", "ms_per_step", "latency_ms",
                                                            "max_abs_vs_plain_px", "accuracy_vs_fp64_oracle",
                                                            "one_launch_per_level", "config")}
            srv = run_serving(args, emit=False, local=local)
            result["serving"] = dict(srv["serving"], config=srv["config"])
            result["warm_start"] = warm_start_report(args.seed)
        print(json.dumps(result), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return result


def run_mixed(args, emit=True):
    """Uneven batch: 8 x 848x800 + 4 x 640x480 + 4 x 424x400 pairs in one batched fused solve
    (float storage), checked per pair against the drop-in path."""
    import torch
    from vfs_b200 import synth
    from vfs_b200.build import build
    from vfs_b200.stereotgv import StereoBatch, StereoTgv
    build()
    dev = torch.device("cuda", 0)
    sizes = [(848, 800)] * 8 + [(640, 480)] * 4 + [(424, 400)] * 4
    sp = synth.SOLVER_PARAMS
    stream = torch.cuda.Stream(device=dev)
    pairs, solvers = [], []
    batch = StereoBatch(half_storage=False, stream=stream)
    batch.set_fine_concurrency(args.fine)
    for k, (w, h) in enumerate(sizes):
        p = pair_cache(w, h, args.seed + 100 + k)
        s = StereoTgv()
        s.set_solve_path(True, False)
        s.limitRange = synth.LIMIT_RANGE
        s.initialize(w, h, sp["beta"], sp["gamma"], sp["alpha0"], sp["alpha1"], sp["timestep_lambda"],
                     sp["lambda_"], synth.n_levels_for(w), sp["fScale"], sp["nWarpIters"], sp["nSolverIters"])
        s.copyMaskToDevice(p["mask"])
        s.loadVectorFields(p["tv"], p["cv"])
        s.set_stream(stream)
        batch.add(s)
        pairs.append(p)
        solvers.append(s)
    d_imgs = [(torch.from_numpy(p["i0"]).to(dev), torch.from_numpy(p["i1"]).to(dev)) for p in pairs]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step():
        for s, (a, b) in zip(solvers, d_imgs):
            s.copy_images_from_device(a, b)
        batch.solve(True)

    def time_steps():
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        out = []
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            torch.cuda.synchronize()
            out.append(e0.elapsed_time(e1))
        return out

    # concurrent per-pair graphs (the default), then the same batch as one launch per iteration
    # step and level over all pairs' tiles (no per-pair graphs, no full-resolution limit)
    ms = time_steps()
    batch.set_mode(True)
    ms_one = time_steps()
    batch.set_mode(False)
    # parity per size class: one more frame, against the drop-in path on a fresh handle pair,
    # and the error of both against the float64 oracle
    worst = 0.0
    acc = {}
    for k in (0, 8, 12):
        w, h = sizes[k]
        ref = StereoTgv()
        ref.limitRange = synth.LIMIT_RANGE
        ref.initialize(w, h, sp["beta"], sp["gamma"], sp["alpha0"], sp["alpha1"], sp["timestep_lambda"],
                       sp["lambda_"], synth.n_levels_for(w), sp["fScale"], sp["nWarpIters"], sp["nSolverIters"])
        ref.copyMaskToDevice(pairs[k]["mask"])
        ref.loadVectorFields(pairs[k]["tv"], pairs[k]["cv"])
        mine = StereoTgv()
        mine.set_solve_path(True, False)
        mine.limitRange = synth.LIMIT_RANGE
        mine.initialize(w, h, sp["beta"], sp["gamma"], sp["alpha0"], sp["alpha1"], sp["timestep_lambda"],
                        sp["lambda_"], synth.n_levels_for(w), sp["fScale"], sp["nWarpIters"], sp["nSolverIters"])
        mine.copyMaskToDevice(pairs[k]["mask"])
        mine.loadVectorFields(pairs[k]["tv"], pairs[k]["cv"])
        ref.copyImagesToDevice(pairs[k]["i0"], pairs[k]["i1"])
        ref.solveStereoForwardMasked()
        # the batch member has solved warmup + steps frames; solve a fresh fused handle once
        mine.copyImagesToDevice(pairs[k]["i0"], pairs[k]["i1"])
        mine.solveStereoForwardMasked()
        u_mine = mine.copy1DDisparityToHost()
        worst = max(worst, float(np.abs(ref.copy1DDisparityToHost() - u_mine).max()))
        acc["%dx%d" % (w, h)] = error_stats([u_mine], [fp64_u(pairs[k], w, h)], [pairs[k]["mask"]])
    per_step = float(np.mean(ms))
    line = {
        "metric": "mixed-size stereo frames/s (one batched fused solve per step)", "value": 16000.0 / per_step,
        "unit": "frames/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_step,
        "higher_is_better": True, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "8x848x800 + 4x640x480 + 4x424x400 pairs, masked solve, 3 warps x 50 iterations",
                   "storage": "fp32", "l2": "flushed (256 MiB write) before every step",
                   "full_resolution_pairs_at_once": "auto" if args.fine < 0 else args.fine},
        "latency_ms": {"p50": float(np.percentile(ms, 50)), "p99": float(np.percentile(ms, 99))},
        "max_abs_vs_plain_px": worst,
        "accuracy_vs_fp64_oracle": dict(acc, sample="the first pair of each size, one frame, fused FP32 (the "
                                        "drop-in path's bits); pixels inside the mask"),
        "one_launch_per_level": {"value": 16000.0 / float(np.mean(ms_one)), "unit": "frames/s",
                                 "ms_per_step": float(np.mean(ms_one)),
                                 "p99_ms": float(np.percentile(ms_one, 99))},
    }
    if emit:
        print(json.dumps(line), flush=True)
    return line


def warm_start_report(seed, n_frames=8, width=424, height=400):
    """Warm starts on a camera sequence with ground truth: mean |u - true disparity| inside the
    mask (where the true disparity is finite), and the GPU time per frame, for cold solves and
    for warm starts from the coarsest level and from two levels below it (those levels are
    skipped).  Fused path, FP16 storage; one stream of width x height."""
    import torch
    from vfs_b200 import synth
    from vfs_b200.stereotgv import StereoTgv
    fields, gen = synth.make_sequence(width, height, seed, n_frames, with_depth=True)
    frames = list(gen)
    sp = synth.SOLVER_PARAMS
    L = synth.n_levels_for(width)
    m = fields["mask"] > 0
    out = {"workload": f"one {width}x{height} stream, {n_frames} frames (<= 5 cm and 3 degrees per frame), "
                       "fused FP16; error inside the mask against the disparity the rendered depth implies"}
    for label, level in (("cold", -1), ("warm_full_pyramid", L - 1), ("warm_skip_2_levels", max(0, L - 3))):
        s = StereoTgv()
        s.set_solve_path(True, True)
        s.limitRange = synth.LIMIT_RANGE
        s.initialize(width, height, sp["beta"], sp["gamma"], sp["alpha0"], sp["alpha1"], sp["timestep_lambda"],
                     sp["lambda_"], L, sp["fScale"], sp["nWarpIters"], sp["nSolverIters"])
        s.copyMaskToDevice(fields["mask"])
        s.loadVectorFields(fields["tv"], fields["cv"])
        s.set_warm_start(level)
        errs, ms = [], []
        for k, (i0, i1, depth) in enumerate(frames):
            s.copyImagesToDevice(i0, i1)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s.solveStereoForwardMasked()
            s.synchronize()
            ms.append(1000 * (time.perf_counter() - t0))
            ut = synth.true_disparity(width, height, depth)
            ok = m & np.isfinite(ut)
            errs.append(float(np.abs(s.copy1DDisparityToHost() - ut)[ok].mean()))
        out[label] = {"start_level": level, "mean_abs_err_px_per_frame": errs,
                      "mean_abs_err_px_after_first": float(np.mean(errs[1:])),
                      "ms_per_frame_after_first": float(np.median(ms[2:] if len(ms) > 2 else ms))}
    return out


def run_serving(args, emit=True, rank=0, world=1, local=0):
    """6 camera streams (4 x 848x800, 2 x 424x400), 120 frames each along smooth random
    trajectories, Poisson arrivals totalling 180 requests/s, served by the continuous-batching
    server (fused, FP16 storage) and by the drop-in path one request at a time.  Under torchrun
    each rank serves the streams `replicas.assign_streams` gives it on its own GPU (the streams
    are independent) and rank 0 reports the job: all requests' latencies, all frames over the
    span from the first arrival to the last completion on any rank."""
    import torch
    from vfs_b200 import synth
    from vfs_b200.build import build
    from vfs_b200.replicas import merge_serving, my_streams
    from vfs_b200.serving import StereoServer, poisson_schedule, replay
    torch.cuda.set_device(local)
    if rank == 0:
        build()
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist.barrier()
        build()
    n_frames = max(8, min(120, args.steps * 12))
    cams_all = [(0, 848, 800), (1, 848, 800), (2, 848, 800), (3, 848, 800), (4, 424, 400), (5, 424, 400)]
    owned = set(my_streams({sid: (w, h) for sid, w, h in cams_all}, world, rank))
    cams = [c for c in cams_all if c[0] in owned]
    data = {}
    for sid, w, h in cams:
        fields, frames = synth.make_sequence_gpu(w, h, args.seed + 7 * sid, n_frames)
        data[sid] = (w, h, fields, frames)
    # one schedule for the whole job (every rank draws the same one), each rank replays its part
    rates = {sid: 30.0 for sid, _, _ in cams_all}
    sched = poisson_schedule(rates, {sid: n_frames for sid, _, _ in cams_all}, seed=args.seed)
    sched = [ev for ev in sched if ev[1] in owned]
    sp = synth.SOLVER_PARAMS
    params = dict(sp, limitRange=synth.LIMIT_RANGE)
    out = {}
    u64 = {}  # float64 oracle solves of the sampled frames, shared by both servers
    for label, kw in (("fused_fp16_batched", dict(path="fused", half_storage=True, max_batch=8, lanes=2)),
                      ("plain_fp32_one_at_a_time", dict(path="plain"))):
        srv = StereoServer(reserve_bytes=1 << 30, **kw)
        for sid, (w, h, fields, frames) in data.items():
            srv.open_stream(sid, w, h, fields["mask"], fields["tv"], fields["cv"], synth.n_levels_for(w), params)
        # warm the server with four frames per stream, so that each pair's graphs are captured
        # for the buffer assignments its frames cycle through before the timed replay
        for _ in range(4):
            for sid, (w, h, fields, frames) in data.items():
                srv.submit(sid, *frames[0])
            srv.run_until_idle()
        srv.done.clear()
        if world > 1:
            torch.distributed.barrier()  # the ranks start their replays together
        t_start = time.perf_counter()
        reqs = replay(srv, sched, {sid: d[3] for sid, d in data.items()}, realtime=True)
        st = srv.stats(since=t_start)
        # error against the float64 oracle on a sample: each stream's last frame (cold starts,
        # so a frame's disparity depends on that frame alone)
        last = {}
        for r in reqs:
            if r.u is not None and not r.cancelled and (r.stream_id not in last or r.seq > last[r.stream_id].seq):
                last[r.stream_id] = r
        us, refs, masks = [], [], []
        for sid, r in sorted(last.items()):
            w, h, fields, frames = data[sid]
            key = (sid, r.seq)
            if key not in u64:
                u64[key] = fp64_u(dict(i0=r.i0, i1=r.i1, mask=fields["mask"], tv=fields["tv"], cv=fields["cv"]), w, h)
            us.append(r.u)
            refs.append(u64[key])
            masks.append(fields["mask"])
        if us:
            st["accuracy_vs_fp64_oracle"] = dict(error_stats(us, refs, masks),
                                                 sample="the last frame of each stream this rank serves; "
                                                        "pixels inside the mask")
        if world > 1:
            d = [r for r in srv.done if r.t_submit >= t_start]
            job = merge_serving([r.latency_ms for r in d], min((r.t_submit for r in d), default=0.0),
                                max((r.t_done for r in d), default=0.0))
            st = dict(st, **job)
        st["arrival_rate_per_s"] = 180.0
        out[label] = st
        del srv
        torch.cuda.synchronize()
    line = {"metric": "serving: 6 camera streams, 180 requests/s Poisson, p50/p99 latency and frames/s",
            "value": out["fused_fp16_batched"].get("frames_per_s"), "unit": "frames/s", "n_gpus": world,
            "higher_is_better": True, "data": "synthetic",
            "config": {"workload": "4 x 848x800 + 2 x 424x400 streams, %d frames each, 30 req/s each" % n_frames,
                       "parallelism": "replicas x%d (streams assigned to ranks by pixels per frame)" % world},
            "serving": out}
    if emit and rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return line


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.mode == "mixed":
        if rank == 0:
            run_mixed(args)
        return
    if args.mode == "serving":
        run_serving(args, rank=rank, world=world, local=local)
        return
    run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()

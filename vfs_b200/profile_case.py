"""A small, self-contained solve for profilers: one batched fused solve of `--batch` seeded
848x800 pairs (no CUDA graph, so every kernel is an ordinary launch; no tile autotuning
unless --autotune 1, so the launch sequence is fixed).

    python -m vfs_b200.profile_case --batch 4 --half 1 [--frames 1] [--path fused|plain]
                                    [--mode concurrent|one_launch] [--autotune 0|1]
                                    [--variant -1..18] [--variants 1,1,8,9,9]

Launch order per frame: pyramid, then per level (coarse to fine) the level kernels and per
warp the prologue (k_warp_start, first warp of a level only), the derivatives, the fused
iterations and the epilogue (k_epilogue_warp_start, which also runs the next warp's prologue,
or k_epilogue_b after a level's last warp).  With the default iteration
variant (or --variant 0..2) each warp has 50 one-iteration launches: in the concurrent mode
each pair's solve is enqueued in turn (pair 0 first), so k_fused_iter launches 600..749 are
pair 0's full-resolution iterations (one pair per launch); in the one-launch mode every
launch carries all pairs, and launches 600..749 are the full-resolution iterations of the
batch.  With --variant 6..9 or 12..13 (K iterations per launch) each warp has 50 / K launches
of k_fused_iter_tb, coarsest level first; with --variant 14..15 each warp of a level that fits
a cluster's shared memory has one launch of k_fused_iter_cluster.
"""
from __future__ import annotations

import argparse
import os

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--half", type=int, default=1)
    ap.add_argument("--frames", type=int, default=1)
    ap.add_argument("--path", default="fused", choices=["fused", "plain"])
    ap.add_argument("--width", type=int, default=848)
    ap.add_argument("--height", type=int, default=800)
    ap.add_argument("--mode", default="concurrent", choices=["concurrent", "one_launch"])
    ap.add_argument("--autotune", type=int, default=0)
    ap.add_argument("--variant", type=int, default=-1, help="force one iteration-kernel variant")
    ap.add_argument("--variants", default="", help="force a variant per level, finest first, e.g. 1,1,8,9,9")
    a = ap.parse_args()
    from . import synth
    from .stereotgv import StereoBatch, StereoTgv
    w, h = a.width, a.height
    cache = f"/tmp/vfs_b200_pair_{w}x{h}_7.npz"
    if os.path.exists(cache):
        d = dict(np.load(cache))
    else:
        p = synth.make_pair(w, h, 7)
        d = dict(i0=p.i0, i1=p.i1, mask=p.mask, tv=p.tv, cv=p.cv)
        np.savez(cache, **d)
    sp = synth.SOLVER_PARAMS
    fused = a.path == "fused"
    batch = StereoBatch(half_storage=bool(a.half)) if fused else None
    if batch is not None:
        batch.set_graph(False)
        batch.set_autotune(bool(a.autotune))
        batch.set_mode(one_launch=a.mode == "one_launch")
        if a.variant >= 0:
            batch.set_iteration_variant(a.variant)
        if a.variants:
            batch.set_iteration_variants([int(v) for v in a.variants.split(",")])
    solvers = []
    for _ in range(a.batch if fused else 1):
        s = StereoTgv()
        s.set_solve_path(fused, bool(a.half) and fused)
        s.limitRange = synth.LIMIT_RANGE
        s.initialize(w, h, sp["beta"], sp["gamma"], sp["alpha0"], sp["alpha1"], sp["timestep_lambda"],
                     sp["lambda_"], synth.n_levels_for(w), sp["fScale"], sp["nWarpIters"], sp["nSolverIters"])
        s.copyMaskToDevice(d["mask"])
        s.loadVectorFields(d["tv"], d["cv"])
        if batch is not None:
            batch.add(s)
        solvers.append(s)
    for _ in range(a.frames):
        for s in solvers:
            s.copyImagesToDevice(d["i0"], d["i1"])
        if batch is not None:
            batch.solve(True)
        else:
            solvers[0].solveStereoForwardMasked()
    u = solvers[0].copy1DDisparityToHost()
    print("done", float(u[h // 2, w // 2]))


if __name__ == "__main__":
    main()

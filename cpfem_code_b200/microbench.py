"""Constitutive micro-benchmark: 2^20 independent FCC material points.

Seeded uniform-SO(3) orientations, Gaussian strain increments scaled to
Frobenius norm 1e-3, CRSS per system uniform in [tau0, 2 tau0], the stress
increment seeded with the elastic predictor so every point takes the plastic
branch of DSTRSS.  Times `fas_gpu_constitutive` (one DSTRSS per point) with
CUDA events on the library stream; reports GP-updates/s and the algorithmic
operation rate from the per-point counts.  Parity with the CPU checker is
covered by tests/test_gpu_parity.py.

    python -m cpfem_code_b200.microbench [--points 1048576] [--reps 5]
"""
import argparse
import json
import sys

import numpy as np

from . import GpuSolver, generator


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--points", type=int, default=1 << 20)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--mode", type=int, default=0, help="FAS_MODE_* mask (8 = one warp per point)")
    a = ap.parse_args()
    p = generator.point_batch(a.points, seed=1)
    g = GpuSolver(p.copy(), mode=a.mode)
    g.constitutive(1, 1)                 # warm-up
    ops = g.cp_ops()
    it, _ = g.cp_stats()
    times = []
    for _ in range(a.reps):
        g.upload(p)                      # same input every repetition
        g.profile(2)
        g.constitutive(1, 1)
        prof = g.profile(0)
        times.append(prof["ms_constitutive"] / 1e3)
    t = float(np.median(times))
    out = {"points": a.points, "mode": a.mode, "s_per_pass": t, "gp_updates_per_s": a.points / t,
           "ops_per_update": float(ops.mean()), "ops_per_s": float(ops.sum()) / t,
           "mean_cpstrs_iters": float(it.mean())}
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())

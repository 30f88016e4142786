"""A small profiling case for ncu: the first Newton iteration of the 64^3
workload (one ELVALS + SUVALS and one complete FACSLS solve), ~1 GB on the
device, inputs larger than L2.

    python -m cpfem_code_b200.profile_case [--workload cube64] [--mode 0]
    python -m cpfem_code_b200.profile_case --adjoint 16384

--adjoint N instead runs the adjoint once on N independent FCC points: a
replay of 4 increments (checkpoints every 2) with its gradients
(k_replay_fwd, k_replay_adj).
"""
import argparse
import sys

import numpy as np

from . import GpuSolver, ReplayHistory, generator


def adjoint_case(n: int) -> int:
    p = generator.point_batch(n, seed=1)
    rng = np.random.default_rng(2)
    de = np.stack([p.de * (1.0 + 0.2 * rng.standard_normal(p.de.shape)) for _ in range(4)])
    dr = 2e-4 * rng.standard_normal((4, n, 3))
    h = ReplayHistory(de, dr, np.full(4, p.tiem[0]), np.ones(n), np.zeros(n), chk_every=2)
    g = GpuSolver(p)
    out = g.adjoint_grad(h)
    print(f"adjoint: {n} points x 4 increments, J {out['J']:.4e}")
    g.close()
    return 0


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="cube64")
    ap.add_argument("--mode", type=int, default=0)
    ap.add_argument("--adjoint", type=int, default=0, help="points of the adjoint case (0: FACSLS case)")
    a = ap.parse_args()
    if a.adjoint:
        return adjoint_case(a.adjoint)
    p = generator.workload(a.workload)
    g = GpuSolver(p, mode=a.mode)
    g.update_node()
    g.elvals(1, 1)
    g.suvals(1)
    sweeps, err = g.facsls()
    print(f"{a.workload}: FACSLS {sweeps} sweeps, error {err:.3e}")
    g.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())

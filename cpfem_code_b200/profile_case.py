"""A small profiling case for ncu: the first Newton iteration of the 64^3
workload (one ELVALS + SUVALS and one complete FACSLS solve), ~1 GB on the
device, inputs larger than L2.

    python -m cpfem_code_b200.profile_case [--workload cube64] [--mode 0]
"""
import argparse
import sys

from . import GpuSolver, generator


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="cube64")
    ap.add_argument("--mode", type=int, default=0)
    a = ap.parse_args()
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

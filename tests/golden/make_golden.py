"""Writes the golden increment fixtures of tests/golden/ with the CPU checker.

    python tests/golden/make_golden.py [--threads N] [--only NAME]

The reference ships no expected outputs and cannot be compiled here (it is
Fortran), so these fixtures are the checker's (oracle/, the C++ restatement
of src/fasolt) own results on the named workloads, recorded once so that the
GPU tests compare against them without re-running the checker:

* ``cube8_colour`` / ``cube8_natural``: the 8^3 cube, one grain per element,
  10 increments to 1 % (generator workload ``cube8``);
* ``cube16_colour``: the 16^3 cube, 20 increments to 2 % (workload
  ``cube16``); ``cube16_natural``: its first 4 increments, the ones whose
  Newton loop converges (increments 5-20 stop at maxit = 100 in either SOR
  order, and the natural order's sequential sweeps make them slow to
  record).

``colour`` runs FACSLS in the device path's multicolour node order;
``natural`` in the reference's own natural DOF order (Stif_sol.f90:189-197,
oracle mode FAS_MODE_SOR_NATURAL).  Each file holds, per increment, the
Newton iteration count, the SOR sweeps of every Newton iteration and the
mean s11 (the macroscopic stress-strain point), and after the last
increment the per-GP stress, slip resistances and accumulated slip and the
nodal coordinates.  ``inputs_sha`` is a digest of the generated inputs, so
tests/test_golden.py can check that the generator still makes the same
problem.
"""
from __future__ import annotations

import argparse
import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# increments recorded: (multicolour order, natural order)
CASES = {
    "cube8": (10, 10),
    "cube16": (20, 4),
}


def inputs_sha(p) -> str:
    """Digest of everything the generator decides: mesh, boundary codes,
    materials, orientations, loading and control."""
    h = hashlib.sha256()
    for a in (p.x, p.ln, p.lg, p.le, p.lt, p.ib, p.sv[:, :3], p.sv[:, 3:3 + int(p.nss.max())], p.e,
              p.ab, p.an, p.ampar, p.tiem, p.x_spec):
        h.update(np.ascontiguousarray(a).tobytes())
    h.update(repr((p.ctrl.toler, p.ctrl.maxit, p.ctrl.alpha)).encode())
    return h.hexdigest()[:32]


def run(name: str, natural: bool, threads: int, ninc: int | None = None) -> dict:
    from cpfem_code_b200 import abi, generator
    from oracle import OracleSolver
    p = generator.workload(name)
    sha = inputs_sha(p)
    ninc = ninc or CASES[name][1 if natural else 0]
    mode = abi.FAS_MODE_SOR_NATURAL if natural else abi.FAS_MODE_PLAIN
    o = OracleSolver(p, 8, mode=mode, threads=threads)
    nits, sweeps, macro = [], [], []
    for inc in range(1, ninc + 1):
        rep, _ = o.increment(inc)
        o.download()
        nits.append(len(rep))
        sweeps.extend(r["sor_sweeps"] for r in rep)
        macro.append(p.st[:, 0].mean())
    o.close()
    ns = int(p.nss.max())
    return dict(inputs_sha=sha, natural=natural, ninc=ninc, newton_iters=np.array(nits, np.int32),
                sor_sweeps=np.array(sweeps, np.int32), macro_s11=np.array(macro), st=p.st.copy(),
                crss=p.sv[:, 3:3 + ns].copy(), cumslip=p.cumslip[:, :ns].copy(), x=p.x.copy())


def path(name: str, natural: bool) -> str:
    return os.path.join(HERE, f"{name}_{'natural' if natural else 'colour'}.npz")


def load(name: str, natural: bool) -> dict:
    with np.load(path(name, natural)) as z:
        return {k: z[k] for k in z.files}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--only", default=None, help="one case, e.g. cube8_natural")
    a = ap.parse_args()
    for name in CASES:
        for natural in (False, True):
            tag = f"{name}_{'natural' if natural else 'colour'}"
            if a.only and a.only != tag:
                continue
            t0 = time.time()
            d = run(name, natural, a.threads)
            np.savez_compressed(path(name, natural), **d)
            print(f"{tag}: {time.time() - t0:.0f} s, Newton {d['newton_iters'].tolist()}", flush=True)


if __name__ == "__main__":
    main()

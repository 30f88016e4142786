"""The consistent-tangent mode on the device against the checker: the
tangent of every constitutive point, and whole increments of the 16^3 cube
whose Newton loops converge (the first four) with identical iteration
counts.  The Newton counts of both tangents are printed side by side."""
import numpy as np
import pytest

from cpfem_code_b200 import GpuSolver, abi, generator
from oracle import OracleSolver

pytestmark = pytest.mark.gpu
TC = abi.FAS_MODE_TANGENT_CONSISTENT


def rel(a, b):
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / s)


def test_point_tangent_matches_checker():
    p = generator.point_batch(2048, seed=11)
    pg, po = p.copy(), p.copy()
    g, o = GpuSolver(pg, mode=TC), OracleSolver(po, 8, mode=TC, threads=8)
    g.constitutive(1, 1)
    o.constitutive(1, 1)
    assert rel(g.tangent(), o.tangent()) < 1e-11
    g.download()
    o.download()
    assert rel(pg.ds, po.ds) < 1e-11   # the stress update itself is unchanged
    g.close()
    o.close()


def test_cube16_newton_counts_both_tangents():
    p = generator.workload("cube16")
    counts = {}
    for tag, mode in (("reference", abi.FAS_MODE_PLAIN), ("consistent", TC)):
        pg, po = p.copy(), p.copy()
        g = GpuSolver(pg, mode=mode)
        o = OracleSolver(po, 8, mode=mode, threads=8) if tag == "consistent" else None
        nits = []
        for inc in range(1, 5):
            rg, _ = g.increment(inc)
            nits.append(len(rg))
            if o is not None:
                ro, _ = o.increment(inc)
                assert [r["sor_sweeps"] for r in rg] == [r["sor_sweeps"] for r in ro]
        g.download()
        if o is not None:
            o.download()
            assert rel(pg.st, po.st) < 1e-10
            o.close()
        g.close()
        counts[tag] = nits
    print(f"16^3 increments 1-4, Newton iterations: reference tangent {counts['reference']}, "
          f"consistent tangent {counts['consistent']}")

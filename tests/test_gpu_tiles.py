"""The persistent tile solve (FAS_MODE_SOR_TILES, k_sor_tiles) against the
colour kernels (one launch per colour) and the checker.

The tile kernel visits every row with the same operands as the global colour
order, so with equal sweep counts its iterates equal the colour kernels' to
the bit; only the stopping test's sum runs in another order (tile shares
instead of per-CTA shares), which moves err in its last bits.
"""
import numpy as np
import pytest

from cpfem_code_b200 import GpuSolver, abi, generator
from oracle import OracleSolver

pytestmark = pytest.mark.gpu
GRID = abi.FAS_MODE_SOR_GRID
TILES = abi.FAS_MODE_SOR_GRID | abi.FAS_MODE_SOR_TILES


def rel(a, b):
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / s) if s > 0 else float(np.abs(a - b).max())


def first_solve(p, mode):
    q = p.copy()
    g = GpuSolver(q, mode=mode)
    g.update_node()
    g.elvals(1, 1)
    g.suvals(1)
    sweeps, err = g.facsls()
    g.download()
    g.close()
    return q, sweeps, err


@pytest.mark.parametrize("n,fp32", [(8, False), (12, False), (12, True), (21, False)])
def test_first_solve_equals_colour_kernels(n, fp32):
    p = generator.cube_config(n=n, ninc=2, grain=1, seed=n)
    extra = abi.FAS_MODE_SOR_FP32 if fp32 else 0
    a, sa, ea = first_solve(p, GRID | extra)
    b, sb, eb = first_solve(p, TILES | extra)
    assert sa == sb
    np.testing.assert_array_equal(a.ddx, b.ddx)
    assert abs(ea - eb) <= 1e-12 * abs(ea)


@pytest.mark.parametrize("fp32", [False, True])
def test_increments_equal_colour_kernels_and_checker(fp32):
    # every boundary face fixed (fs3pre's xfree = 1): the increments converge
    p = generator.structured_cube(n=(12, 12, 12), ninc=3, grain=2, seed=3, xfree=1)
    extra = abi.FAS_MODE_SOR_FP32 if fp32 else 0
    pa, pb, po = p.copy(), p.copy(), p.copy()
    ga, gb = GpuSolver(pa, mode=GRID | extra), GpuSolver(pb, mode=TILES | extra)
    o = OracleSolver(po, 8, threads=8) if not fp32 else None
    for inc in (1, 2, 3):
        ra, _ = ga.increment(inc)
        rb, _ = gb.increment(inc)
        assert [r["sor_sweeps"] for r in ra] == [r["sor_sweeps"] for r in rb]
        if o is not None:
            ro, _ = o.increment(inc)
            assert [r["sor_sweeps"] for r in ro] == [r["sor_sweeps"] for r in rb]
    ga.download()
    gb.download()
    for name in ("x", "dx", "st", "sv"):
        np.testing.assert_array_equal(getattr(pa, name), getattr(pb, name))
    if o is not None:
        o.download()
        assert rel(pb.st, po.st) < 1e-10
        assert rel(pb.x, po.x) < 1e-10


def test_tile_layout_covers_every_node():
    """Large enough for one tile per SM: the solve touches every DOF (a
    converged solve leaves no row of the right-hand side unvisited)."""
    p = generator.cube_config(n=24, ninc=1, grain=2, seed=24)
    b, sb, _ = first_solve(p, TILES)
    a, sa, _ = first_solve(p, GRID)
    assert sa == sb
    np.testing.assert_array_equal(a.ddx, b.ddx)

"""20-node, 8-Gauss-point bricks (``lt = 22``, SHAPE_22) on the sm_100a path
against the CPU checker, through the C ABI.

Rows of a 20-node brick mesh hold up to 81 node blocks, so these meshes use
the 81-slot row layout; small meshes solve in one CTA (three slots per
lane), FAS_MODE_SOR_GRID forces the 81-slot colour kernels.  The
tolerances are those of the 8-node parity tests: 1e-11 relative for FP64
state after one pass, 1e-10 after whole increments, bit-exact for integers
(pattern, colouring, iteration counts).
"""
import numpy as np
import pytest

from cpfem_code_b200 import GpuSolver, abi, generator
from oracle import OracleSolver

pytestmark = pytest.mark.gpu
LD = 256          # >= 3 x 81 columns per DOF row


def rel(a, b):
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / s) if s > 0 else float(np.abs(a - b).max())


def pair(p, threads=8, mode=abi.FAS_MODE_PLAIN):
    pg, po = p.copy(), p.copy()
    return GpuSolver(pg, mode=mode), OracleSolver(po, 8, threads=threads), pg, po


@pytest.mark.parametrize("n", [(1, 1, 1), (2, 2, 2), (3, 2, 2)])
def test_pattern_and_colouring_20_node(n):
    p = generator.structured_cube(n=n, ninc=1, seed=1, nodes=20)
    g, o, _, _ = pair(p)
    np.testing.assert_array_equal(g.pattern(LD), o.pattern(LD))
    cg, ng = g.colouring()
    co, no = o.colouring()
    np.testing.assert_array_equal(cg, co)
    assert ng == no
    col = cg[p.ln - 1]
    assert all(len(set(r)) == 20 for r in col)   # no two nodes of an element share a colour


def test_elvals_suvals_facsls_20_node():
    p = generator.structured_cube(n=(2, 2, 2), ninc=2, seed=3, nodes=20)
    g, o, pg, po = pair(p)
    for s in (g, o):
        s.update_node()
        s.elvals(1, 1)
    g.download()
    o.download()
    assert rel(pg.fc, po.fc) < 1e-11
    assert rel(pg.ds, po.ds) < 1e-11
    Kg, Ko = g.stiffness(LD), o.stiffness(LD)
    assert rel(Kg, Ko) < 1e-11
    for s in (g, o):
        s.suvals(1)
    g.download()
    o.download()
    assert rel(pg.ddx, po.ddx) < 1e-11
    sg, so = g.facsls(), o.facsls()
    assert sg[0] == so[0]
    g.download()
    o.download()
    assert rel(pg.ddx, po.ddx) < 1e-10


@pytest.mark.parametrize("n,ninc,mode", [((1, 1, 1), 2, abi.FAS_MODE_PLAIN),      # one-CTA solve
                                         ((2, 2, 2), 2, abi.FAS_MODE_PLAIN),
                                         ((3, 3, 2), 1, abi.FAS_MODE_PLAIN),
                                         ((2, 2, 2), 2, abi.FAS_MODE_SOR_GRID),   # 81-slot colour kernels
                                         ((3, 3, 2), 1, abi.FAS_MODE_SOR_GRID)])
def test_increments_match_20_node(n, ninc, mode):
    p = generator.structured_cube(n=n, ninc=ninc, seed=7, nodes=20)
    g, o, pg, po = pair(p, mode=mode)
    for inc in range(1, ninc + 1):
        rg, _ = g.increment(inc)
        ro, _ = o.increment(inc)
        assert [r["sor_sweeps"] for r in rg] == [r["sor_sweeps"] for r in ro]
        assert len(rg) == len(ro)
        g.download()
        o.download()
        for name in ("st", "ep", "x", "dx", "eps"):
            assert rel(getattr(pg, name), getattr(po, name)) < 1e-10, name
        assert rel(pg.sv[:, :15], po.sv[:, :15]) < 1e-10
        assert abs(pg.st[:, 0].mean() - po.st[:, 0].mean()) <= 1e-10 * abs(po.st[:, 0].mean())


@pytest.mark.parametrize("n,nodes,tie", [((3, 3, 3), 8, (True, True, True)),
                                         ((3, 3, 3), 8, (False, True, True)),
                                         ((2, 2, 2), 20, (True, True, True))])
def test_increments_with_periodic_ties(n, nodes, tie):
    """SETTIES's tie elements (periodic boundary conditions, lt 1-6) after the
    bricks: the pattern, the penalty rows and whole increments match the
    checker."""
    p = generator.structured_cube(n=n, ninc=2, seed=5, xfree=1, nodes=nodes, ties=tie)
    assert p.meta["ties"] > 0
    g, o, pg, po = pair(p)
    np.testing.assert_array_equal(g.pattern(LD), o.pattern(LD))
    for inc in (1, 2):
        rg, _ = g.increment(inc)
        ro, _ = o.increment(inc)
        assert [r["sor_sweeps"] for r in rg] == [r["sor_sweeps"] for r in ro]
        g.download()
        o.download()
        for name in ("st", "x", "dx"):
            assert rel(getattr(pg, name), getattr(po, name)) < 1e-10, name


def test_fp32_sor_refinement_20_node():
    """The tuned form (FP32 matrix sweeps, FP64 residual refinement) on
    81-slot rows: FP32 rows are bulk-copied like FP64 rows; the stress stays
    within the stated error of the FP64 checker."""
    p = generator.structured_cube(n=(3, 3, 2), ninc=1, seed=5, nodes=20)
    g, o, pg, po = pair(p, mode=abi.FAS_MODE_SOR_GRID | abi.FAS_MODE_SOR_FP32)
    g.increment(1)
    o.increment(1)
    g.download()
    o.download()
    per_point = np.abs(pg.st - po.st).max() / np.abs(po.st).max()
    macro = abs(pg.st[:, 0].mean() - po.st[:, 0].mean()) / abs(po.st[:, 0].mean())
    assert per_point < 1e-5 and macro < 1e-6

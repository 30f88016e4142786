"""10-node tetrahedra (``lt = 21``, SHAPE_21, four Gauss points) and 15-node
wedges (``lt = 23``, SHAPE_23, six Gauss points) on the sm_100a path against
the CPU checker, through the C ABI.

The meshes split every brick of the lattice into 6 tetrahedra (along its
main diagonal) or 2 wedges (along a diagonal plane of its x-y faces), with
mid-edge nodes; a node then joins up to 24 tetrahedra or 12 wedges and up to
65 or 71 node blocks per row (the 81-slot layout).  Tolerances as for the
other element types: 1e-11 relative for FP64 state after one pass, 1e-10
after whole increments, bit-exact for integers.
"""
import numpy as np
import pytest

from cpfem_code_b200 import GpuSolver, abi, generator
from oracle import OracleSolver

pytestmark = pytest.mark.gpu
LD = 256


def rel(a, b):
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / s) if s > 0 else float(np.abs(a - b).max())


def pair(p, threads=8, mode=abi.FAS_MODE_PLAIN):
    pg, po = p.copy(), p.copy()
    return GpuSolver(pg, mode=mode), OracleSolver(po, 8, threads=threads), pg, po


@pytest.mark.parametrize("nodes", [10, 15])
def test_pattern_and_colouring(nodes):
    p = generator.structured_cube(n=(2, 2, 2), ninc=1, seed=1, nodes=nodes)
    g, o, _, _ = pair(p)
    np.testing.assert_array_equal(g.pattern(LD), o.pattern(LD))
    cg, ng = g.colouring()
    co, no = o.colouring()
    np.testing.assert_array_equal(cg, co)
    assert ng == no
    col = cg[p.ln - 1]
    assert all(len(set(r)) == nodes for r in col)


@pytest.mark.parametrize("nodes", [10, 15])
def test_elvals_suvals_facsls(nodes):
    p = generator.structured_cube(n=(2, 2, 2), ninc=2, seed=3, nodes=nodes)
    g, o, pg, po = pair(p)
    for s in (g, o):
        s.update_node()
        s.elvals(1, 1)
    g.download()
    o.download()
    assert rel(pg.fc, po.fc) < 1e-11
    assert rel(pg.ds, po.ds) < 1e-11
    assert rel(g.stiffness(LD), o.stiffness(LD)) < 1e-11
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


@pytest.mark.parametrize("nodes,n,xfree,mode", [(10, (2, 2, 2), 1, abi.FAS_MODE_PLAIN),      # one-CTA solve
                                                (10, (4, 4, 4), 3, abi.FAS_MODE_PLAIN),      # colour kernels
                                                (15, (2, 2, 2), 1, abi.FAS_MODE_PLAIN),
                                                (15, (4, 4, 3), 3, abi.FAS_MODE_PLAIN),
                                                (15, (3, 3, 3), 1, abi.FAS_MODE_SOR_GRID)])
def test_increments_match(nodes, n, xfree, mode):
    p = generator.structured_cube(n=n, ninc=2, seed=5, nodes=nodes, xfree=xfree)
    g, o, pg, po = pair(p, mode=mode)
    for inc in (1, 2):
        rg, _ = g.increment(inc)
        ro, _ = o.increment(inc)
        assert [r["sor_sweeps"] for r in rg] == [r["sor_sweeps"] for r in ro]
        g.download()
        o.download()
        for name in ("st", "x", "dx"):
            assert rel(getattr(pg, name), getattr(po, name)) < 1e-10, name
        assert rel(pg.sv[:, :15], po.sv[:, :15]) < 1e-10

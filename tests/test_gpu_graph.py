"""NRITER as one CUDA graph per increment (FAS_MODE_GRAPH) against the
host-driven loop.

The graph holds the same launches with the same shapes and operands: the
Newton loop (Stif_sol.f90:32-77) and FACSLS's sweep loop
(Stif_sol.f90:190-212) become conditional while nodes whose conditions the
device sets, the damping factor alp2 is computed on the device from the same
norms, and the sweeps run four to a pass as in the host loop's chunks (a
sweep after convergence does nothing); the FP32 solve runs its cycles of 16
sweeps, fold and FP64 residual as the loop body.  So iterates, report lines and
counters equal the host loop's to the bit, and the FAFERR codes of a failed
iteration are the same.
"""
import numpy as np
import pytest

from cpfem_code_b200 import GpuSolver, abi, generator

import faferr_cases

pytestmark = pytest.mark.gpu
GRAPH = abi.FAS_MODE_GRAPH
GRID = abi.FAS_MODE_SOR_GRID
STATE = ("x", "dx", "st", "ep", "sv", "eps", "rt", "srate", "cumslip")


def run(p, mode, incs):
    q = p.copy()
    g = GpuSolver(q, mode=mode)
    reps = [g.increment(inc)[0] for inc in incs]
    prof = g.profile(0)
    g.download()
    g.close()
    return q, reps, prof


CASES = {
    # 8^3 one-point bricks: grid-wide sweeps, one launch per colour
    "cube8": (lambda: generator.structured_cube(n=(8, 8, 8), ninc=3, grain=2, seed=5, xfree=1), 0),
    # 3^3: 64 nodes, the one-CTA solve under the graph's if node
    "cube3": (lambda: generator.structured_cube(n=(3, 3, 3), ninc=3, grain=1, seed=6, xfree=1), 0),
    # the small mesh with the grid-wide sweeps forced
    "cube3_grid": (lambda: generator.structured_cube(n=(3, 3, 3), ninc=3, grain=1, seed=6, xfree=1), GRID),
    # 20-node bricks: the 81-slot colour kernel
    "brick20": (lambda: generator.structured_cube(n=(4, 4, 4), ninc=3, grain=1, seed=7, xfree=1, nodes=20),
                GRID),
    # the FP32 solve: cycles of 16 sweeps, fold and FP64 residual
    "cube8_fp32": (lambda: generator.structured_cube(n=(8, 8, 8), ninc=3, grain=2, seed=5, xfree=1),
                   abi.FAS_MODE_SOR_FP32),
    "brick20_fp32": (lambda: generator.structured_cube(n=(4, 4, 4), ninc=3, grain=1, seed=7, xfree=1, nodes=20),
                     GRID | abi.FAS_MODE_SOR_FP32),
    # constitutive passes from the device queue
    "cube8_queue": (lambda: generator.structured_cube(n=(8, 8, 8), ninc=3, grain=2, seed=5, xfree=1),
                    abi.FAS_MODE_CP_QUEUE),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_graph_equals_host_loop(case):
    make, extra = CASES[case]
    p = make()
    a, ra, pa = run(p, extra, (1, 2, 3))
    b, rb, pb = run(p, extra | GRAPH, (1, 2, 3))
    assert ra == rb
    for name in STATE:
        np.testing.assert_array_equal(getattr(a, name), getattr(b, name), err_msg=name)
    for key in ("sor_sweeps", "n_constitutive", "gp_updates", "n_assembly"):
        assert pa[key] == pb[key], key


def test_graph_kept_per_increment_and_dropped_on_mode_change():
    """A second run of the same increments reuses the graphs; a mode change
    rebuilds them with the new mode's launches."""
    p = generator.structured_cube(n=(6, 6, 6), ninc=4, grain=1, seed=8, xfree=1)
    a, ra, _ = run(p, 0, (1, 2, 3, 4))
    q = p.copy()
    g = GpuSolver(q, mode=GRAPH)
    rb = [g.increment(1)[0], g.increment(2)[0]]
    g.set_mode(GRAPH | abi.FAS_MODE_CP_QUEUE)
    rb += [g.increment(3)[0]]
    g.set_mode(GRAPH)
    rb += [g.increment(4)[0]]
    g.download()
    g.close()
    assert ra == rb
    for name in STATE:
        np.testing.assert_array_equal(getattr(a, name), getattr(q, name), err_msg=name)


@pytest.mark.parametrize("case", ["903", "904"])
def test_graph_faferr_codes(case):
    make, call, code = faferr_cases.CASES[case]
    p = make()
    got = []
    for mode in (0, GRAPH):
        g = GpuSolver(p.copy(), mode=mode)
        with pytest.raises(abi.FasError) as ei:
            call(g)
        got.append((ei.value.code, g.last_report))
        g.close()
    assert got[0][0] == got[1][0] == code
    assert got[0][1] == got[1][1]

"""Symmetric FP32 rows (FAS_MODE_SOR_SYM with FAS_MODE_SOR_FP32) on the device.

The FP32 sweeps stream each off-diagonal block once and push its transposed
product into per-node accumulators with vector atomic adds.  That is the
same iteration as the full FP32 rows up to FP32 rounding, but the order of
the atomic adds varies, so these tests hold the results to the tuned form's
error bounds against the FP64 checker (1e-5 per point, 1e-6 macroscopic)
and to the full FP32 rows' results within FP32-sweep rounding, not to the
bit.  The streamed bytes per sweep (fas_gpu_profile) show which rows ran.
"""
import numpy as np
import pytest

from cpfem_code_b200 import GpuSolver, abi, generator
from oracle import OracleSolver

pytestmark = pytest.mark.gpu

FP32 = abi.FAS_MODE_SOR_GRID | abi.FAS_MODE_SOR_FP32
SYM = FP32 | abi.FAS_MODE_SOR_SYM
SYM_ROW_BYTES = (136 + 16) * 4      # brow_of(15) FP32 values + crow_of(15) column ids


def _assembled(p, mode):
    g = GpuSolver(p.copy(), mode=mode)
    g.update_node()
    g.elvals(1, 1)
    g.suvals(1)
    return g


def _bytes_per_sweep(g):
    g.profile(1)
    sweeps, err = g.facsls()
    prof = g.profile(0)
    return sweeps, err, prof["sor_bytes"] / max(prof["sor_sweeps"], 1)


@pytest.mark.parametrize("n", [(12, 12, 12), (16, 12, 9)])
def test_sym_facsls_matches_full_fp32_rows(n):
    """One FACSLS of the first Newton iteration: the symmetric rows' solution
    equals the full FP32 rows' to FP32-sweep rounding, with the same sweep
    count to within two, and the sweeps stream 608 bytes per row."""
    p = generator.structured_cube(n=n, ninc=1, seed=3)
    a, b = _assembled(p, FP32), _assembled(p, SYM)
    try:
        sa, _, _ = _bytes_per_sweep(a)
        sb, _, bps = _bytes_per_sweep(b)
        assert bps == pytest.approx(SYM_ROW_BYTES * p.nnod)
        xa, xb = a.download(p.copy()).ddx, b.download(p.copy()).ddx
        scale = np.abs(xa).max()
        d = np.abs(xa - xb).max() / scale
        print(f"{n}: sweeps full {sa} symmetric {sb}, solution difference {d:.2e}")
        assert abs(sa - sb) <= 2
        assert d < 1e-5
    finally:
        a.close()
        b.close()


def test_sym_increments_against_checker():
    """Two increments of the 12^3 cube in the tuned form on symmetric rows
    against the FP64 checker: the tuned form's error bounds."""
    p = generator.structured_cube(n=(12, 12, 12), ninc=2, seed=5)
    pg, po = p.copy(), p.copy()
    g, o = GpuSolver(pg, mode=SYM), OracleSolver(po, 8, threads=8)
    try:
        for inc in (1, 2):
            rg, _ = g.increment(inc)
            ro, _ = o.increment(inc)
            assert abs(len(rg) - len(ro)) <= 1
        g.download()
        o.download()
        smax = np.abs(po.st).max()
        per_point = np.abs(pg.st - po.st).max() / smax
        macro = abs(pg.st[:, 0].mean() - po.st[:, 0].mean()) / abs(po.st[:, 0].mean())
        print(f"symmetric FP32 rows: per-point {per_point:.2e}, macroscopic {macro:.2e}")
        assert per_point < 1e-5 and macro < 1e-6
    finally:
        g.close()


def test_sym_graph_increment():
    """The increment as one CUDA graph (FAS_MODE_GRAPH) on symmetric rows:
    the same Newton count as the host-driven loop and results within the
    tuned form's bounds of it."""
    p = generator.structured_cube(n=(12, 12, 12), ninc=1, seed=5)
    ph, pgr = p.copy(), p.copy()
    h, gr = GpuSolver(ph, mode=SYM), GpuSolver(pgr, mode=SYM | abi.FAS_MODE_GRAPH)
    try:
        rh, _ = h.increment(1)
        rr, _ = gr.increment(1)
        assert abs(len(rh) - len(rr)) <= 1
        h.download()
        gr.download()
        smax = np.abs(ph.st).max()
        assert np.abs(ph.st - pgr.st).max() / smax < 1e-5
    finally:
        h.close()
        gr.close()


def test_sym_no_effect_on_20_node_rows():
    """20-node (81-slot) rows keep the full FP32 rows: bit-identical
    results with and without FAS_MODE_SOR_SYM."""
    p = generator.structured_cube(n=(3, 3, 3), ninc=1, seed=7, nodes=20)
    a, b = _assembled(p, FP32), _assembled(p, SYM)
    try:
        sa, _, ba = _bytes_per_sweep(a)
        sb, _, bb = _bytes_per_sweep(b)
        assert sa == sb and ba == bb
        np.testing.assert_array_equal(a.download(p.copy()).ddx, b.download(p.copy()).ddx)
    finally:
        a.close()
        b.close()

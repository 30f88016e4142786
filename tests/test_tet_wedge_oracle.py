"""The checker's SHAPE_21 (10-node tetrahedron) and SHAPE_23 (15-node
wedge): spot values of the reference's tabulated local derivatives
(src/fasolt/Shapef.f90:127-159, 383-432), the patch test (a linear
displacement field's gradient is recovered exactly on a distorted element),
the element volume as the sum of the GP weights, and whole increments on
the generated meshes."""
import ctypes as C

import numpy as np
import pytest

from cpfem_code_b200 import generator

dp = C.POINTER(C.c_double)


def _table(lib, name, ng, nn):
    t = np.zeros(ng * 3 * nn)
    getattr(lib, name)(t.ctypes.data_as(dp))
    return t.reshape(ng, 3, nn)   # [g, j, i] = dndn(j+1, i+1, g+1)


def test_shape21_table_spot_values(oracle_lib):
    t = _table(oracle_lib, "ora_shape21_table", 4, 10)
    # dndn(1, 6, 1), dndn(2, 3, 2), dndn(3, 1, 1), dndn(1, 9, 3) of the reference
    assert t[0, 0, 5] == -2.341641
    assert t[1, 1, 2] == 1.341641
    assert t[0, 2, 0] == 1.341641
    assert t[2, 0, 8] == 1.788854


def test_shape23_table_spot_values(oracle_lib):
    t = _table(oracle_lib, "ora_shape23_table", 6, 15)
    # dndn(1, 5, 1), dndn(3, 7, 1), dndn(2, 3, 1), dndn(3, 10, 4) of the reference
    assert t[0, 0, 4] == 0.596225
    assert t[0, 2, 6] == 0.7698
    assert t[0, 1, 2] == -0.596225
    assert t[3, 2, 9] == 0.496011
    # dndn(1, 2, 2) is one of the entries the reference's tabulation rounds
    # one unit higher (2.103135)
    assert abs(t[1, 0, 1] - 2.103135) <= 1.0000001e-6


def _distorted(nodes):
    rng = np.random.default_rng(0)
    A = np.eye(3) + 0.1 * rng.standard_normal((3, 3))
    p = generator.structured_cube(n=(1, 1, 1), ninc=1, seed=1, nodes=nodes)
    x = p.x.reshape(-1, 3) @ A.T
    return p, x, abs(np.linalg.det(A))


@pytest.mark.parametrize("nodes,lt,ng", [(10, 21, 4), (15, 23, 6)])
def test_patch_and_volume(oracle_lib, nodes, lt, ng):
    p, x, vol = _distorted(nodes)
    rng = np.random.default_rng(1)
    grad = rng.standard_normal((3, 3))
    u = x @ grad.T
    W = 0.0
    for e in range(p.nlmnt):
        ids = p.ln[e, :nodes] - 1
        xe = np.ascontiguousarray(x[ids].reshape(-1))
        for g in range(ng):
            d = np.zeros(3 * nodes)
            w = oracle_lib.ora_shape_elem(lt, g, xe.ctypes.data_as(dp), d.ctypes.data_as(dp))
            assert w > 0
            W += w
            np.testing.assert_allclose(u[ids].T @ d.reshape(nodes, 3), grad, atol=1e-12)
    assert abs(W - vol) < 1e-5 * vol


@pytest.mark.parametrize("nodes", [10, 15])
def test_increment_converges(oracle_lib, nodes):
    from oracle import OracleSolver
    p = generator.structured_cube(n=(2, 2, 2), ninc=1, seed=1, nodes=nodes, xfree=1)
    o = OracleSolver(p, 8, threads=4)
    rep, _ = o.increment(1)
    o.download()
    o.close()
    assert len(rep) < p.ctrl.maxit
    assert p.st[:, 0].mean() > 0

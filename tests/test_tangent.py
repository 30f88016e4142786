"""The consistent tangent (FAS_MODE_TANGENT_CONSISTENT) of the checker
against central finite differences of its own stress update.

On 64 FCC points (the constitutive micro-benchmark's inputs) DSTRSS is run
with the strain increment moved by +-h in each component; the symmetrised
difference quotient d t_i / d de_j is compared with the returned tangent.
With CPSTRS converged tightly (toler 1e-12) the finite differences are the
derivative of the converged local system, which both tangents should equal:
the consistent one by construction (the implicit-function derivative at the
converged stress), CPSTRS's own chi because at convergence its last iterate
is the converged stress.  The device kernels are held to the checker's
tangent in tests/test_gpu_tangent.py.
"""
import numpy as np
import pytest

from cpfem_code_b200 import abi, generator
from cpfem_code_b200.problem import Control

H = 1e-8   # absolute step on strain increments of norm 1e-3


def _run(oracle_solver, p, mode):
    q = p.copy()
    o = oracle_solver(q, 8, mode=mode, threads=4)
    o.constitutive(1, 1)
    o.download()
    T = o.tangent().transpose(0, 2, 1)   # [g, i, j] = chi(i, j)
    o.close()
    return q, T


def _fd(oracle_solver, p):
    fd = np.zeros((p.ngps, 6, 6))
    for j in range(6):
        qp, qm = p.copy(), p.copy()
        qp.de[:, j] += H
        qm.de[:, j] -= H
        a, _ = _run(oracle_solver, qp, abi.FAS_MODE_PLAIN)
        b, _ = _run(oracle_solver, qm, abi.FAS_MODE_PLAIN)
        fd[:, :, j] = (a.ds - b.ds) / (2 * H)
    return 0.5 * (fd + fd.transpose(0, 2, 1))


@pytest.mark.parametrize("mode", [abi.FAS_MODE_TANGENT_CONSISTENT, abi.FAS_MODE_PLAIN])
def test_tangent_against_finite_differences(oracle_lib, mode):
    from oracle import OracleSolver
    p = generator.point_batch(64, seed=5, ctrl=Control(toler=1e-12, maxit=100))
    _, T = _run(OracleSolver, p, mode)
    sym = _fd(OracleSolver, p)
    scale = np.abs(sym).max(axis=(1, 2))
    err = np.abs(T - sym).max(axis=(1, 2)) / scale
    # a point whose active set changes within +-H shows a kink; the bulk
    # of the points matches to the finite differences' own accuracy
    assert np.median(err) < 1e-8
    assert np.quantile(err, 0.9) < 1e-6


def test_consistent_tangent_equals_cpstrs_chi_at_convergence(oracle_lib):
    """At tight convergence the re-evaluation at the converged stress
    changes the tangent only by the size of the last correction."""
    from oracle import OracleSolver
    p = generator.point_batch(64, seed=5, ctrl=Control(toler=1e-12, maxit=100))
    _, Tr = _run(OracleSolver, p, abi.FAS_MODE_PLAIN)
    _, Tc = _run(OracleSolver, p, abi.FAS_MODE_TANGENT_CONSISTENT)
    assert np.abs(Tc - Tr).max() / np.abs(Tr).max() < 1e-8

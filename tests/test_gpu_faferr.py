"""The reference's remaining FAFERR codes raised on the device path by
data-only faults, each against the checker's code on the same input.

* 903, zero SOR diagonal (Stif_sol.f90:183-185): a node that belongs to no
  element and carries no boundary code, so its rows stay empty.
* 904, SOR not converged (Stif_sol.f90:213): a 4^3 cube whose `toler` is
  too tight for 1000 sweeps.
* 910, zero pivot in FACTOR (crys-cons.f90:65-66, the log-slip matrix of
  SLPFTA): a material with rate exponent m = 0 and no hardening, so every
  diagonal entry gam*ah(i,i) + m of the active-set matrix is exactly zero.
* 987, slip Newton failed (crys-cons.f90:108): maxit = 1 (the global
  iteration cap also caps SLPFTA's loop, crys-cons.f90:105) with strain
  increments of Frobenius norm 0.05.

905, 906 and 920 are covered in test_gpu_parity.py.  tests/test_faferr.py
checks the same inputs against the checker alone on the CPU.
"""
import numpy as np
import pytest

from cpfem_code_b200 import GpuSolver, abi, generator
from oracle import OracleSolver

import faferr_cases

pytestmark = pytest.mark.gpu


def _code(run):
    with pytest.raises(abi.FasError) as ei:
        run()
    return ei.value.code


@pytest.mark.parametrize("case", sorted(faferr_cases.CASES))
def test_faferr_code_matches_checker(case):
    make, call, code = faferr_cases.CASES[case]
    p = make()
    pg, po = p.copy(), p.copy()
    g, o = GpuSolver(pg), OracleSolver(po, 8, threads=4)
    got = (_code(lambda: call(g)), _code(lambda: call(o)))
    assert got == (code, code), got
    if case in ("904",):
        # the same Newton iteration raised it: the state before the failing
        # FACSLS (x, dx of the finished iterations) agrees
        g.download()
        o.download()
        s = np.abs(po.x).max()
        assert np.abs(pg.x - po.x).max() <= 1e-10 * s
    g.close()
    o.close()

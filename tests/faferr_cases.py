"""Data-only inputs that make the reference raise its FAFERR codes 903, 904,
910 and 987 (no fault is injected into any code; each input is one the
reference's own checks reject).  Shared by tests/test_faferr.py (checker,
CPU) and tests/test_gpu_faferr.py (device path against the checker)."""
import numpy as np

from cpfem_code_b200 import generator
from cpfem_code_b200.problem import Control


def orphan_node_cube():
    """2^3 cube plus one node that no element uses and no boundary code
    holds: its three rows of the stiffness stay empty (diagonal 0)."""
    p = generator.structured_cube(n=(2, 2, 2), ninc=1, seed=1, xfree=1)
    p.nnod += 1
    xyz = p.x.reshape(-1, 3)
    p.x = np.concatenate([p.x, xyz.max(axis=0) + 1.0])
    for name in ("dx", "fc", "ddx"):
        setattr(p, name, np.concatenate([getattr(p, name), np.zeros(3)]))
    p.ib = np.concatenate([p.ib, np.zeros(1, p.ib.dtype)])
    return p


def tight_toler_cube():
    """4^3 cube in uniaxial tension with toler = 1e-4: 1000 SOR sweeps do
    not bring the relative change below toler^2."""
    return generator.structured_cube(n=(4, 4, 4), ninc=1, seed=2, xfree=3, ctrl=Control(toler=1e-4))


def rate_free_points():
    """FCC points whose material has m = 0 and no hardening (h0 = 0,
    A3 = 0): SLPFTA's matrix gam*ah + diag(m) is exactly zero."""
    m = dict(generator.fcc_aluminium())
    am = m["ampar"].copy()
    am[:, 0] = 0.0
    am[:, 1] = 0.0
    am[:, 2] = 0.0
    m["ampar"] = am
    return generator.point_batch(64, seed=3, material=m)


def one_iteration_points():
    """FCC points with maxit = 1 and strain increments of norm 0.05: one
    SLPFTA iteration leaves tauerr above 0.5."""
    return generator.point_batch(64, seed=3, ctrl=Control(maxit=1), strain_norm=0.05)


# code: (input, call on a solver, expected FAFERR code)
CASES = {
    "903": (orphan_node_cube, lambda s: s.increment(1), 903),
    "904": (tight_toler_cube, lambda s: s.increment(1), 904),
    "910": (rate_free_points, lambda s: s.constitutive(1, 1), 910),
    "987": (one_iteration_points, lambda s: s.constitutive(1, 1), 987),
}

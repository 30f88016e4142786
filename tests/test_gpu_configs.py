"""The device path on the small named configurations, against the checker's
recorded results (tests/golden/, written by tests/golden/make_golden.py).

* ``cube8``: the 8^3 FCC cube, one grain per element, 10 increments to 1 %.
* ``cube16``: the 16^3 FCC cube, 20 increments to 2 % (the natural-order
  record covers its first 4 increments, whose Newton loops converge).

Against the checker in the device's multicolour SOR order the device path
must take the same Newton iterations and SOR sweeps and agree to 1e-10 in
every GP's stress, slip resistances and accumulated slip, in the nodal
coordinates and in the macroscopic stress-strain curve (mean s11 after
every increment).

Against the checker in the reference's natural DOF order
(Stif_sol.f90:189-197) the two SOR orders stop at different iterates, so
the results differ by what the stopping test lets through.  The bound is
the solver tolerance `toler` (1e-3 in these workloads): the macroscopic
curve within toler on both cubes, and every GP's stress within toler of the
largest stress on the 16^3 cube, whose increments converge.  The 8^3 cube
stagnates at maxit = 100 Newton iterations in 9 of its 10 increments (the
reference's SOR stops too early for NRITER to converge, in either order),
so its per-GP difference is not bounded by toler and is only reported.
"""
import os
import sys

import numpy as np
import pytest

from cpfem_code_b200 import GpuSolver, generator

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402

pytestmark = pytest.mark.gpu


def rel(a, b):
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / s) if s > 0 else float(np.abs(a - b).max())


def run_device(name: str, ninc: int, snap: int):
    """`ninc` increments on the device; the state after increment `snap`
    is kept too."""
    p = generator.workload(name)
    assert make_golden.inputs_sha(p) == make_golden.load(name, False)["inputs_sha"]
    g = GpuSolver(p)
    nits, sweeps, macro, at_snap = [], [], [], None
    for inc in range(1, ninc + 1):
        rep, _ = g.increment(inc)
        g.download()
        nits.append(len(rep))
        sweeps.extend(r["sor_sweeps"] for r in rep)
        macro.append(p.st[:, 0].mean())
        if inc == snap:
            at_snap = p.copy()
    g.close()
    return p, np.array(nits), np.array(sweeps), np.array(macro), at_snap


@pytest.fixture(scope="module", params=["cube8", "cube16"])
def device_run(request):
    name = request.param
    ninc, nnat = make_golden.CASES[name]
    return name, run_device(name, ninc, nnat)


def test_matches_checker_in_colour_order(device_run):
    name, (p, nits, sweeps, macro, _) = device_run
    gold = make_golden.load(name, False)
    np.testing.assert_array_equal(nits, gold["newton_iters"])
    np.testing.assert_array_equal(sweeps, gold["sor_sweeps"])
    ns = gold["crss"].shape[1]
    assert rel(p.st, gold["st"]) < 1e-10
    assert rel(p.sv[:, 3:3 + ns], gold["crss"]) < 1e-10
    assert rel(p.cumslip[:, :ns], gold["cumslip"]) < 1e-10
    assert rel(p.x, gold["x"]) < 1e-10
    assert np.abs(macro - gold["macro_s11"]).max() <= 1e-10 * np.abs(gold["macro_s11"]).max()


def test_ordering_difference_within_toler(device_run):
    """Multicolour (device) against natural order (reference): the
    difference is held under the solver tolerance."""
    name, (_, nits, sweeps, macro, p) = device_run
    nat = make_golden.load(name, True)
    k = int(nat["ninc"])
    nits, macro = nits[:k], macro[:k]
    toler = p.ctrl.toler
    d_macro = float(np.abs(macro - nat["macro_s11"]).max() / np.abs(nat["macro_s11"]).max())
    d_point = rel(p.st, nat["st"])
    ns = nat["crss"].shape[1]
    d_crss = rel(p.sv[:, 3:3 + ns], nat["crss"])
    print(f"{name}: colour vs natural SOR order: macro s11 {d_macro:.2e}, per-GP stress {d_point:.2e}, "
          f"slip resistance {d_crss:.2e} (toler {toler:g}); Newton iterations "
          f"{nits.tolist()} vs {nat['newton_iters'].tolist()}")
    assert d_macro < toler
    if name == "cube16":
        assert d_point < toler
        assert d_crss < toler

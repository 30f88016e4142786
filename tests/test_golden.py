"""The golden increment fixtures (tests/golden/) are the checker's own
results on the generator's problems: the generator still makes the same
inputs, and the checker reproduces the first increment of the 8^3 fixtures
in both SOR orders (the device tests compare against the fixtures without
re-running the checker)."""
import os
import sys

import numpy as np
import pytest

from cpfem_code_b200 import abi, generator

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402


@pytest.mark.parametrize("name", list(make_golden.CASES))
def test_generator_reproduces_fixture_inputs(name):
    p = generator.workload(name)
    sha = make_golden.inputs_sha(p)
    for natural in (False, True):
        assert make_golden.load(name, natural)["inputs_sha"] == sha


@pytest.mark.parametrize("natural", [False, True])
def test_checker_reproduces_first_increment(oracle_lib, natural):
    from oracle import OracleSolver
    gold = make_golden.load("cube8", natural)
    p = generator.workload("cube8")
    o = OracleSolver(p, 8, mode=abi.FAS_MODE_SOR_NATURAL if natural else abi.FAS_MODE_PLAIN, threads=4)
    rep, _ = o.increment(1)
    o.download()
    o.close()
    n = int(gold["newton_iters"][0])
    assert len(rep) == n
    assert [r["sor_sweeps"] for r in rep] == gold["sor_sweeps"][:n].tolist()
    np.testing.assert_allclose(p.st[:, 0].mean(), gold["macro_s11"][0], rtol=1e-13)


def test_fixture_shapes():
    for name in make_golden.CASES:
        for natural in (False, True):
            g = make_golden.load(name, natural)
            p = generator.workload(name)
            assert int(g["ninc"]) == make_golden.CASES[name][1 if natural else 0]
            assert g["newton_iters"].shape == (g["ninc"],)
            assert g["sor_sweeps"].shape == (int(g["newton_iters"].sum()),)
            assert g["st"].shape == (p.ngps, 6)
            assert bool(g["natural"]) == natural

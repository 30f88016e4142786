"""Adjoint of the constitutive update: the replay of Gauss-point strain
histories (fas_gpu_adjoint_forward) and its gradients (fas_gpu_adjoint_grad).

The replay is DSTRSS per increment from the elastic predictor, then
UPDATE_GPTV's commit.  The checker's restatement of it is pinned here (CPU)
against the checker's own DSTRSS and commit calls.  The device replay must
equal the checker's (1e-10 relative, as the other constitutive parity
tests).  The gradients have no reference counterpart: they are checked
against central finite differences of the device replay itself, at a
local tolerance of 1e-11 so that the replay is a smooth function of its
inputs.  The bar is 2e-5 of the largest entry of each gradient block.
"""
import numpy as np
import pytest

from cpfem_code_b200 import GpuSolver, ReplayHistory, abi, generator
from oracle import OracleSolver

TOL_FD = 2e-5


def history(p, ninc, seed, chk=2, q=(0.3, 0.5, 0.8)):
    """Strain increments around each point's direction, small spins, equal
    time steps; weights and targets that make J of order one."""
    rng = np.random.default_rng(seed)
    base = p.de.copy()
    de = np.stack([base * (1.0 + 0.2 * rng.standard_normal(base.shape)) for _ in range(ninc)])
    dr = 2e-4 * rng.standard_normal((ninc, p.ngps, 3))
    dt = np.full(ninc, p.tiem[0])
    w = 1e6 * (0.5 + rng.random(p.ngps))
    y = 1e-3 * rng.standard_normal(p.ngps)
    return ReplayHistory(de, dr, dt, w, y, q=q, chk_every=chk)


def points(n, seed, material=None, tau0=25.0):
    p = generator.point_batch(n, seed=seed, material=material, tau0=tau0)
    p.ctrl.toler = 1e-11
    return p


def qq(q):
    q = np.asarray(q, float) / np.linalg.norm(q)
    return np.array([q[0] ** 2, q[1] ** 2, q[2] ** 2, q[1] * q[2], q[2] * q[0], q[0] * q[1]])


# ------------------------------------------------------------------ CPU
def test_checker_replay_is_dstrss_then_commit():
    """The checker's replay equals stepping its DSTRSS (constitutive pass)
    and UPDATE_GPTV with the elastic predictor and dsv = 0 each increment."""
    p = points(6, seed=2)
    h = history(p, 3, seed=4)
    J, eq = OracleSolver(p.copy(), 8).adjoint_forward(h)
    q = p.copy()
    s = OracleSolver(q, 8)
    for n in range(h.ninc):
        q.de[:] = h.de[n]
        q.dr[:] = h.dr[n]
        q.dsv[:] = 0.0
        q.ds[:] = generator.elastic_predictor(q.e[0], q.sv[:, :3], q.de)
        s.upload(q)
        s.constitutive(1, 1)
        s.update_gptv()
        s.download(q)
    eq2 = s.lattice_strain() @ qq(h.q)
    np.testing.assert_allclose(eq, eq2, rtol=0, atol=1e-8 * np.abs(eq2).max())
    J2 = 0.5 * np.sum(h.w * (eq2 - h.y) ** 2)
    assert abs(J - J2) <= 1e-7 * J2


def test_checker_replay_rejects_bad_descriptors():
    p = points(2, seed=1)
    o = OracleSolver(p, 8)
    h = history(p, 2, seed=1)
    h.q = (0.0, 0.0, 0.0)
    with pytest.raises(abi.FasError) as e:
        o.adjoint_forward(h)
    assert e.value.code == abi.FAS_E_ARG


def test_history_shapes_are_checked():
    p = points(2, seed=1)
    with pytest.raises(ValueError):
        ReplayHistory(np.zeros((2, 2, 5)), np.zeros((2, 2, 3)), np.ones(2), np.ones(2), np.zeros(2))


# ------------------------------------------------------------------ GPU
@pytest.mark.gpu
@pytest.mark.parametrize("material,n,ninc", [(None, 64, 6), ("hcp", 32, 4)])
def test_replay_matches_checker(material, n, ninc):
    mat = generator.hcp_zirconium() if material == "hcp" else None
    p = points(n, seed=5, material=mat, tau0=30.0)
    h = history(p, ninc, seed=6)
    g = GpuSolver(p.copy())
    try:
        J, eq = g.adjoint_forward(h)
        before = g.download(p.copy())
    finally:
        g.close()
    Jo, eqo = OracleSolver(p.copy(), 8).adjoint_forward(h)
    assert abs(J - Jo) <= 1e-10 * Jo
    np.testing.assert_allclose(eq, eqo, rtol=0, atol=1e-10 * np.abs(eqo).max())
    # the handle's own state is untouched by a replay
    np.testing.assert_array_equal(before.sv, p.sv)
    np.testing.assert_array_equal(before.st, p.st)


def _fd(g, p, h, field, idx, step):
    vals = []
    for sgn in (1.0, -1.0):
        q = p.copy()
        getattr(q, field)[idx] += sgn * step
        g.upload(q)
        vals.append(g.adjoint_forward(h)[0])
    g.upload(p)
    return (vals[0] - vals[1]) / (2.0 * step)


def _close(ad, fd):
    ad, fd = np.asarray(ad), np.asarray(fd)
    scale = np.abs(fd).max()
    assert scale > 0
    assert np.abs(ad - fd).max() <= TOL_FD * scale, (ad, fd)


@pytest.mark.gpu
def test_gradients_match_finite_differences():
    """Euler angles, slip resistances, starting stress and the hardening
    parameters, over 5 increments with checkpoints every 3 (two segments)."""
    p = points(5, seed=7)
    p.st[:] = 5.0 * np.random.default_rng(3).standard_normal(p.st.shape)
    h = history(p, 5, seed=8, chk=3)
    g = GpuSolver(p.copy())
    try:
        out = g.adjoint_grad(h)
        J, _ = g.adjoint_forward(h)
        assert abs(out["J"] - J) <= 1e-13 * J
        ns = int(p.nss[0])
        ad_e, fd_e, ad_c, fd_c, ad_s, fd_s = [], [], [], [], [], []
        for i in range(p.ngps):
            for k in range(3):
                ad_e.append(out["sv"][i, k])
                fd_e.append(_fd(g, p, h, "sv", (i, k), 1e-6))
            for k in range(ns):
                ad_c.append(out["sv"][i, 3 + k])
                fd_c.append(_fd(g, p, h, "sv", (i, 3 + k), 1e-3))
            for k in range(6):
                ad_s.append(out["st"][i, k])
                fd_s.append(_fd(g, p, h, "st", (i, k), 1e-3))
        _close(ad_e, fd_e)
        _close(ad_c, fd_c)
        _close(ad_s, fd_s)
        assert np.all(out["sv"][:, 3 + ns:] == 0.0)
    finally:
        g.close()
    # hardening parameters: a uniform shift of ampar(k) over the systems
    steps = {0: 1e-6, 1: 1e-3, 2: 1e-3, 4: 1e-3}
    ad_p, fd_p = [], []
    for k, step in steps.items():
        vals = []
        for sgn in (1.0, -1.0):
            q = p.copy()
            q.ampar[0, :ns, k] += sgn * step
            gq = GpuSolver(q)
            try:
                vals.append(gq.adjoint_forward(h)[0])
            finally:
                gq.close()
        ad_p.append(out["ampar"][0, k])
        fd_p.append((vals[0] - vals[1]) / (2.0 * step))
    for a, f in zip(ad_p, fd_p):
        assert abs(a - f) <= TOL_FD * max(abs(f), 1e-30) + 1e-9, (ad_p, fd_p)
    assert np.all(out["ampar"][0, [3, 5, 6, 7, 8, 9]] == 0.0)


@pytest.mark.gpu
def test_hcp_gradients_match_finite_differences():
    """30 slip systems (the 32-system kernels), twins inactive."""
    p = points(3, seed=9, material=generator.hcp_zirconium(), tau0=30.0)
    h = history(p, 3, seed=10, chk=2)
    g = GpuSolver(p.copy())
    try:
        out = g.adjoint_grad(h)
        ad, fd = [], []
        for i in range(p.ngps):
            for k in (0, 1, 2, 3, 7, 20):
                ad.append(out["sv"][i, k])
                fd.append(_fd(g, p, h, "sv", (i, k), 1e-6 if k < 3 else 1e-3))
        _close(ad, fd)
    finally:
        g.close()


@pytest.mark.gpu
def test_checkpoint_interval_does_not_change_gradients():
    """The reverse sweep recomputes each segment with the forward sweep's
    code, so every checkpoint interval gives the same bits."""
    p = points(16, seed=11)
    outs = []
    g = GpuSolver(p.copy())
    try:
        for chk in (1, 2, 5, 9):
            outs.append(g.adjoint_grad(history(p, 5, seed=12, chk=chk)))
    finally:
        g.close()
    for o in outs[1:]:
        assert o["J"] == outs[0]["J"]
        for key in ("st", "sv", "ampar"):
            np.testing.assert_array_equal(o[key], outs[0][key])


@pytest.mark.gpu
def test_autograd_function_gradcheck():
    """The torch wrapper of the calibration harness against torch's own
    finite differences."""
    import torch
    from cpfem_code_b200.calibration import LatticeStrainObjective
    p = points(2, seed=13)
    h = history(p, 3, seed=14, chk=2)
    ns = int(p.nss[0])
    g = GpuSolver(p.copy())
    try:
        euler = torch.tensor(p.sv[:, 0:3], dtype=torch.float64, requires_grad=True)
        crss = torch.tensor(p.sv[:, 3:3 + ns], dtype=torch.float64, requires_grad=True)
        f = lambda e, c: LatticeStrainObjective.apply(e, c, g, h)  # noqa: E731
        assert torch.autograd.gradcheck(f, (euler, crss), eps=1e-6, atol=1e-6, rtol=1e-4)
    finally:
        g.close()


@pytest.mark.gpu
def test_adjoint_rejects_too_many_systems():
    """Materials of more than 32 systems are outside the adjoint's kernels."""
    m = generator.fcc_aluminium()
    big = dict(m)
    reps = 3   # 36 systems: the FCC set three times
    big.update(ns=12 * reps, ab=np.tile(m["ab"], (reps, 1)), an=np.tile(m["an"], (reps, 1)),
               ampar=np.tile(m["ampar"], (reps, 1)), ssang=np.zeros(12 * reps),
               smatrx=np.ones((12 * reps, 12 * reps)))
    p = points(2, seed=15, material=big)
    g = GpuSolver(p)
    try:
        with pytest.raises(abi.FasError) as e:
            g.adjoint_forward(history(p, 2, seed=1))
        assert e.value.code == abi.FAS_E_RANGE
    finally:
        g.close()

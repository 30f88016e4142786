"""Known-answer tests that pin the CPU checker to physics and to the
reference's formulas.  The reference ships no tests or golden outputs
(parity is unpinned by the reference itself), so these KATs are what ties the
restatement down: each checks one routine against an independent derivation.
"""
import ctypes as C
import math

import numpy as np
import pytest

from cpfem_code_b200 import generator

D = C.POINTER(C.c_double)


def dp(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(D)


def test_spower_clamps(oracle_lib):
    L = oracle_lib
    # SPOWER (crys-cons.f90:210-230): sign(a)|a|^b, zero below 1e-35,
    # exponent argument clamped to +-80
    assert L.ora_spower(0.0, 3.0) == 0.0
    assert L.ora_spower(1e-36, 0.5) == 0.0
    assert L.ora_spower(2.0, 3.0) == pytest.approx(8.0, rel=1e-14)
    assert L.ora_spower(-2.0, 3.0) == pytest.approx(-8.0, rel=1e-14)
    assert L.ora_spower(10.0, 100.0) == pytest.approx(math.exp(80.0), rel=1e-14)
    assert L.ora_spower(10.0, -100.0) == pytest.approx(math.exp(-80.0), rel=1e-14)


def test_fj2vom_measures(oracle_lib):
    L = oracle_lib
    # strain measure: isochoric uniaxial strain e -> e
    e = 1e-3
    v = np.array([e, -e / 2, -e / 2, 0, 0, 0])
    assert L.ora_fj2vom(0, dp(v)) == pytest.approx(e, rel=1e-14)
    # stress measure is (2/3) of von Mises: uniaxial s -> 2s/3, shear t -> 2t/sqrt(3)
    s = np.array([3.0, 0, 0, 0, 0, 0])
    assert L.ora_fj2vom(1, dp(s)) == pytest.approx(2.0, rel=1e-14)
    t = np.array([0, 0, 0, 1.0, 0, 0])
    assert L.ora_fj2vom(1, dp(t)) == pytest.approx(2.0 / math.sqrt(3.0), rel=1e-14)


def test_lu_against_numpy(oracle_lib):
    rng = np.random.default_rng(0)
    for n in (1, 2, 6, 12, 30):
        a = rng.standard_normal((n, n)) + n * np.eye(n)
        b = rng.standard_normal(n)
        x = b.copy()
        rc = oracle_lib.ora_factor_solve(n, dp(a.T.copy()), x.ctypes.data_as(D))
        assert rc == 0
        np.testing.assert_allclose(x, np.linalg.solve(a, b), rtol=1e-12, atol=1e-12)
    # zero pivot -> 910 (FACTOR's ifail, crys-cons.f90:257)
    a = np.array([[0.0, 1.0], [1.0, 0.0]])
    x = np.ones(2)
    assert oracle_lib.ora_factor_solve(2, dp(a.T.copy()), x.ctypes.data_as(D)) == 910


def _bunge(ph1, phi, ph2):
    """Independent Bunge (z-x-z) sample->crystal matrix g = Z(ph2) X(phi) Z(ph1)."""
    def rz(t):
        c, s = math.cos(t), math.sin(t)
        return np.array([[c, s, 0], [-s, c, 0], [0, 0, 1.0]])

    def rx(t):
        c, s = math.cos(t), math.sin(t)
        return np.array([[1.0, 0, 0], [0, c, s], [0, -s, c]])
    return rz(ph2) @ rx(phi) @ rz(ph1)


def test_ctmatrx_is_bunge_matrix(oracle_lib):
    rng = np.random.default_rng(1)
    for _ in range(20):
        e = rng.random(3) * np.array([2 * math.pi, math.pi, 2 * math.pi])
        a = np.zeros(9)
        aug = np.zeros(3)
        oracle_lib.ora_ctmatrx(*e, a.ctypes.data_as(D), aug.ctypes.data_as(D))
        A = a.reshape(3, 3, order="F")
        np.testing.assert_allclose(A, _bunge(*e), atol=1e-14)
        np.testing.assert_allclose(A @ A.T, np.eye(3), atol=1e-14)
        np.testing.assert_allclose(aug, [math.sin(e[2]), math.cos(e[2]), math.sin(e[1])])


def _compliance_tensor_rotated(e9, g):
    """Full 4th-order rotation of the cubic/hexagonal compliance."""
    s11, s22, s33, s23, s31, s12, s44, s55, s66 = e9
    S = np.zeros((3, 3, 3, 3))
    S[0, 0, 0, 0], S[1, 1, 1, 1], S[2, 2, 2, 2] = s11, s22, s33
    for (i, j, v) in ((1, 2, s23), (2, 0, s31), (0, 1, s12)):
        S[i, i, j, j] = S[j, j, i, i] = v
    for (i, j, v) in ((1, 2, s44), (2, 0, s55), (0, 1, s66)):
        for (a, b) in ((i, j), (j, i)):
            for (c, d) in ((i, j), (j, i)):
                S[a, b, c, d] = v / 4.0
    R = g.T   # crystal -> sample
    Sr = np.einsum("ia,jb,kc,ld,abcd->ijkl", R, R, R, R, S)
    idx = [(0, 0), (1, 1), (2, 2), (1, 2), (2, 0), (0, 1)]
    M = np.zeros((6, 6))
    for I, (i, j) in enumerate(idx):
        for J, (k, l) in enumerate(idx):
            M[I, J] = Sr[i, j, k, l] * (2 if I >= 3 else 1) * (2 if J >= 3 else 1)
    return M


def test_elastc_against_tensor_rotation(oracle_lib):
    """ELASTC (ela-plas.f90:34-76) is the exact rotated compliance in its
    normal 3x3 block, but because `mult` depends on the row only and term3
    keeps two of the four shear products, every normal-shear entry and every
    off-diagonal shear-shear entry of a cubic crystal is exactly half the
    tensor value; the shear block is exact only for isotropic crystals.  The checker keeps
    this behaviour of the reference; these assertions pin it."""
    e9 = generator.cubic_compliance(108.2e3, 61.3e3, 28.5e3)
    hcp = np.array([10.2e-6, 10.2e-6, 8.01e-6, -2.46e-6, -2.46e-6, -4.09e-6, 29.94e-6, 29.94e-6, 28.58e-6])
    iso = np.array([1e-5, 1e-5, 1e-5, -3e-6, -3e-6, -3e-6, 2.6e-5, 2.6e-5, 2.6e-5])
    rng = np.random.default_rng(2)
    off = ~np.eye(3, dtype=bool)
    for e in (e9, hcp, iso):
        # crystal frame: the engineering compliance itself
        out = np.zeros(36)
        oracle_lib.ora_elastc(dp(e), dp(np.zeros(3)), out.ctypes.data_as(D))
        np.testing.assert_allclose(out.reshape(6, 6, order="F"),
                                   _compliance_tensor_rotated(e, np.eye(3)), rtol=1e-14, atol=1e-22)
        for _ in range(10):
            eu = rng.random(3) * np.array([2 * math.pi, math.pi, 2 * math.pi])
            oracle_lib.ora_elastc(dp(e), dp(eu), out.ctypes.data_as(D))
            M = out.reshape(6, 6, order="F")
            T = _compliance_tensor_rotated(e, _bunge(*eu))
            tol = dict(rtol=1e-11, atol=1e-18)
            np.testing.assert_allclose(M[:3, :3], T[:3, :3], **tol)
            np.testing.assert_allclose(M[:3, 3:], T[:3, 3:] / 2, **tol)
            np.testing.assert_allclose(M[3:, :3], T[3:, :3] / 2, **tol)
            if e is e9:
                np.testing.assert_allclose(M[3:, 3:][off], T[3:, 3:][off] / 2, **tol)
            np.testing.assert_allclose(M, M.T, rtol=1e-15, atol=0)
            if e is iso:
                np.testing.assert_allclose(M[3:, 3:], T[3:, 3:], **tol)
    # vectorised generator restatement agrees with the checker
    eu = rng.random((5, 3))
    S = generator.rotated_compliance(e9, eu)
    for k in range(5):
        out = np.zeros(36)
        oracle_lib.ora_elastc(dp(e9), dp(eu[k]), out.ctypes.data_as(D))
        np.testing.assert_allclose(S[k], out.reshape(6, 6, order="F"), rtol=1e-13)


def test_tens_rot_small_rotation(oracle_lib):
    # TENS_ROT rotates by the first-order rotation R with R_ii = sqrt(1-...)
    a = np.array([100.0, -20.0, 5.0, 3.0, -7.0, 11.0])
    b = np.zeros(6)
    oracle_lib.ora_tens_rot(dp(np.zeros(3)), dp(a), b.ctypes.data_as(D))
    np.testing.assert_allclose(b, a, rtol=1e-15)
    r = np.array([1e-3, -2e-3, 5e-4])
    oracle_lib.ora_tens_rot(dp(r), dp(a), b.ctypes.data_as(D))
    R = np.array([[math.sqrt(1 - r[1] ** 2 - r[2] ** 2), r[2], -r[1]],
                  [-r[2], math.sqrt(1 - r[0] ** 2 - r[2] ** 2), r[0]],
                  [r[1], -r[0], math.sqrt(1 - r[0] ** 2 - r[1] ** 2)]])
    T = np.array([[a[0], a[5], a[4]], [a[5], a[1], a[3]], [a[4], a[3], a[2]]])
    N = R.T @ T @ R
    np.testing.assert_allclose(b, [N[0, 0], N[1, 1], N[2, 2], N[1, 2], N[2, 0], N[0, 1]], rtol=1e-13)


def test_shape12_patch(oracle_lib):
    # SHAPE_12: a linear displacement field gives its exact gradient, the
    # weight is the element volume, shape derivatives sum to zero
    rng = np.random.default_rng(3)
    xi = generator.BRICK8.astype(float)
    F = np.eye(3) + 0.2 * rng.standard_normal((3, 3))
    x = (xi - 0.5) @ F.T * 0.7 + 1.3
    dn = np.zeros(24)
    w = oracle_lib.ora_shape12(dp(x.reshape(-1)), dn.ctypes.data_as(D))
    dndx = dn.reshape(8, 3)
    assert w == pytest.approx(abs(np.linalg.det(F)) * 0.7 ** 3, rel=1e-13)
    np.testing.assert_allclose(dndx.sum(axis=0), 0.0, atol=1e-13)
    G = rng.standard_normal((3, 3))
    u = x @ G.T
    grad = dndx.T @ u           # grad[a, b] = d u_b / d x_a
    np.testing.assert_allclose(grad, G.T, rtol=1e-12, atol=1e-13)


def test_shape22_table(oracle_lib):
    # SHAPE_22's tabulated local derivatives: serendipity functions at the
    # GP coordinate 0.57735, rounded to 6 decimals.  Spot values of the
    # reference table (Shapef.f90:259-264): dndn(1,1,1), dndn(1,2,1),
    # dndn(2,1,1), dndn(3,9,1).
    t = np.zeros(480)
    oracle_lib.ora_shape22_table(t.ctypes.data_as(D))
    dn = t.reshape(8, 3, 20)                       # [gp][local coord][node]
    assert dn[0, 0, 0] == -0.407229
    assert dn[0, 0, 1] == 0.718233
    assert dn[0, 1, 0] == -0.407229
    assert dn[0, 2, 8] == 0.718233
    # every table entry has 6 decimals; each GP's derivatives sum to ~0
    np.testing.assert_allclose(np.round(t * 1e6), t * 1e6, atol=1e-6)
    np.testing.assert_allclose(dn.sum(axis=2), 0.0, atol=5e-6)


@pytest.mark.parametrize("g", range(8))
def test_shape22_patch(oracle_lib, g):
    # SHAPE_22 on an affinely distorted 20-node brick: a linear displacement
    # field gives its gradient and the eight weights add up to the volume,
    # to the 6-decimal precision of the tabulated derivatives
    rng = np.random.default_rng(5)
    xi = generator.BRICK20_HALF.astype(float) / 2.0
    F = np.eye(3) + 0.2 * rng.standard_normal((3, 3))
    x = (xi - 0.5) @ F.T * 0.7 + 1.3
    dn = np.zeros(60)
    w = oracle_lib.ora_shape22(g, dp(x.reshape(-1)), dn.ctypes.data_as(D))
    dndx = dn.reshape(20, 3)
    assert w == pytest.approx(abs(np.linalg.det(F)) * 0.7 ** 3 / 8.0, rel=2e-5)
    G = rng.standard_normal((3, 3))
    grad = dndx.T @ (x @ G.T)
    np.testing.assert_allclose(grad, G.T, rtol=0, atol=2e-5 * np.abs(G).max())


def _point_problem(n, toler=1e-3, iel=1, seed=4, h0=150.0):
    from cpfem_code_b200.problem import Control
    mat = generator.fcc_aluminium(h0=h0)
    p = generator.point_batch(n, seed=seed, material=mat, ctrl=Control(toler=toler))
    p.le[:] = iel
    return p, mat


def test_elastic_only_point_is_hooke(oracle_lib):
    """DSTRSS's elastic branch (Sig_eps.f90:130-145): t = S(phi)^-1 de."""
    from oracle import OracleSolver
    p, mat = _point_problem(32, iel=-1)
    st0 = p.st.copy()
    o = OracleSolver(p, 8)
    o.constitutive(1, 1)
    o.download()
    S = generator.rotated_compliance(mat["e"], p.sv[:, :3])
    t = np.linalg.solve(S, p.de[:, :, None])[:, :, 0]
    np.testing.assert_allclose(p.ds, t - st0, rtol=1e-12, atol=1e-9)
    chi = o.tangent()
    np.testing.assert_allclose(chi.transpose(0, 2, 1), np.linalg.inv(S), rtol=1e-10)
    assert (p.dep == 0).all()


def _schmid(mat, euler):
    a = np.stack([_bunge(*e) for e in euler])            # sample -> crystal
    d = np.einsum("nlj,sl->nsj", a, mat["ab"])            # slip direction, sample
    nrm = np.einsum("nlj,sl->nsj", a, mat["an"])
    b = np.stack([d[..., 0] * nrm[..., 0], d[..., 1] * nrm[..., 1], d[..., 2] * nrm[..., 2],
                  d[..., 1] * nrm[..., 2] + d[..., 2] * nrm[..., 1],
                  d[..., 2] * nrm[..., 0] + d[..., 0] * nrm[..., 2],
                  d[..., 0] * nrm[..., 1] + d[..., 1] * nrm[..., 0]], axis=-1)
    return b                                               # [n, ns, 6]


def test_converged_point_satisfies_crystal_plasticity(oracle_lib):
    """With a tight tolerance the CPSTRS fixed point must satisfy, checked
    independently in numpy: the additive split de = b.gamma + S (s - t)
    (Cpstrs.f90:96-98), the power-law flow rule gamma = dt (tau/s1)^(1/m) on
    every slipping system (crys-cons.f90:71), and PLASTC's Voce hardening
    s1 = s0 + sum_j smatrx_ij theta_j |gamma_j| (ela-plas.f90:155-183)."""
    from oracle import OracleSolver
    p, mat = _point_problem(24, toler=1e-10)
    s0 = p.sv[:, 3:15].copy()
    de = p.de.copy()
    o = OracleSolver(p, 8)
    o.constitutive(1, 1)
    o.download()
    it, err = o.cp_stats()
    assert (it > 0).all() and (err <= 1e-10).all()
    dt = p.tiem[0]
    m = mat["ampar"][0, 0]
    sig = p.ds                                   # st = 0, so ds is the stress
    # CPSTRS resolves in the frame sv + dsv of its entry (dsv = 0 here)
    b = _schmid(mat, p.sv[:, :3])
    tau = np.einsum("nsk,nk->ns", b, sig)
    rate = p.srate[:, :12]
    gam = np.sign(tau) * rate * dt
    s1 = s0 + p.dsv[:, 3:15]
    act = rate > 1e-6 * rate.max(axis=1, keepdims=True)
    np.testing.assert_allclose(rate[act], (np.abs(tau) / s1)[act] ** (1 / m), rtol=1e-6)
    S = generator.rotated_compliance(mat["e"], p.sv[:, :3])
    resid = de - np.einsum("nsk,ns->nk", b, gam) - np.einsum("nij,nj->ni", S, sig)
    assert np.abs(resid).max() < 1e-9 * np.abs(de).max()
    theta = mat["ampar"][0, 1] * np.clip(1 - s0 / mat["ampar"][0, 4], 0, None)
    np.testing.assert_allclose(
        s1, s0 + np.einsum("ij,nj,nj->ni", mat["smatrx"], theta, np.abs(gam)), rtol=1e-12)


def test_lattice_strain_is_compliance_times_stress(oracle_lib):
    """ELASEPS (data_out.f90:263-361) = the ELASTC compliance at sv(1:3)
    times the stress."""
    from oracle import OracleSolver
    p, mat = _point_problem(16)
    rng = np.random.default_rng(9)
    p.st[:] = rng.standard_normal(p.st.shape) * 50.0
    o = OracleSolver(p, 8)
    e = o.lattice_strain()
    S = generator.rotated_compliance(mat["e"], p.sv[:, :3])
    np.testing.assert_allclose(e, np.einsum("nij,nj->ni", S, p.st), rtol=1e-13, atol=1e-20)


def test_20_node_brick_increment_matches_8_node():
    # One grain, one element, uniaxial tension: the field is close to
    # homogeneous, which both bricks represent, so the 20-node, 8-GP brick
    # (SHAPE_22) and the 8-node, 1-GP brick (SHAPE_12) give nearly the same
    # mean stress; the 20-node Newton loop converges like the 8-node one
    from oracle import OracleSolver
    out = {}
    for nodes in (8, 20):
        p = generator.structured_cube(n=(1, 1, 1), nodes=nodes, ninc=2, seed=3)
        o = OracleSolver(p, 8, threads=2)
        for inc in (1, 2):
            rep, _ = o.increment(inc)
            assert len(rep) < p.ctrl.maxit and rep[-1]["sdx"] < p.ctrl.toler
        o.download()
        out[nodes] = p.st[:, 0].mean()
        assert np.isfinite(p.st).all()
    assert out[20] == pytest.approx(out[8], rel=2e-3)


@pytest.mark.parametrize("nodes,inc_steps", [(8, 1), (20, 1), (8, 3)])
def test_assembled_stiffness_is_symmetric(nodes, inc_steps):
    """The checker's assembled stiffness (ELVALS + SUVALS) is symmetric:
    K_ij = K_ji to rounding on the rows of free DOFs, and exactly where the
    penalty terms sit (they touch diagonal entries only).  This holds in the
    elastic first iteration and after plastic increments (the tangent chi
    is symmetric), and is the property the device's symmetric FP32 rows
    (FAS_MODE_SOR_SYM) rely on when they store each off-diagonal block once."""
    from oracle import OracleSolver
    p = generator.structured_cube(n=(4, 3, 3) if nodes == 8 else (2, 2, 2), ninc=inc_steps, seed=3,
                                  nodes=nodes)
    o = OracleSolver(p, 8, threads=4)
    for inc in range(1, inc_steps):
        o.increment(inc)
    o.update_node()
    o.elvals(inc_steps, 1)
    o.suvals(inc_steps)
    ld = 96 if nodes == 8 else 256       # columns per DOF row: 27 or 81 nodes x 3
    IS, SS = o.pattern(ld), o.stiffness(ld)
    n = 3 * p.nnod
    K = np.zeros((n, n))
    for r in range(n):
        K[r, r] = SS[r, 0]
        for k in range(1, IS[r, 0] + 1):
            K[r, IS[r, k] - 1] = SS[r, k]
    pen = np.diag(K) > 1e15
    assert pen.any() and (~pen).any()
    free = K[np.ix_(~pen, ~pen)]
    assert np.abs(free - free.T).max() <= 1e-14 * np.abs(free).max()
    off = K - np.diag(np.diag(K))
    assert np.abs(off - off.T).max() <= 1e-14 * np.abs(free).max()

"""The structured-brick generator against brute-force restatements of
fs3pre's ADDEL_8NQ + SWEEP, SETBOUNDS and SETKINC."""
import numpy as np
import pytest

from cpfem_code_b200 import generator


def _addel_sweep(nx, ny, nz, dxl, nodes=8):
    """ADDEL_8NQ / ADDEL_20NQ (fs3pre.f90:183-291) then SWEEP
    (fs3p-swp.f90:53-109), literally: append the element's nodes, then remove
    every node that lies within the tolerance of an earlier one, renumbering
    the topology.  The tolerance is SETSWTOL's half of the shortest
    intra-element distance (fs3p-swp.f90:7-45)."""
    local = generator.BRICK8 if nodes == 8 else generator.BRICK20_HALF / 2.0
    xs, ln = [], []
    for iz in range(nz):
        for iy in range(ny):
            for ix in range(nx):
                x0 = np.array([dxl[0] * ix, dxl[1] * iy, dxl[2] * iz])
                el = []
                for off in local:
                    xs.append(x0 + dxl * off)
                    el.append(len(xs))
                ln.append(el)
    x = np.array(xs)
    ln = np.array(ln)
    e0 = x[ln[0] - 1]
    d2 = ((e0[:, None, :] - e0[None, :, :]) ** 2).sum(-1)
    tol = 0.5 * np.sqrt(d2[np.triu_indices(len(local), 1)].min())
    i_test = 1
    while i_test < len(x):
        i_test += 1
        j = 1
        common = False
        while j < i_test - 1 and not common:
            j += 1
            common = np.sqrt(((x[i_test - 1] - x[j - 1]) ** 2).sum()) < tol
        if common:
            x = np.delete(x, i_test - 1, axis=0)
            ln = np.where(ln == i_test, j, ln)
            ln = np.where(ln > i_test, ln - 1, ln)
            i_test -= 1
    return x.reshape(-1), ln


@pytest.mark.parametrize("n", [(1, 1, 1), (2, 2, 2), (2, 1, 3)])
def test_numbering_matches_sweep_20_node(n):
    p = generator.structured_cube(n=n, lengths=(1.0, 2.0, 0.5), ninc=1, nodes=20)
    dxl = np.array([1.0 / n[0], 2.0 / n[1], 0.5 / n[2]])
    x, ln = _addel_sweep(*n, dxl, nodes=20)
    assert p.nnod == len(x) // 3
    np.testing.assert_array_equal(p.ln, ln)
    np.testing.assert_allclose(p.x, x, rtol=0, atol=1e-15)
    assert (p.lt == 22).all() and (p.nd == 20).all() and (p.np_ == 8).all()
    # ADDEL_20NQ's GP numbering: 8 * element - 8 + i
    np.testing.assert_array_equal(p.lg.ravel(), np.arange(1, 8 * p.nlmnt + 1))
    assert p.ngps == 8 * p.nlmnt


@pytest.mark.parametrize("n", [(1, 1, 1), (2, 2, 2), (3, 2, 1), (2, 3, 4)])
def test_numbering_matches_sweep(n):
    p = generator.structured_cube(n=n, lengths=(1.0, 2.0, 0.5), ninc=1)
    dxl = np.array([1.0 / n[0], 2.0 / n[1], 0.5 / n[2]])
    x, ln = _addel_sweep(*n, dxl)
    assert p.nnod == len(x) // 3 == np.prod(np.array(n) + 1)
    np.testing.assert_array_equal(p.ln, ln)
    np.testing.assert_array_equal(p.x, x)
    np.testing.assert_array_equal(p.lg[:, 0], np.arange(1, p.nlmnt + 1))


def test_bounds_xfree3_uniaxial():
    p = generator.structured_cube(n=(2, 2, 2), xfree=3, ninc=1)
    xyz = p.x.reshape(-1, 3)
    lo = np.isclose(xyz[:, 0], 0.0)
    hi = np.isclose(xyz[:, 0], 1.0)
    origin = np.all(np.isclose(xyz, 0.0), axis=1)
    inner = np.all((xyz > 0) & (xyz < 1), axis=1)
    assert (p.ib[origin] == 700).all()            # l_side 21 keeps the 'all fixed' default
    assert (p.ib[lo & ~origin] == 100).all()
    assert (p.ib[hi] == 800).all()
    assert (p.ib[inner] == 0).all()
    assert (p.ib[~lo & ~hi & ~inner] == 1).all()


@pytest.mark.parametrize("xfree", [0, 1, 2])
def test_bounds_other_options(xfree):
    p = generator.structured_cube(n=(2, 2, 2), xfree=xfree, ninc=1)
    xyz = p.x.reshape(-1, 3)
    surf = ~np.all((xyz > 0) & (xyz < 1), axis=1)
    if xfree == 0:
        assert (p.ib[surf] == 5000).all()
    if xfree == 1:
        corner = np.all(np.isclose(xyz, 1.0), axis=1)
        assert (p.ib[corner] == 1400).all()
    if xfree == 2:
        # x faces free, y and z faces specified
        xlo_only = np.isclose(xyz[:, 0], 0) & (xyz[:, 1] > 0) & (xyz[:, 1] < 1) & (xyz[:, 2] > 0) & (xyz[:, 2] < 1)
        assert (p.ib[xlo_only] == 1).all()
    assert (p.ib[~surf] == 0).all()


def test_setkinc_tables():
    tiem, xs = generator.setkinc((1.0, 1.0, 1.0), 3, (1e-3, 5.0, 5.0), 3)
    np.testing.assert_allclose(tiem, 1e-3)
    # x-spec code 8: mask xx, target = e11 * current length, compounding
    L = 1.0
    for i in range(3):
        np.testing.assert_array_equal(xs[i, 7, :6], [1, 0, 0, 0, 0, 0])
        assert xs[i, 7, 6] == pytest.approx(1e-3 * L)
        L += 1e-3 * L
        assert xs[i, 0, 6] == 0.0
        np.testing.assert_array_equal(xs[i, 49, :6], [1, 0, 1, 0, 0, 1])
        assert xs[i, 49, 6] == 1e-3 and xs[i, 49, 10] == 0.0


def test_grains_and_materials():
    a = generator.fcc_aluminium()
    b = dict(a, name="fcc-b")
    p = generator.structured_cube(n=(4, 4, 4), grain=2, materials=[a, b], fractions=[0.5, 0.5], seed=3)
    gid = p.meta["grain_id"]
    assert gid.max() == 7
    for g in range(8):
        sel = gid == g
        assert len(np.unique(p.le[sel])) == 1
        assert np.unique(p.sv[sel, :3], axis=0).shape[0] == 1
    assert set(np.unique(p.le)) <= {1, 2}
    assert (p.sv[:, 3:15] == 25.0).all()


def test_hcp_systems_geometry():
    ab, an, lab = generator.hcp_systems(1.593)
    counts = {k: lab.count(k) for k in set(lab)}
    assert counts == {"basal": 3, "prism": 3, "pyr1ca": 12, "pyr2ca": 6, "twin": 6}
    np.testing.assert_allclose(np.linalg.norm(ab, axis=1), 1.0, rtol=1e-14)
    np.testing.assert_allclose(np.linalg.norm(an, axis=1), 1.0, rtol=1e-14)
    np.testing.assert_allclose((ab * an).sum(axis=1), 0.0, atol=1e-14)
    c = np.array([0.0, 0.0, 1.0])
    lab = np.array(lab)
    # basal normals are c; prism normals and <a> directions lie in the basal plane
    np.testing.assert_allclose(an[lab == "basal"] @ c, 1.0)
    np.testing.assert_allclose(an[lab == "prism"] @ c, 0.0, atol=1e-15)
    # <c+a>: angle to c is atan(1/(c/a)) * ... |b.c| = c/a / sqrt(1 + (c/a)^2)
    ca = 1.593
    np.testing.assert_allclose(np.abs(ab[lab == "pyr1ca"] @ c), ca / np.sqrt(1 + ca ** 2), rtol=1e-12)
    # {10-12} plane normal: tan(angle to c) = 2 / (sqrt(3) c/a) ... cos = l/ca / |n|
    n = np.array([1.0, 1 / np.sqrt(3), 2 / ca])
    np.testing.assert_allclose(an[lab == "twin"] @ c, n[2] / np.linalg.norm(n), rtol=1e-12)
    # the six twin variants are related by 60 degree rotations about c
    ang = np.sort(np.degrees(np.arctan2(an[lab == "twin"][:, 1], an[lab == "twin"][:, 0])) % 360)
    np.testing.assert_allclose(np.diff(ang), 60.0, atol=1e-9)


def test_hcp_material_and_mixed_workload():
    z = generator.hcp_zirconium()
    assert z["ssang"][np.array(z["labels"]) == "twin"] == pytest.approx(85.2, abs=0.05)
    p = generator.mixed_config(n=4, ninc=2)
    assert set(np.unique(p.le)) == {1, 2}
    hcp = p.le == 1
    assert (p.sv[hcp, 3:33] == z["tau0"][None, :]).all()
    assert (p.sv[~hcp, 3:15] == 25.0).all() and (p.sv[~hcp, 15:33] == 0).all()
    assert p.nsv == 33 and p.twinprob == 1.0 and p.twinlim == 1


def _setties_literal(x, ib, tol, tie):
    """SETTIES (fs3p-bkc.f90:316-405) as the reference's nested loops."""
    xyz = x.reshape(-1, 3)
    lo, hi = xyz.min(axis=0), xyz.max(axis=0)
    out = []
    for i1 in range(len(xyz)):
        for j1 in range(3):
            if tie[j1] and abs(xyz[i1, j1] - lo[j1]) < tol:
                j2, j3 = (j1 + 1) % 3, (j1 + 2) % 3
                for i2 in range(len(xyz)):
                    if (abs(xyz[i2, j1] - hi[j1]) < tol and abs(xyz[i1, j2] - xyz[i2, j2]) < tol
                            and abs(xyz[i1, j3] - xyz[i2, j3]) < tol):
                        c = ib[i1] // 100
                        lt = {1: j1 + 4, 2: j1 + 4, 3: j1 + 4, 6: 1, 18: 1, 20: 1,
                              5: 2, 16: 2, 19: 2, 4: 3, 15: 3, 17: 3}.get(c)
                        if lt:
                            out.append((i1 + 1, i2 + 1, lt))
    return out


@pytest.mark.parametrize("nodes,xfree,tie", [(8, 1, (True, True, True)), (8, 3, (False, True, True)),
                                             (20, 1, (True, False, True))])
def test_ties_match_literal_setties(nodes, xfree, tie):
    p = generator.structured_cube(n=(2, 3, 2), ninc=1, xfree=xfree, nodes=nodes, ties=tie)
    nb = 12
    x = p.x
    tol = 0.5 * min(1 / 2, 1 / 3, 1 / 2) / (1 if nodes == 8 else 2)
    ref = _setties_literal(x, p.ib, tol, tie)
    assert p.nlmnt == nb + len(ref) and p.meta["ties"] == len(ref) > 0
    t = np.array(ref)
    np.testing.assert_array_equal(p.ln[nb:, :2], t[:, :2])
    np.testing.assert_array_equal(p.lt[nb:], t[:, 2])
    assert (p.nd[nb:] == 2).all() and (p.np_[nb:] == 0).all() and (p.le[nb:] == 0).all()
    assert (p.ln[nb:, 2:] == 0).all() and (p.lg[nb:] == 0).all()

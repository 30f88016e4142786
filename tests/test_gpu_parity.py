"""Parity of the sm_100a path with the CPU checker on identical inputs.

Every call goes through the C ABI (libfasgpu.so).  Tolerances: the plain
path computes in FP64 like the checker's double restatement, so per-GP
stresses, slips and state agree to 1e-11 relative; integer data (pattern,
colouring, iteration counts, operation counts, twin flags) must be
bit-exact.
"""
import numpy as np
import pytest

from cpfem_code_b200 import GpuSolver, abi, generator
from cpfem_code_b200.problem import Control
from oracle import OracleSolver

pytestmark = pytest.mark.gpu
RTOL = 1e-11


def rel(a, b):
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / s) if s > 0 else float(np.abs(a - b).max())


def pair(p, threads=4, mode=abi.FAS_MODE_PLAIN):
    pg, po = p.copy(), p.copy()
    return GpuSolver(pg, mode=mode), OracleSolver(po, 8, threads=threads), pg, po


@pytest.mark.parametrize("mode", [abi.FAS_MODE_PLAIN, abi.FAS_MODE_CP_WARP, abi.FAS_MODE_CP_QUEUE])
def test_constitutive_points(mode):
    """One thread per point (default) and one warp per point."""
    p = generator.point_batch(2048, seed=11)
    g, o, pg, po = pair(p, mode=mode)
    g.constitutive(1, 1)
    o.constitutive(1, 1)
    g.download()
    o.download()
    assert rel(pg.ds, po.ds) < RTOL
    assert rel(pg.dsv[:, :15], po.dsv[:, :15]) < RTOL
    assert rel(pg.srate[:, :12], po.srate[:, :12]) < RTOL
    assert rel(pg.dep, po.dep) < RTOL
    assert rel(g.tangent(), o.tangent()) < RTOL
    ig, eg = g.cp_stats()
    io, eo = o.cp_stats()
    np.testing.assert_array_equal(ig, io)
    np.testing.assert_array_equal(g.cp_ops(), o.cp_ops())
    assert (ig > 0).all()


def test_constitutive_points_fp32_descriptors():
    """REAL(4) module arrays through the same ABI give the FP64 result of
    the float values."""
    p = generator.point_batch(256, seed=5)
    for name in ("sv", "ds", "de", "st", "dsv", "dr"):
        setattr(p, name, getattr(p, name).astype(np.float32).astype(np.float64))
    g = GpuSolver(p.copy())
    g.constitutive(1, 1)
    ref = g.download().ds.copy()
    q = p.copy()
    g2 = GpuSolver(q, upload=False)
    d = q.state_descriptor()
    keep = {}
    for name in ("x", "dx", "fc", "ddx", "eps", "dep", "st", "ep", "ds", "de", "rt", "dr",
                 "sv", "dsv", "srate", "cumslip"):
        keep[name] = np.ascontiguousarray(getattr(q, name), dtype=np.float32)
        setattr(d, name, abi.ptr(keep[name]))
    d.real_bytes = 4
    import ctypes as C
    abi.check(g2._lib.fas_gpu_upload_state(g2._h, C.byref(d)), "upload")
    g2.constitutive(1, 1)
    out = np.zeros((p.ngps, 6), np.float32)
    d2 = abi.FasState(real_bytes=4, nsv=q.nsv, ld_sv=abi.SVLD, ld_slip=abi.FAS_MAXSS, ds=abi.ptr(out))
    abi.check(g2._lib.fas_gpu_download_state(g2._h, C.byref(d2)), "download")
    np.testing.assert_allclose(out, ref.astype(np.float32), rtol=1e-6)


@pytest.mark.parametrize("n", [(2, 2, 2), (3, 2, 4), (4, 4, 4)])
def test_pattern_and_colouring_bit_exact(n):
    p = generator.structured_cube(n=n, ninc=2, seed=1)
    g, o, _, _ = pair(p)
    np.testing.assert_array_equal(g.pattern(), o.pattern())
    cg, ng = g.colouring()
    co, no = o.colouring()
    np.testing.assert_array_equal(cg, co)
    assert ng == no == 8
    # no two nodes of one element share a colour
    col = cg[p.ln - 1]
    assert all(len(set(r)) == 8 for r in col)


def test_elvals_suvals_facsls():
    p = generator.cube_config(n=4, ninc=4, grain=1, seed=3)
    g, o, pg, po = pair(p)
    for s in (g, o):
        s.update_node()
        s.elvals(1, 1)
    g.download()
    o.download()
    np.testing.assert_array_equal(pg.fc == 0, po.fc == 0)
    assert rel(pg.fc, po.fc) < RTOL
    Kg, Ko = g.stiffness(), o.stiffness()
    assert rel(Kg, Ko) < RTOL
    for s in (g, o):
        s.suvals(1)
    g.download()
    o.download()
    assert rel(pg.ddx, po.ddx) < RTOL
    Kg, Ko = g.stiffness(), o.stiffness()
    pen = Ko > 1e15
    assert rel(Kg[pen], Ko[pen]) < 1e-15
    assert rel(Kg[~pen], Ko[~pen]) < RTOL
    sg, so = g.facsls(), o.facsls()
    assert sg[0] == so[0]
    g.download()
    o.download()
    assert rel(pg.ddx, po.ddx) < 1e-10


@pytest.mark.parametrize("n,ninc,mode", [((2, 2, 2), 3, abi.FAS_MODE_PLAIN),
                                         ((3, 3, 3), 2, abi.FAS_MODE_PLAIN),
                                         ((8, 8, 8), 1, abi.FAS_MODE_PLAIN),
                                         ((3, 3, 3), 1, abi.FAS_MODE_SOR_GRID),
                                         ((8, 8, 8), 1, abi.FAS_MODE_SOR_GRID),
                                         ((4, 4, 4), 2, abi.FAS_MODE_CP_WARP)])
def test_increments_match(n, ninc, mode):
    """Both SOR launch shapes (one CTA, and grid-wide colour launches) give
    the checker's iterates."""
    p = generator.structured_cube(n=n, ninc=ninc, seed=7)
    g, o, pg, po = pair(p, threads=8, mode=mode)
    for inc in range(1, ninc + 1):
        rg, _ = g.increment(inc)
        ro, _ = o.increment(inc)
        assert [r["sor_sweeps"] for r in rg] == [r["sor_sweeps"] for r in ro]
        assert len(rg) == len(ro)
        np.testing.assert_allclose([r["sdx"] for r in rg], [r["sdx"] for r in ro], rtol=1e-8)
        g.download()
        o.download()
        for name in ("st", "ep", "x", "dx", "eps"):
            assert rel(getattr(pg, name), getattr(po, name)) < 1e-10, name
        assert rel(pg.sv[:, :15], po.sv[:, :15]) < 1e-10
        assert rel(pg.cumslip[:, :12], po.cumslip[:, :12]) < 1e-10
        # macroscopic stress-strain point: volume-weighted mean s11
        assert abs(pg.st[:, 0].mean() - po.st[:, 0].mean()) <= 1e-10 * abs(po.st[:, 0].mean())


def _collapsing_problem():
    p = generator.cube_config(n=3, ninc=2, grain=1, seed=2)
    return p


@pytest.mark.parametrize("case", ["906", "905", "920"])
def test_error_codes_match(case):
    p = _collapsing_problem()
    xyz = p.x.reshape(-1, 3)
    if case == "906":
        p.dx[:] = 0.0
        p.dx[3 * 20] = 0.9          # one huge strain increment
    elif case == "905":
        # a large rigid spin of every node about z
        c = xyz - xyz.mean(axis=0)
        p.dx.reshape(-1, 3)[:, 0] = -0.9 * c[:, 1]
        p.dx.reshape(-1, 3)[:, 1] = 0.9 * c[:, 0]
    else:
        xyz[p.ln[13] - 1] = xyz[p.ln[13][0] - 1]   # element 14 collapses to a point
    g, o, pg, po = pair(p)
    codes = []
    for s in (g, o):
        with pytest.raises(abi.FasError) as ei:
            s.elvals(1, 1)
        codes.append(ei.value.code)
    assert codes[0] == codes[1] == int(case)


def _twinning_material():
    """FCC slip plus twin systems on the same planes (ssang = 60 deg) with a
    low twin CRSS, so the twin trigger of SLPINI fires."""
    m = generator.fcc_aluminium()
    ns = 24
    ab = np.vstack([m["ab"], m["ab"]])
    an = np.vstack([m["an"], m["an"]])
    ampar = np.vstack([m["ampar"], m["ampar"]])
    ssang = np.concatenate([np.zeros(12), np.full(12, 60.0)])
    return dict(name="fcc-twin", ns=ns, e=m["e"], ssang=ssang, ab=ab, an=an, ampar=ampar,
                smatrx=np.ones((ns, ns)))


def test_twin_trigger_and_reorientation():
    mat = _twinning_material()
    p = generator.structured_cube(n=(3, 3, 3), ninc=2, materials=[mat], tau0=[30.0],
                                  twinlim=1, twinprob=1.0, seed=4)
    p.sv[:, 3 + 12:3 + 24] = 8.0            # twin CRSS below the flow stress
    g, o, pg, po = pair(p)
    for inc in (1, 2):
        rg, evg = g.increment(inc)
        ro, evo = o.increment(inc)
        assert len(rg) == len(ro)
        assert [(e["gp"], e["sys"]) for e in evg] == [(e["gp"], e["sys"]) for e in evo]
        for a, b in zip(evg, evo):
            np.testing.assert_allclose(a["euler_new"], b["euler_new"], rtol=1e-10, atol=1e-12)
        g.download()
        o.download()
        np.testing.assert_array_equal(pg.timestwinned, po.timestwinned)
        np.testing.assert_array_equal(pg.twinsys, po.twinsys)
        assert rel(pg.sv[:, :27], po.sv[:, :27]) < 1e-9
    assert pg.timestwinned.sum() > 0


def test_fp32_sor_refinement_error():
    """Tuned FACSLS (FP32 matrix sweeps, FP64 residual refinement) against
    the FP64 checker: the macroscopic stress and every GP's stress stay
    within the stated error after two increments."""
    p = generator.structured_cube(n=(12, 12, 12), ninc=2, seed=5)
    g, o, pg, po = pair(p, threads=8, mode=abi.FAS_MODE_SOR_GRID | abi.FAS_MODE_SOR_FP32)
    for inc in (1, 2):
        g.increment(inc)
        o.increment(inc)
    g.download()
    o.download()
    smax = np.abs(po.st).max()
    per_point = np.abs(pg.st - po.st).max() / smax
    macro = abs(pg.st[:, 0].mean() - po.st[:, 0].mean()) / abs(po.st[:, 0].mean())
    print(f"fp32 SOR: per-point {per_point:.2e}, macroscopic {macro:.2e}")
    assert per_point < 1e-5 and macro < 1e-6


@pytest.mark.parametrize("mode", [abi.FAS_MODE_PLAIN, abi.FAS_MODE_CP_WARP, abi.FAS_MODE_CP_QUEUE])
def test_mixed_fcc_hcp_increment(mode):
    """Mixed FCC (12 systems) / HCP (30 systems, with twins) grains: the
    32-system kernel instantiations against the checker, including twin
    triggers and reorientation."""
    p = generator.mixed_config(n=6, ninc=2)
    g, o, pg, po = pair(p, threads=8, mode=mode)
    for inc in (1, 2):
        rg, evg = g.increment(inc)
        ro, evo = o.increment(inc)
        assert len(rg) == len(ro)
        assert [(e["gp"], e["sys"]) for e in evg] == [(e["gp"], e["sys"]) for e in evo]
        g.download()
        o.download()
        assert rel(pg.st, po.st) < 1e-10
        assert rel(pg.sv[:, :33], po.sv[:, :33]) < 1e-10
        np.testing.assert_array_equal(pg.timestwinned, po.timestwinned)


def test_lattice_strain():
    p = generator.structured_cube(n=(3, 3, 3), ninc=1, seed=3)
    g, o, pg, po = pair(p)
    g.increment(1)
    o.increment(1)
    assert rel(g.lattice_strain(), o.lattice_strain()) < 1e-10

"""fs3pre's .fmt and .ori readers (SETMATC, src/prepro/fs3p-matl.f90:75-108;
SETSTATE option 4, src/prepro/fs3p-gps.f90:227-236) on files written in
those layouts, with the irregular spacing and tabs such files carry."""
import numpy as np

from cpfem_code_b200 import generator, inputs


def _write_fmt(path, m, nmpar=6):
    ns = m["ns"]
    with open(path, "w") as f:
        f.write(f"{nmpar}\n{ns}\n")
        f.write(" ".join(f"{v:.6e}" for v in m["e"]) + "\n")
        f.write(" ".join(f"{v:g}" for v in m["ssang"]) + "\n")
        for i in range(ns):
            f.write(" " + "  ".join(f"{v: .6f}" for v in (*m["ab"][i], *m["an"][i])) + " \t\n")
        for i in range(ns):
            f.write(" ".join(f"{v:.6g}" for v in m["ampar"][i, :nmpar]) + " \n")
        for i in range(ns):      # line i = smatrx(1:ns, i)
            f.write(" ".join(f"{v:.6g}" for v in np.asarray(m["smatrx"])[:, i]) + "\n")


def test_read_fmt_roundtrip(tmp_path):
    m = generator.fcc_aluminium()
    m["smatrx"] = np.arange(144, dtype=float).reshape(12, 12) / 7.0   # not symmetric
    path = str(tmp_path / "alu.fmt")
    _write_fmt(path, m)
    r = inputs.read_fmt(path)
    assert r["ns"] == 12 and r["nmpar"] == 6 and r["name"] == "alu"
    np.testing.assert_allclose(r["e"], m["e"], rtol=1e-6)
    np.testing.assert_allclose(r["ab"], m["ab"], atol=1e-6)
    np.testing.assert_allclose(r["an"], m["an"], atol=1e-6)
    np.testing.assert_allclose(r["ampar"][:, :6], m["ampar"][:, :6], rtol=1e-5)
    np.testing.assert_allclose(r["smatrx"], m["smatrx"], rtol=1e-5)
    # the packed tables hold smatrx(i, j) at [k, j, i], as the .fsd writer expects
    nss, *_, smatrx = generator.pack_materials([r])
    assert smatrx[0, 3, 5] == r["smatrx"][5, 3]


def test_read_ori_drives_generator(tmp_path):
    rng = np.random.default_rng(2)
    n = (2, 2, 1)
    ngps = 8 * 4
    ang = rng.random((ngps, 3)) * [6.28, 3.14, 6.28]
    path = str(tmp_path / "grains.ori")
    with open(path, "w") as f:
        for a in ang:
            f.write(f"   1.0000000e+00 {a[0]:15.7e} {a[1]:15.7e} {a[2]:15.7e}\n")
    eg = inputs.read_ori(path, ngps)
    np.testing.assert_allclose(eg, ang, rtol=1e-7)
    p = generator.structured_cube(n=n, ninc=1, nodes=20, euler_gp=eg)
    np.testing.assert_allclose(p.sv[:, :3], eg)

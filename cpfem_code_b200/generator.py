"""Structured-brick problem generator with fs3pre's semantics.

The reference builds its input with the interactive pre-processor ``fs3pre``
(src/prepro/fs3pre.f90) and writes a ``.fsd`` file.  This module produces the
same tables directly, for 8-node one-Gauss-point bricks (``lt = 12``) and
20-node eight-Gauss-point bricks (``lt = 22``):

* elements in (z, y, x) loop order with ADDEL_8NQ's or ADDEL_20NQ's local
  node order (src/prepro/fs3pre.f90:183-291);
* node numbers in first-occurrence order, which is what SWEEP's duplicate
  removal leaves (src/prepro/fs3p-swp.f90:53-109), computed with one sort
  instead of the O(nnod^2) sweep;
* SETBOUNDS codes for the four ``xfree`` options (src/prepro/fs3p-bkc.f90:9-174);
* SETKINC loading tables (src/prepro/fs3p-bkc.f90:182-308);
* random orientations per grain with fs3pre's uniform-SO(3) formulas
  (src/prepro/fs3p-gps.f90:105-110), seeded; grains are g x g x g blocks;
* SETMATC's equal initial slip resistance (src/prepro/fs3p-matl.f90:106-125).
"""
from __future__ import annotations

import itertools
import math

import numpy as np

from . import abi
from .problem import Control, Problem

# ADDEL_8NQ local node offsets (fs3pre.f90:193-196)
BRICK8 = np.array([(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0),
                   (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)], dtype=np.int64)
# ADDEL_20NQ local node offsets in half edges (fs3pre.f90:250-255): bottom
# face corners and mid-sides anticlockwise from the origin, the four
# vertical mid-edges, then the top face like the bottom one
BRICK20_HALF = np.array([(0, 0, 0), (1, 0, 0), (2, 0, 0), (2, 1, 0), (2, 2, 0), (1, 2, 0), (0, 2, 0),
                         (0, 1, 0), (0, 0, 1), (2, 0, 1), (2, 2, 1), (0, 2, 1), (0, 0, 2), (1, 0, 2),
                         (2, 0, 2), (2, 1, 2), (2, 2, 2), (1, 2, 2), (0, 2, 2), (0, 1, 2)], dtype=np.int64)



def _tet10_templates():
    """The 6 tetrahedra of a brick split along its main diagonal (Kuhn's
    triangulation), as 10-node elements in half edges: corners 1, 3, 5, 10
    with 1, 3, 5 anticlockwise seen from 10 (SHAPE_21's convention,
    src/fasolt/Shapef.f90:91-100), mid-edge nodes 2 (1,3), 4 (3,5), 6 (1,5),
    7 (1,10), 8 (3,10), 9 (5,10)."""
    out = []
    for perm in itertools.permutations(range(3)):
        v = [np.zeros(3, np.int64)]
        for k in perm[:2]:
            w = v[-1].copy()
            w[k] += 2
            v.append(w)
        v.append(np.array([2, 2, 2], np.int64))
        c1, c3, c5, c10 = v
        if np.dot(np.cross(c3 - c1, c5 - c1), c10 - c1) < 0:
            c3, c5 = c5, c3
        m = lambda a, b: (a + b) // 2
        out.append(np.array([c1, m(c1, c3), c3, m(c3, c5), c5, m(c1, c5), m(c1, c10), m(c3, c10), m(c5, c10), c10]))
    return out


def _wedge15_templates():
    """The 2 wedges of a brick split along the diagonal plane of its x-y
    faces, as 15-node elements in half edges: base corners 1, 3, 5
    anticlockwise seen from the top, top corners 10, 12, 14 above them,
    mid-edge nodes as SHAPE_23 numbers them (src/fasolt/Shapef.f90:348-356)."""
    out = []
    for tri in (((0, 0), (2, 0), (2, 2)), ((0, 0), (2, 2), (0, 2))):
        b = [np.array([x, y, 0], np.int64) for x, y in tri]
        t = [c + np.array([0, 0, 2]) for c in b]
        m = lambda a, c: (a + c) // 2
        out.append(np.array([b[0], m(b[0], b[1]), b[1], m(b[1], b[2]), b[2], m(b[2], b[0]),
                             m(b[0], t[0]), m(b[1], t[1]), m(b[2], t[2]),
                             t[0], m(t[0], t[1]), t[1], m(t[1], t[2]), t[2], m(t[2], t[0])]))
    return out


# element family: (element type lt, Gauss points, lattice step in the
# templates, node templates per brick of the lattice)
FAMILIES = {
    8: (12, 1, 1, [BRICK8]),
    10: (21, 4, 2, _tet10_templates()),
    15: (23, 6, 2, _wedge15_templates()),
    20: (22, 8, 2, [BRICK20_HALF]),
}

# ----------------------------------------------------------------- materials
def cubic_compliance(c11: float, c12: float, c44: float) -> np.ndarray:
    """e(1:9) = S11,S22,S33,S23,S31,S12,S44,S55,S66 (1/MPa) of a cubic crystal
    from stiffnesses in MPa (the .fmt compliance line, ela-plas.f90:56-74)."""
    d = (c11 - c12) * (c11 + 2.0 * c12)
    s11 = (c11 + c12) / d
    s12 = -c12 / d
    s44 = 1.0 / c44
    return np.array([s11, s11, s11, s12, s12, s12, s44, s44, s44])


def fcc_systems() -> tuple[np.ndarray, np.ndarray]:
    """The 12 {111}<110> systems in the order of src/prepro/crysdat.f90 and
    sample_input_files/aluminium2.fmt: three directions on each of the
    planes (111), (11-1), (-111), (1-11)."""
    planes = [(1, 1, 1), (1, 1, -1), (-1, 1, 1), (1, -1, 1)]
    dirs = [[(0, 1, -1), (-1, 0, 1), (1, -1, 0)],
            [(0, 1, 1), (-1, 0, -1), (1, -1, 0)],
            [(0, 1, -1), (1, 0, 1), (-1, -1, 0)],
            [(0, -1, -1), (-1, 0, 1), (1, 1, 0)]]
    ab, an = [], []
    for p, ds in zip(planes, dirs):
        for d in ds:
            assert sum(a * b for a, b in zip(p, d)) == 0
            ab.append(np.array(d, float) / math.sqrt(2.0))
            an.append(np.array(p, float) / math.sqrt(3.0))
    return np.array(ab), np.array(an)


def fcc_aluminium(m: float = 0.05, h0: float = 150.0, tau_sat: float = 80.0,
                  c11=108.2e3, c12=61.3e3, c44=28.5e3) -> dict:
    """FCC aluminium: power-law flow with exponent 1/m, Voce hardening
    theta = h0 (1 - s/tau_sat) (PLASTC with A3 = 0, A4 = 1, A6 = 0,
    ela-plas.f90:127-170) and a latent matrix of ones."""
    ab, an = fcc_systems()
    ns = 12
    ampar = np.zeros((ns, 10))
    ampar[:, 0] = m
    ampar[:, 1] = h0
    ampar[:, 2] = 0.0
    ampar[:, 3] = 1.0
    ampar[:, 4] = tau_sat
    ampar[:, 5] = 0.0
    return dict(name="fcc-al", ns=ns, e=cubic_compliance(c11, c12, c44),
                ssang=np.zeros(ns), ab=ab, an=an, ampar=ampar,
                smatrx=np.ones((ns, ns)))


def _mb_direction(uvtw, ca):
    """Miller-Bravais direction [uvtw] -> Cartesian, a1 along x."""
    u, v, t, w = uvtw
    return np.array([u - 0.5 * v - 0.5 * t, (v - t) * math.sqrt(3.0) / 2.0, w * ca])


def _mb_normal(hkil, ca):
    """Miller-Bravais plane (hkil) -> Cartesian normal, a1 along x."""
    h, k, i, l = hkil
    return np.array([h, (h + 2.0 * k) / math.sqrt(3.0), l / ca])


def _family(planes, dirs, ca):
    """All (plane, direction) pairs of the two index families that satisfy
    the zone law h*u + k*v + i*t + l*w = 0, planes in the given order."""
    out = []
    for pl in planes:
        for d in dirs:
            if sum(a * b for a, b in zip(pl, d)) == 0:
                n = _mb_normal(pl, ca)
                b = _mb_direction(d, ca)
                out.append((b / np.linalg.norm(b), n / np.linalg.norm(n)))
    return out


def _perms4(base):
    """The six hexagonal variants of a Miller-Bravais index (cyclic
    permutations of the first three indices, and their negatives in those
    indices), duplicates removed, order kept."""
    h, k, i, l = base
    seen, out = set(), []
    for a, b, c in ((h, k, i), (i, h, k), (k, i, h), (-h, -k, -i), (-i, -h, -k), (-k, -i, -h)):
        t = (a, b, c, l)
        if t not in seen:
            seen.add(t)
            out.append(t)
    return out


def hcp_systems(ca: float = 1.593):
    """30 HCP systems: basal <a> (3), prismatic <a> (3), first-order
    pyramidal <c+a> (12), second-order pyramidal <c+a> (6) and {10-12}
    tension twins (6) -- the families of
    additional_files/slip_systems/Zirconium that the mixed workload uses,
    derived here from their Miller-Bravais indices for c/a = `ca`.
    Returns ab, an (unit vectors) and a family label per system."""
    a_dirs = [(2, -1, -1, 0), (-1, 2, -1, 0), (-1, -1, 2, 0)]
    ca_dirs = _perms4((-1, -1, 2, 3))
    fam = []
    fam += [(s, "basal") for s in _family([(0, 0, 0, 1)], a_dirs, ca)]
    fam += [(s, "prism") for s in _family(_perms4((1, 0, -1, 0))[:3], a_dirs, ca)]
    fam += [(s, "pyr1ca") for s in _family(_perms4((1, 0, -1, 1)), ca_dirs, ca)]
    fam += [(s, "pyr2ca") for s in _family(_perms4((1, 1, -2, 2)), ca_dirs, ca)]
    twin_dirs = [d for d in _perms4((-1, 0, 1, 1))]
    fam += [(s, "twin") for s in _family(_perms4((1, 0, -1, 2)), twin_dirs, ca)]
    ab = np.array([f[0][0] for f in fam])
    an = np.array([f[0][1] for f in fam])
    labels = [f[1] for f in fam]
    return ab, an, labels


def hcp_zirconium(ca: float = 1.593, m: float = 0.05) -> dict:
    """HCP zirconium: compliances of additional_files/compliances (Zr line),
    the 30 systems of :func:`hcp_systems`, Voce hardening per family and
    {10-12} twins that reorient by 180 - 2 atan(sqrt(3)/(c/a)) degrees
    (85.2 for c/a = 1.593) -- the twin test of SLPINI needs |ssang| > 1.5."""
    ab, an, labels = hcp_systems(ca)
    ns = len(labels)
    assert ns == 30
    e = np.array([10.2e-6, 10.2e-6, 8.01e-6, -2.46e-6, -2.46e-6, -4.09e-6, 29.94e-6, 29.94e-6, 28.58e-6])
    tw = 180.0 - 2.0 * math.degrees(math.atan(math.sqrt(3.0) / ca))
    crss = {"basal": 45.0, "prism": 25.0, "pyr1ca": 90.0, "pyr2ca": 90.0, "twin": 30.0}
    ampar = np.zeros((ns, 10))
    ssang = np.zeros(ns)
    tau0 = np.zeros(ns)
    for k, lab in enumerate(labels):
        ampar[k, :6] = (m, 200.0, 0.0, 1.0, 2.5 * crss[lab], 0.0)
        tau0[k] = crss[lab]
        if lab == "twin":
            ssang[k] = tw
    return dict(name="hcp-zr", ns=ns, e=e, ssang=ssang, ab=ab, an=an, ampar=ampar,
                smatrx=np.ones((ns, ns)), tau0=tau0, labels=labels)


def pack_materials(mats: list[dict]):
    """Material tables in the FAS_CPL layout (ld_ss = 60)."""
    nm = len(mats)
    L = abi.FAS_MAXSS
    nss = np.array([m["ns"] for m in mats], np.int32)
    e = np.zeros((nm, 9))
    ssang = np.zeros((nm, L))
    ab = np.zeros((nm, L, 3))
    an = np.zeros((nm, L, 3))
    ampar = np.zeros((nm, L, 10))
    smatrx = np.zeros((nm, L, L))
    for k, m in enumerate(mats):
        ns = m["ns"]
        e[k] = m["e"]
        ssang[k, :ns] = m["ssang"]
        ab[k, :ns] = m["ab"]
        an[k, :ns] = m["an"]
        ampar[k, :ns] = m["ampar"]
        # smatrx(i, j, k) lives at [k, j, i]
        smatrx[k, :ns, :ns] = np.asarray(m["smatrx"]).T
    return nss, e, ssang, ab, an, ampar, smatrx


# ----------------------------------------------------------------- boundary codes
_FULL = {1: 100, 4: 200, 16: 300, 5: 400, 17: 500, 20: 600, 21: 700,
         2: 800, 8: 900, 32: 1000, 10: 1100, 34: 1200, 40: 1300, 42: 1400,
         9: 1500, 33: 1600, 6: 1700, 36: 1800, 18: 1900, 24: 2000,
         26: 2100, 38: 2200, 41: 2300, 37: 2400, 25: 2500, 22: 2600}
_FREEX = {1: 1, 2: 1, 5: 200, 6: 200, 9: 900, 10: 900, 17: 300, 18: 300,
          33: 1000, 34: 1000, 22: 600, 25: 2000, 26: 2000, 37: 1800, 38: 1800,
          41: 1300, 42: 1300}
_JUSTX = {**{k: 1 for k in (4, 8, 16, 20, 24, 32, 36, 40)},
          **{k: 100 for k in (1, 5, 9, 17, 25, 33, 37, 41)},
          **{k: 800 for k in (6, 10, 18, 22, 26, 34, 38, 42)}}


def setbounds(x: np.ndarray, tolerance: float, xfree: int) -> np.ndarray:
    """SETBOUNDS, src/prepro/fs3p-bkc.f90:9-174."""
    xyz = x.reshape(-1, 3)
    lo, hi = xyz.min(axis=0), xyz.max(axis=0)
    ib = np.zeros(xyz.shape[0], np.int32)
    for i in range(xyz.shape[0]):
        side = 0
        for j in range(3):
            if abs(xyz[i, j] - lo[j]) < tolerance:
                side += 2 ** (2 * j)
            if abs(xyz[i, j] - hi[j]) < tolerance:
                side += 2 ** (2 * j + 1)
        if side == 0:
            continue
        code = _FULL.get(side, 1)
        if xfree == 0:
            code = 5000
        elif xfree == 2:
            code = _FREEX.get(side, code)
        elif xfree == 3:
            code = _JUSTX.get(side, code)
        ib[i] = code
    return ib


def setties(x: np.ndarray, ib: np.ndarray, tolerance: float, tie=(True, True, True)) -> list:
    """SETTIES, src/prepro/fs3p-bkc.f90:316-405: tie elements for periodic
    boundary conditions.  For every node i1 on a lower face of a tied
    direction j1 (nodes and directions in the reference's loop order), every
    node i2 on the opposite face with the same other two coordinates gets a
    tie element (i1, i2) whose type follows i1's boundary class ib/100:
    classes 1-3 tie the two directions other than j1 (lt = j1 + 3), classes
    6/18/20, 5/16/19 and 4/15/17 tie x, y and z alone (lt 1, 2, 3); other
    classes get none.  Returns [(i1, i2, lt)] with 1-based node ids."""
    xyz = x.reshape(-1, 3)
    lo, hi = xyz.min(axis=0), xyz.max(axis=0)
    cls = ib // 100
    out = []
    for i1 in range(xyz.shape[0]):
        for j1 in range(3):
            if not (tie[j1] and abs(xyz[i1, j1] - lo[j1]) < tolerance):
                continue
            j2, j3 = (j1 + 1) % 3, (j1 + 2) % 3
            far = np.nonzero((np.abs(xyz[:, j1] - hi[j1]) < tolerance)
                             & (np.abs(xyz[i1, j2] - xyz[:, j2]) < tolerance)
                             & (np.abs(xyz[i1, j3] - xyz[:, j3]) < tolerance))[0]
            c = int(cls[i1])
            if c in (1, 2, 3):
                lt = j1 + 1 + 3
            elif c in (6, 18, 20):
                lt = 1
            elif c in (5, 16, 19):
                lt = 2
            elif c in (4, 15, 17):
                lt = 3
            else:
                continue
            out.extend((i1 + 1, int(i2) + 1, lt) for i2 in far)
    return out


def setkinc(xl, xfree: int, eps_inc, ninc1: int):
    """SETKINC, src/prepro/fs3p-bkc.f90:182-308: tiem and x_spec tables.
    `eps_inc` = (e11, e22, e33) increments; components the chosen `xfree`
    does not read are ignored as fs3pre ignores them."""
    ex, ey, ez = (float(v) for v in eps_inc)
    if xfree == 2:
        ex = 0.0
    elif xfree == 3:
        ey = ez = 0.0
    tiem = np.zeros(ninc1)
    xs = np.zeros((ninc1, abi.XSLD, 15))
    masks = {1: (1, 0, 0, 0, 0, 0), 2: (0, 0, 1, 0, 0, 0), 3: (0, 0, 0, 0, 0, 1),
             4: (1, 0, 1, 0, 0, 0), 5: (1, 0, 0, 0, 0, 1), 6: (0, 0, 1, 0, 0, 1),
             7: (1, 0, 1, 0, 0, 1)}
    for k in range(8, 15):
        masks[k] = masks[k - 7]
    for k, mk in zip(range(15, 21), (4, 5, 4, 6, 5, 6)):
        masks[k] = masks[mk]
    for k in range(21, 27):
        masks[k] = masks[7]
    xc, yc, zc = (float(v) for v in xl)
    for i in range(ninc1):
        tiem[i] = math.sqrt(ex ** 2 + ey ** 2 + ez ** 2)
        for code, mk in masks.items():
            xs[i, code - 1, :6] = mk
        dxs, dys, dzs = ex * xc, ey * yc, ez * zc
        xc, yc, zc = xc + dxs, yc + dys, zc + dzs
        for code in (8, 11, 12, 14, 17, 19, 21, 22, 26):
            xs[i, code - 1, 6] = dxs
        for code in (9, 11, 13, 14, 15, 20, 21, 23, 25):
            xs[i, code - 1, 10] = dys
        for code in (10, 12, 13, 14, 16, 18, 22, 23, 24):
            xs[i, code - 1, 14] = dzs
        xs[i, 49, :6] = (1, 0, 1, 0, 0, 1)
        xs[i, 49, 6] = ex
        xs[i, 49, 8] = 0.0
        xs[i, 49, 10] = ey
        xs[i, 49, 14] = ez
    return tiem, xs


# ----------------------------------------------------------------- the cube
def structured_cube(n=(8, 8, 8), lengths=(1.0, 1.0, 1.0), xfree: int = 3,
                    eps_inc=(1.0e-3, 0.0, 0.0), ninc: int = 10, grain: int = 1,
                    materials: list[dict] | None = None, fractions=None,
                    tau0: float | list[float] = 25.0, seed: int = 0,
                    twinlim: int = 0, twinprob: float = 0.0,
                    ctrl: Control | None = None, nodes: int = 8, ties=(False, False, False),
                    euler_gp: np.ndarray | None = None) -> Problem:
    """An nx x ny x nz brick of bricks with fs3pre's numbering, boundary
    codes, loading and per-grain random orientations (see module docstring).

    `nodes` = 8 gives ADDEL_8NQ's one-point bricks (``lt = 12``), 20 gives
    ADDEL_20NQ's 20-node, 8-point bricks (``lt = 22``, fs3pre.f90:241-291).
    `euler_gp` = [ngps, 3] Euler angles per Gauss point (an ``.ori`` file,
    see inputs.read_ori) in place of the random grain orientations.
    `ties` = (x, y, z) faces to tie for periodic boundary conditions: SETTIES's
    2-node tie elements follow the bricks (fs3pre.f90:171).
    `grain` = edge of the cubic grains in elements.  With several materials,
    each grain draws its material from `fractions` (fs3p-matl.f90:33-57
    draws per element; here per grain so grains stay single-phase)."""
    nx, ny, nz = (int(v) for v in n)
    if nodes not in FAMILIES:
        raise ValueError("nodes must be 8, 10, 15 or 20")
    materials = materials or [fcc_aluminium()]
    ltype, npg, h, tmpl = FAMILIES[nodes]
    nsub = len(tmpl)                         # elements per brick of the lattice
    nel = nx * ny * nz * nsub
    dxl = np.array([lengths[0] / nx, lengths[1] / ny, lengths[2] / nz])
    iz, iy, ix = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    # element order: x fastest, the sub-elements of one brick together
    ix, iy, iz = (np.repeat(a.ravel(), nsub) for a in (ix, iy, iz))
    # node positions on the lattice of half (quadratic) or whole edges (8 nodes)
    off_e = np.tile(np.stack(tmpl), (nx * ny * nz, 1, 1))    # [nel, nodes, 3]
    gx = h * ix[:, None] + off_e[:, :, 0]
    gy = h * iy[:, None] + off_e[:, :, 1]
    gz = h * iz[:, None] + off_e[:, :, 2]
    key = (gx + (h * nx + 1) * (gy + (h * ny + 1) * gz)).ravel()
    uniq, first, inv = np.unique(key, return_index=True, return_inverse=True)
    order = np.argsort(first, kind="stable")
    rank = np.empty_like(order)
    rank[order] = np.arange(order.size)
    ln = (rank[inv].reshape(nel, nodes) + 1).astype(np.int32)
    nnod = uniq.size
    # coordinates from the first-occurrence element: x0 + delx * xyz
    fo = first[order]
    fe, fa = fo // nodes, fo % nodes
    x0 = np.stack([dxl[0] * ix[fe], dxl[1] * iy[fe], dxl[2] * iz[fe]], axis=1)
    xyz = x0 + dxl[None, :] * (off_e[fe, fa] / float(h))
    x = np.ascontiguousarray(xyz.reshape(-1))
    tolerance = 0.5 * float(dxl.min()) / h   # SETSWTOL: 0.5 * shortest intra-element distance
    ib = setbounds(x, tolerance, xfree)

    rng = np.random.default_rng(seed)
    gxn, gyn, gzn = -(-nx // grain), -(-ny // grain), -(-nz // grain)
    ngr = gxn * gyn * gzn
    grain_id = (ix // grain) + gxn * ((iy // grain) + gyn * (iz // grain))
    u = rng.random((ngr, 3))
    euler = np.stack([6.2832 * u[:, 0], np.arccos(2.0 * u[:, 1] - 1.0), 6.2832 * u[:, 2]], axis=1)
    nm = len(materials)
    if nm > 1:
        fr = np.asarray(fractions if fractions is not None else [1.0] * nm, float)
        cum = np.cumsum(fr / fr.sum())
        r = rng.random(ngr)
        grain_mat = 1 + np.sum(r[:, None] > cum[None, :-1], axis=1)
    else:
        grain_mat = np.ones(ngr, np.int64)
    le = grain_mat[grain_id].astype(np.int32)

    nss, e, ssang, ab, an, ampar, smatrx = pack_materials(materials)
    tiem, x_spec = setkinc(lengths, xfree, eps_inc, ninc)
    nsv = 3 + int(nss.max())
    ngps = npg * nel
    lt = np.full(nel, ltype, np.int32)
    nd = np.full(nel, nodes, np.int32)
    npa = np.full(nel, npg, np.int32)
    lg = np.arange(1, ngps + 1, dtype=np.int32).reshape(nel, npg)
    le_all = le
    tl = setties(x, ib, tolerance, ties) if any(ties) else []
    if tl:
        nt = len(tl)
        t = np.array(tl, np.int32)
        ln = np.vstack([ln, np.pad(t[:, :2], ((0, 0), (0, nodes - 2)))])
        lt = np.concatenate([lt, t[:, 2]])
        nd = np.concatenate([nd, np.full(nt, 2, np.int32)])
        npa = np.concatenate([npa, np.zeros(nt, np.int32)])
        lg = np.vstack([lg, np.zeros((nt, npg), np.int32)])
        le_all = np.concatenate([le, np.zeros(nt, np.int32)])
    prob = Problem(
        nlmnt=len(lt), nnod=nnod, ngps=ngps, le=le_all, lt=lt, nd=nd, np_=npa, ln=ln, lg=lg, ib=ib,
        nss=nss, e=e, ssang=ssang, ab=ab, an=an, ampar=ampar, smatrx=smatrx,
        nmpar=6, twinlim=twinlim, twinprob=twinprob, tiem=tiem, x_spec=x_spec,
        f_spec=np.zeros((ninc, abi.XSLD, 3)), nxs=50, nfs=0,
        ctrl=ctrl or Control(), nsv=nsv)
    prob.zero_state()
    prob.x[:] = x
    gp_grain = np.repeat(grain_id, npg)      # the element's GPs share its grain
    prob.sv[:, 0:3] = euler[gp_grain]
    if euler_gp is not None:
        eg = np.asarray(euler_gp, float)
        if eg.shape != (ngps, 3):
            raise ValueError(f"euler_gp must be [{ngps}, 3]")
        prob.sv[:, 0:3] = eg
    t0 = np.broadcast_to(np.asarray(tau0, float), (nm,))
    gp_le = np.repeat(le, npg)
    for k in range(nm):
        sel = gp_le == k + 1
        if "tau0" in materials[k]:
            prob.sv[sel, 3:3 + nss[k]] = np.asarray(materials[k]["tau0"], float)[None, :]
        else:
            prob.sv[sel, 3:3 + nss[k]] = t0[k]
    prob.meta.update(dict(n=(nx, ny, nz), lengths=tuple(lengths), xfree=xfree, grain=grain, nodes=nodes,
                          ties=len(tl),
                          seed=seed, grain_id=grain_id.astype(np.int32),
                          materials=[m["name"] for m in materials]))
    return prob


def point_batch(npts: int, seed: int = 1, tau0: float = 25.0, strain_norm: float = 1.0e-3,
                material: dict | None = None, ctrl: Control | None = None) -> Problem:
    """Mesh-free batch of independent FCC material points (the constitutive
    micro-benchmark): uniform-SO(3) orientations, Gaussian strain increments
    rescaled to Frobenius norm `strain_norm`, CRSS uniform in [tau0, 2 tau0],
    zero spin and start stress, and the stress increment seeded with the
    elastic predictor S^-1 de so the plastic branch of DSTRSS runs."""
    material = material or fcc_aluminium()
    rng = np.random.default_rng(seed)
    nss, e, ssang, ab, an, ampar, smatrx = pack_materials([material])
    ns = int(nss[0])
    u = rng.random((npts, 3))
    euler = np.stack([6.2832 * u[:, 0], np.arccos(2.0 * u[:, 1] - 1.0), 6.2832 * u[:, 2]], axis=1)
    g = rng.standard_normal((npts, 3, 3))
    g = 0.5 * (g + g.transpose(0, 2, 1))
    g *= strain_norm / np.linalg.norm(g, axis=(1, 2))[:, None, None]
    de = np.stack([g[:, 0, 0], g[:, 1, 1], g[:, 2, 2],
                   2 * g[:, 1, 2], 2 * g[:, 2, 0], 2 * g[:, 0, 1]], axis=1)
    tiem = np.full(1, strain_norm)
    prob = Problem(
        nlmnt=0, nnod=0, ngps=npts, le=np.ones(npts, np.int32), lt=np.zeros(0, np.int32),
        nd=np.zeros(0, np.int32), np_=np.zeros(0, np.int32), ln=np.zeros((0, 8), np.int32),
        lg=np.zeros((0, 1), np.int32), ib=np.zeros(0, np.int32),
        nss=nss, e=e, ssang=ssang, ab=ab, an=an, ampar=ampar, smatrx=smatrx,
        nmpar=6, twinlim=0, twinprob=0.0, tiem=tiem,
        x_spec=np.zeros((1, abi.XSLD, 15)), f_spec=np.zeros((1, abi.XSLD, 3)),
        nxs=0, nfs=0, ctrl=ctrl or Control(), nsv=3 + ns)
    prob.zero_state()
    prob.sv[:, 0:3] = euler
    prob.sv[:, 3:3 + ns] = tau0 * (1.0 + rng.random((npts, ns)))
    prob.de[:] = de
    # elastic predictor in the rotated crystal frame
    prob.ds[:] = elastic_predictor(e[0], euler, de)
    return prob


def rotated_compliance(e9: np.ndarray, euler: np.ndarray) -> np.ndarray:
    """Vectorised ELASTC (ela-plas.f90:12-86) for many orientations:
    [n, 6, 6] compliances with engineering shears."""
    ph1, phi, ph2 = euler[:, 0], euler[:, 1], euler[:, 2]
    c1, s1, c2, s2, c, s = np.cos(ph1), np.sin(ph1), np.cos(ph2), np.sin(ph2), np.cos(phi), np.sin(phi)
    a = np.zeros((euler.shape[0], 3, 3))
    a[:, 0, 0] = c1 * c2 - s1 * s2 * c
    a[:, 1, 0] = -c1 * s2 - s1 * c2 * c
    a[:, 2, 0] = s1 * s
    a[:, 0, 1] = s1 * c2 + c1 * s2 * c
    a[:, 1, 1] = -s1 * s2 + c1 * c2 * c
    a[:, 2, 1] = -c1 * s
    a[:, 0, 2] = s2 * s
    a[:, 1, 2] = c2 * s
    a[:, 2, 2] = c
    at = a.transpose(0, 2, 1)
    pi = [0, 1, 2, 1, 2, 0]
    pj = [0, 1, 2, 2, 0, 1]
    S = np.zeros((euler.shape[0], 6, 6))
    for I in range(6):
        i, j = pi[I], pj[I]
        mult = 1.0 if I < 3 else 2.0
        for J in range(6):
            k, l = pi[J], pj[J]
            A = lambda p, q: at[:, p, q]
            t1 = (A(i, 0) * A(j, 0) * A(k, 0) * A(l, 0) * e9[0] + A(i, 1) * A(j, 1) * A(k, 1) * A(l, 1) * e9[1]
                  + A(i, 2) * A(j, 2) * A(k, 2) * A(l, 2) * e9[2])
            t2 = (A(i, 1) * A(j, 1) * A(k, 2) * A(l, 2) * e9[3] + A(i, 2) * A(j, 2) * A(k, 1) * A(l, 1) * e9[3]
                  + A(i, 2) * A(j, 2) * A(k, 0) * A(l, 0) * e9[4] + A(i, 0) * A(j, 0) * A(k, 2) * A(l, 2) * e9[4]
                  + A(i, 0) * A(j, 0) * A(k, 1) * A(l, 1) * e9[5] + A(i, 1) * A(j, 1) * A(k, 0) * A(l, 0) * e9[5])
            t3 = (A(i, 1) * A(j, 2) * A(k, 1) * A(l, 2) * e9[6] + A(i, 2) * A(j, 1) * A(k, 2) * A(l, 1) * e9[6]
                  + A(i, 2) * A(j, 0) * A(k, 2) * A(l, 0) * e9[7] + A(i, 0) * A(j, 2) * A(k, 0) * A(l, 2) * e9[7]
                  + A(i, 0) * A(j, 1) * A(k, 0) * A(l, 1) * e9[8] + A(i, 1) * A(j, 0) * A(k, 1) * A(l, 0) * e9[8])
            S[:, I, J] = mult * (t1 + t2 + 0.5 * t3)
    iu = np.triu_indices(6, 1)
    S[:, iu[1], iu[0]] = S[:, iu[0], iu[1]]
    return S


def elastic_predictor(e9: np.ndarray, euler: np.ndarray, de: np.ndarray) -> np.ndarray:
    S = rotated_compliance(e9, euler)
    return np.linalg.solve(S, de[:, :, None])[:, :, 0]


# ----------------------------------------------------------------- named workloads
def cube_config(n: int, ninc: int, grain: int, seed: int, eps: float = 1.0e-3,
                ctrl: Control | None = None, nodes: int = 8) -> Problem:
    """FCC aluminium n^3 cube in uniaxial tension along x ("just x faces",
    xfree = 3), strain increment `eps` per increment, grains of grain^3
    elements with seeded uniform-SO(3) orientations; `nodes` = 8 or 20."""
    return structured_cube(n=(n, n, n), xfree=3, eps_inc=(eps, 0.0, 0.0), ninc=ninc,
                           grain=grain, seed=seed, ctrl=ctrl, nodes=nodes)


def mixed_config(n: int = 32, ninc: int = 20, seed: int = 32, eps: float = 1.0e-3,
                 ctrl: Control | None = None) -> Problem:
    """n^3 cube of 50/50 random HCP-Zr / FCC-Al grains of 2^3 elements in
    uniaxial tension; HCP is material 1 (DoReorient reads material 1's
    tables, Fasolt3.f90:103,124-125), twins fire with probability 1, at most
    once per GP."""
    return structured_cube(n=(n, n, n), xfree=3, eps_inc=(eps, 0.0, 0.0), ninc=ninc, grain=2,
                           materials=[hcp_zirconium(), fcc_aluminium()], fractions=[0.5, 0.5],
                           seed=seed, twinlim=1, twinprob=1.0, ctrl=ctrl)


WORKLOADS = {
    # 8^3 FCC, one grain per element, 10 increments to 1 %
    "cube8": dict(n=8, ninc=10, grain=1, seed=8),
    # 16^3 FCC, 20 increments to 2 %
    "cube16": dict(n=16, ninc=20, grain=1, seed=16),
    # 64^3 FCC, grains of 2^3 elements, 50 increments to 5 %
    "cube64": dict(n=64, ninc=50, grain=2, seed=64),
    # the reference sample's mesh: 10^3 20-node bricks, one grain per element
    "brick20_10": dict(n=10, ninc=10, grain=1, seed=10, nodes=20),
    # 32^3 20-node bricks (262,144 GPs), grains of 2^3 elements
    "brick20_32": dict(n=32, ninc=50, grain=2, seed=32, nodes=20),
}


def workload(name: str, **over) -> Problem:
    if name.startswith("mixed"):
        kw = dict(n=int(name[5:] or 32))
        kw.update(over)
        return mixed_config(**kw)
    kw = dict(WORKLOADS[name])
    kw.update(over)
    return cube_config(**kw)

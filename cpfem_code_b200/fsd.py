"""FASOLT3 problem / result files: ``.fsd`` (from fs3pre) and ``.frs`` (from
fasolt3's save points).

Both are Fortran unformatted sequential files: every WRITE is one record
framed by a 4-byte little-endian length before and after it.  The record
order is that of WTDATA (src/fasolt/Faslt_io_nowin.f90:185-299, and
src/prepro/fs3p-io_nowin.f90:10-117 for ``.fsd``), which RDDATA reads back
(src/fasolt/Faslt_io_nowin.f90:9-146).  The only difference between the two
files is the first record: ``ninc1`` in an ``.fsd``, the saved increment
``inc`` in an ``.frs``.  Reals are REAL(4) as the reference ships
(``real_bytes = 8`` writes the layout a REAL(8) build would use).
"""
from __future__ import annotations

import struct

import numpy as np

from . import abi
from .problem import Problem


class _Writer:
    def __init__(self, f, rb: int):
        self.f = f
        self.rt = "<f4" if rb == 4 else "<f8"

    def rec(self, *parts):
        payload = b"".join(parts)
        n = struct.pack("<i", len(payload))
        self.f.write(n + payload + n)

    def ints(self, *v):
        return np.asarray(v, "<i4").tobytes()

    def reals(self, v):
        return np.asarray(v, dtype=np.float64).astype(self.rt).tobytes()


class _Reader:
    def __init__(self, buf: bytes, rb: int):
        self.b = buf
        self.o = 0
        self.rt = "<f4" if rb == 4 else "<f8"

    def rec(self) -> bytes:
        (n,) = struct.unpack_from("<i", self.b, self.o)
        data = self.b[self.o + 4:self.o + 4 + n]
        (m,) = struct.unpack_from("<i", self.b, self.o + 4 + n)
        if m != n:
            raise ValueError(f"corrupt record at byte {self.o}: markers {n} != {m}")
        self.o += 8 + n
        return data

    def ints(self):
        return np.frombuffer(self.rec(), "<i4")

    def reals(self):
        return np.frombuffer(self.rec(), self.rt).astype(np.float64)


def write(path: str, p: Problem, first_record: int | None = None, real_bytes: int = 4) -> None:
    """WTDATA's record sequence for problem `p`.  `first_record` defaults to
    ninc1 (an ``.fsd``); pass the increment number for an ``.frs``."""
    p.zero_state()
    first = p.ninc1 if first_record is None else int(first_record)
    nmpar = int(p.nmpar)
    with open(path, "wb") as f:
        w = _Writer(f, real_bytes)
        w.rec(w.ints(first))
        w.rec(w.ints(p.nlmnt, p.nnod, p.ngps, p.nsv))
        for e in range(p.nlmnt):
            nd, npe = int(p.nd[e]), int(p.np_[e])
            w.rec(w.ints(p.le[e], p.lt[e], nd, npe))
            w.rec(w.ints(*p.ln[e, :nd]))
            w.rec(w.ints(*p.lg[e, :npe]))
        x = p.x.reshape(-1, 3)
        dx = p.dx.reshape(-1, 3)
        fc = p.fc.reshape(-1, 3)
        for n in range(p.nnod):
            w.rec(w.ints(p.ib[n]))
            w.rec(w.reals(np.concatenate([x[n], dx[n]])))
            w.rec(w.reals(fc[n]))
        for g in range(p.ngps):
            w.rec(w.reals([p.eps[g], p.dep[g]]))
            w.rec(w.reals(p.sv[g, :p.nsv]))
            w.rec(w.reals(p.dsv[g, :p.nsv]))
            for name, k in (("ep", 6), ("de", 6), ("st", 6), ("ds", 6), ("rt", 3), ("dr", 3)):
                w.rec(w.reals(getattr(p, name)[g, :k]))
        w.rec(w.ints(p.nmatl, nmpar))
        for m in range(p.nmatl):
            ns = int(p.nss[m])
            w.rec(w.ints(ns))
            w.rec(w.ints(p.twinlim))
            w.rec(w.reals([p.twinprob]))
            w.rec(w.reals(p.e[m]))
            w.rec(w.reals(p.ssang[m, :ns]))
            for i in range(ns):
                w.rec(w.reals(np.concatenate([p.ab[m, i], p.an[m, i]])))
            for i in range(ns):
                w.rec(w.reals(p.ampar[m, i, :nmpar]))
            for i in range(ns):
                w.rec(w.reals(p.smatrx[m, i, :ns]))      # smatrx(1:ns, i)
        w.rec(w.reals([0.0, 0.0, 0.0]))                   # amu, anu, aga
        w.rec(w.ints(p.ninc1, p.nxs, p.nfs))
        for i in range(p.ninc1):
            w.rec(w.reals([p.tiem[i]]))
            for j in range(p.nxs):
                w.rec(w.reals(p.x_spec[i, j]))
            for j in range(p.nfs):
                w.rec(w.reals(p.f_spec[i, j]))


def read(path: str, real_bytes: int = 4) -> tuple[Problem, int]:
    """RDDATA's record sequence.  Returns the problem and the first record
    (ninc1 of an ``.fsd``, the saved increment of an ``.frs``)."""
    with open(path, "rb") as f:
        r = _Reader(f.read(), real_bytes)
    first = int(r.ints()[0])
    nlmnt, nnod, ngps, nsv = (int(v) for v in r.ints())
    le, lt, nd, npe = (np.zeros(nlmnt, np.int32) for _ in range(4))
    lns, lgs = [], []
    for e in range(nlmnt):
        le[e], lt[e], nd[e], npe[e] = r.ints()
        lns.append(r.ints()[:nd[e]])
        lgs.append(r.ints()[:npe[e]])
    if nlmnt and (nd.max() > 20 or npe.max() > 8):
        raise ValueError("elements with more than 20 nodes or 8 Gauss points")
    ln = np.zeros((nlmnt, max(int(nd.max()) if nlmnt else 1, 1)), np.int32)
    lg = np.zeros((nlmnt, max(int(npe.max()) if nlmnt else 1, 1)), np.int32)
    for e in range(nlmnt):
        ln[e, :nd[e]] = lns[e]
        lg[e, :npe[e]] = lgs[e]
    ib = np.zeros(nnod, np.int32)
    x = np.zeros(3 * nnod)
    dx = np.zeros(3 * nnod)
    fc = np.zeros(3 * nnod)
    for n in range(nnod):
        ib[n] = r.ints()[0]
        v = r.reals()
        x[3 * n:3 * n + 3], dx[3 * n:3 * n + 3] = v[:3], v[3:6]
        fc[3 * n:3 * n + 3] = r.reals()
    st = {k: np.zeros((ngps, n)) for k, n in (("ep", 6), ("de", 6), ("st", 6), ("ds", 6), ("rt", 3), ("dr", 3))}
    eps, dep = np.zeros(ngps), np.zeros(ngps)
    sv = np.zeros((ngps, abi.SVLD))
    dsv = np.zeros((ngps, abi.SVLD))
    for g in range(ngps):
        eps[g], dep[g] = r.reals()
        sv[g, :nsv] = r.reals()
        dsv[g, :nsv] = r.reals()
        for k in ("ep", "de", "st", "ds", "rt", "dr"):
            st[k][g] = r.reals()
    nmatl, nmpar = (int(v) for v in r.ints())
    L = abi.FAS_MAXSS
    nss = np.zeros(nmatl, np.int32)
    e9 = np.zeros((nmatl, 9))
    ssang = np.zeros((nmatl, L))
    ab = np.zeros((nmatl, L, 3))
    an = np.zeros((nmatl, L, 3))
    ampar = np.zeros((nmatl, L, 10))
    smatrx = np.zeros((nmatl, L, L))
    twinlim, twinprob = 0, 0.0
    for m in range(nmatl):
        ns = int(r.ints()[0])
        nss[m] = ns
        twinlim = int(r.ints()[0])
        twinprob = float(r.reals()[0])
        e9[m] = r.reals()
        ssang[m, :ns] = r.reals()
        for i in range(ns):
            v = r.reals()
            ab[m, i], an[m, i] = v[:3], v[3:6]
        for i in range(ns):
            ampar[m, i, :nmpar] = r.reals()
        for i in range(ns):
            smatrx[m, i, :ns] = r.reals()
    r.reals()                                              # amu, anu, aga
    ninc1, nxs, nfs = (int(v) for v in r.ints())
    tiem = np.zeros(ninc1)
    x_spec = np.zeros((ninc1, abi.XSLD, 15))
    f_spec = np.zeros((ninc1, abi.XSLD, 3))
    for i in range(ninc1):
        tiem[i] = r.reals()[0]
        for j in range(nxs):
            x_spec[i, j] = r.reals()
        for j in range(nfs):
            f_spec[i, j] = r.reals()
    p = Problem(nlmnt=nlmnt, nnod=nnod, ngps=ngps, le=le, lt=lt, nd=nd, np_=npe, ln=ln, lg=lg, ib=ib,
                nss=nss, e=e9, ssang=ssang, ab=ab, an=an, ampar=ampar, smatrx=smatrx, nmpar=nmpar,
                twinlim=twinlim, twinprob=twinprob, tiem=tiem, x_spec=x_spec, f_spec=f_spec,
                nxs=nxs, nfs=nfs, nsv=nsv, x=x, dx=dx, fc=fc, eps=eps, dep=dep, sv=sv, dsv=dsv, **st)
    p.zero_state()
    return p, first

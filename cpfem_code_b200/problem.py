"""Host-side container of one FASOLT3 problem.

Mirrors the FAS_COM / FAS_CPL module arrays (src/fasolt/fas-com-mod.f90:9-80)
that RDDATA fills (src/fasolt/Faslt_io_nowin.f90:9-146).  Every array keeps
the Fortran memory layout (axes reversed, C-ordered), 1-based index values,
and is handed to the C ABI by pointer through :meth:`descriptors`.
"""
from __future__ import annotations

import copy
from dataclasses import dataclass, field

import numpy as np

from . import abi


@dataclass
class Control:
    """fafcdf.dat (FSINIT, src/fasolt/Fasolt3.f90:216-218)."""
    toler: float = 1.0e-3
    maxit: int = 100
    alpha: float = 20.0
    afactor: float = 1.0
    efix: float = 1.0e20
    smalp: float = 0.1
    smalf: float = 10.0
    smald: float = 1.0e-5
    smale: float = 0.5
    smalr: float = 0.5
    twin_seed: int = 0x5EED


@dataclass
class Problem:
    # ---- mesh (FAS_COM)
    nlmnt: int
    nnod: int
    ngps: int
    le: np.ndarray          # [nlmnt] material code (negative: elastic only)
    lt: np.ndarray          # [nlmnt] element type (12 = 8-node 1-GP brick)
    nd: np.ndarray          # [nlmnt] nodes per element
    np_: np.ndarray         # [nlmnt] Gauss points per element
    ln: np.ndarray          # [nlmnt, 8] 1-based node ids   == ln(8, nlmnt)
    lg: np.ndarray          # [nlmnt, 1] 1-based GP ids     == lg(1, nlmnt)
    ib: np.ndarray          # [nnod] boundary codes
    # ---- materials (FAS_CPL)
    nss: np.ndarray         # [nmatl]
    e: np.ndarray           # [nmatl, 9]
    ssang: np.ndarray       # [nmatl, 60]
    ab: np.ndarray          # [nmatl, 60, 3]
    an: np.ndarray          # [nmatl, 60, 3]
    ampar: np.ndarray       # [nmatl, 60, 10]
    smatrx: np.ndarray      # [nmatl, 60, 60]  == smatrx(60, 60, nmatl)
    nmpar: int = 6
    twinlim: int = 0
    twinprob: float = 0.0
    # ---- loading (RDDATA control records)
    tiem: np.ndarray = None       # [ninc1]
    x_spec: np.ndarray = None     # [ninc1, 99, 15] == x_spec(15, 99, ninc1)
    f_spec: np.ndarray = None     # [ninc1, 99, 3]
    nxs: int = 50
    nfs: int = 0
    ctrl: Control = field(default_factory=Control)
    # ---- state
    nsv: int = 15
    x: np.ndarray = None
    dx: np.ndarray = None
    fc: np.ndarray = None
    ddx: np.ndarray = None
    eps: np.ndarray = None
    dep: np.ndarray = None
    st: np.ndarray = None         # [ngps, 6]
    ep: np.ndarray = None
    ds: np.ndarray = None
    de: np.ndarray = None
    rt: np.ndarray = None         # [ngps, 3]
    dr: np.ndarray = None
    sv: np.ndarray = None         # [ngps, 63]
    dsv: np.ndarray = None
    timestwinned: np.ndarray = None
    twinsys: np.ndarray = None
    srate: np.ndarray = None      # [ngps, 60]
    cumslip: np.ndarray = None
    meta: dict = field(default_factory=dict)

    @property
    def nmatl(self) -> int:
        return int(self.nss.shape[0])

    @property
    def ninc1(self) -> int:
        return int(self.tiem.shape[0])

    def zero_state(self) -> None:
        """Allocate the state arrays, zero except what the caller sets."""
        nd3, g = 3 * self.nnod, self.ngps
        f8 = np.float64
        for name, shape in (("x", nd3), ("dx", nd3), ("fc", nd3), ("ddx", nd3),
                            ("eps", g), ("dep", g), ("st", (g, 6)), ("ep", (g, 6)),
                            ("ds", (g, 6)), ("de", (g, 6)), ("rt", (g, 3)), ("dr", (g, 3)),
                            ("sv", (g, abi.SVLD)), ("dsv", (g, abi.SVLD)),
                            ("srate", (g, abi.FAS_MAXSS)), ("cumslip", (g, abi.FAS_MAXSS))):
            if getattr(self, name) is None:
                setattr(self, name, np.zeros(shape, f8))
        if self.timestwinned is None:
            self.timestwinned = np.zeros(g, np.int32)
        if self.twinsys is None:
            self.twinsys = np.zeros(g, np.int32)

    def copy(self) -> "Problem":
        return copy.deepcopy(self)

    def first_points(self, n: int) -> "Problem":
        """The first n points of a mesh-free point batch (nlmnt == 0), with
        their state, as a batch of their own."""
        if self.nlmnt != 0:
            raise ValueError("first_points needs a mesh-free point batch")
        n = min(int(n), self.ngps)
        out = copy.copy(self)
        out.ngps = n
        out.le = self.le[:n].copy()
        out.meta = dict(self.meta)
        for name in ("eps", "dep", "st", "ep", "ds", "de", "rt", "dr", "sv", "dsv",
                     "timestwinned", "twinsys", "srate", "cumslip"):
            a = getattr(self, name)
            if a is not None:
                setattr(out, name, a[:n].copy())
        for name in ("e", "ssang", "ab", "an", "ampar", "smatrx", "nss", "tiem", "x_spec", "f_spec",
                     "x", "dx", "fc", "ddx"):
            a = getattr(self, name)
            if a is not None:
                setattr(out, name, a.copy())
        return out

    # ------------------------------------------------------------ descriptors
    def descriptors(self):
        """(mesh, matl, ctrl) ctypes descriptors pointing into this object."""
        mesh = abi.FasMesh(
            nlmnt=self.nlmnt, nnod=self.nnod, ngps=self.ngps,
            le=abi.iptr(self.le), lt=abi.iptr(self.lt), nd=abi.iptr(self.nd),
            np=abi.iptr(self.np_), ln=abi.iptr(self.ln), ld_ln=self.ln.shape[1],
            lg=abi.iptr(self.lg), ld_lg=self.lg.shape[1], ib=abi.iptr(self.ib))
        matl = abi.FasMatl(
            real_bytes=8, nmatl=self.nmatl, nmpar=self.nmpar, ld_ss=abi.FAS_MAXSS,
            nss=abi.iptr(self.nss), e=abi.ptr(self.e), ssang=abi.ptr(self.ssang),
            ab=abi.ptr(self.ab), an=abi.ptr(self.an), ampar=abi.ptr(self.ampar),
            smatrx=abi.ptr(self.smatrx), twinlim=int(self.twinlim),
            twinprob=float(self.twinprob))
        c = self.ctrl
        ctrl = abi.FasCtrl(
            real_bytes=8, maxit=int(c.maxit), toler=c.toler, alpha=c.alpha,
            afactor=c.afactor, efix=c.efix, smale=c.smale, smalr=c.smalr,
            ninc1=self.ninc1, nxs=int(self.nxs), nfs=int(self.nfs), ld_xs=abi.XSLD,
            tiem=abi.ptr(self.tiem), x_spec=abi.ptr(self.x_spec),
            f_spec=abi.ptr(self.f_spec), twin_seed=int(c.twin_seed))
        return mesh, matl, ctrl

    def state_descriptor(self) -> abi.FasState:
        """FasState over this object's state arrays (FP64)."""
        self.zero_state()
        return abi.FasState(
            real_bytes=8, nsv=int(self.nsv), ld_sv=abi.SVLD, ld_slip=abi.FAS_MAXSS,
            x=abi.ptr(self.x), dx=abi.ptr(self.dx), fc=abi.ptr(self.fc), ddx=abi.ptr(self.ddx),
            eps=abi.ptr(self.eps), dep=abi.ptr(self.dep),
            st=abi.ptr(self.st), ep=abi.ptr(self.ep), ds=abi.ptr(self.ds), de=abi.ptr(self.de),
            rt=abi.ptr(self.rt), dr=abi.ptr(self.dr), sv=abi.ptr(self.sv), dsv=abi.ptr(self.dsv),
            timestwinned=abi.iptr(self.timestwinned), twinsys=abi.iptr(self.twinsys),
            srate=abi.ptr(self.srate), cumslip=abi.ptr(self.cumslip))

    def state_bytes(self) -> int:
        """Bytes of the FP64 state that one upload (or download) moves."""
        self.zero_state()
        names = ("x", "dx", "fc", "ddx", "eps", "dep", "st", "ep", "ds", "de", "rt", "dr",
                 "sv", "dsv", "timestwinned", "twinsys", "srate", "cumslip")
        return int(sum(getattr(self, n).nbytes for n in names))

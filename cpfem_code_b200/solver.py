"""Python face of the C ABI, with the reference's routine names.

:class:`GpuSolver` drives ``libfasgpu.so`` (the sm_100a implementation) the
way the Fortran driver (src/fasolt/Fasolt3.f90:38-60) drives its routines:
``update_node``, ``nriter``, ``update_gptv``, ``do_reorient`` per increment,
or the finer ``elvals`` / ``suvals`` / ``facsls`` steps of NRITER
(src/fasolt/Stif_sol.f90:10-88).  A non-zero status raises
:class:`~cpfem_code_b200.abi.FasError` carrying the FAFERR code the reference
would have raised.  There is no CPU fallback: without the built library or
without a B200 the constructor raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi
from .problem import Problem

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libfasgpu.so")
_lib = None


def load_library(path: str | None = None) -> C.CDLL:
    """Load the device library once.  Raises if it has not been built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"{p} is missing: build it with `python -m cpfem_code_b200.build` "
            "(the GPU path has no CPU fallback)")
    lib = C.CDLL(p)
    abi.declare(lib, "fas_gpu")
    if path is None:
        _lib = lib
    return lib


class _SolverBase:
    """Shared driver logic over a library with the fasolt_gpu.h signatures."""

    prefix = "fas_gpu"

    def __init__(self, lib: C.CDLL, prob: Problem, handle: C.c_void_p):
        self._lib = lib
        self.prob = prob
        self._h = handle
        self._fn = lambda name: getattr(self._lib, f"{self.prefix}_{name}")

    # ---- lifecycle
    def close(self) -> None:
        if self._h:
            self._fn("destroy")(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _call(self, name: str, *args) -> int:
        if not self._h:
            raise abi.FasError(abi.FAS_E_STATE, name)
        return abi.check(self._fn(name)(self._h, *args), f"{self.prefix}_{name}")

    def set_mode(self, mode: int) -> None:
        self._call("set_mode", C.c_uint32(mode))

    # ---- state transfer
    def upload(self, prob: Problem | None = None) -> None:
        p = prob or self.prob
        self._call("upload_state", C.byref(p.state_descriptor()))

    def download(self, prob: Problem | None = None) -> Problem:
        p = prob or self.prob
        self._call("download_state", C.byref(p.state_descriptor()))
        return p

    # ---- reference routines
    def update_node(self) -> None:
        self._call("update_node")

    def elvals(self, inc: int, nit: int = 1) -> None:
        self._call("elvals", inc, nit)

    def suvals(self, inc: int) -> None:
        self._call("suvals", inc)

    def facsls(self) -> tuple[int, float]:
        sweeps, err = C.c_int32(0), C.c_double(0.0)
        self._call("facsls", C.byref(sweeps), C.byref(err))
        return sweeps.value, err.value

    def nriter(self, inc: int, cap: int = 128) -> list[dict]:
        rep = (abi.FasIterReport * cap)()
        n = C.c_int32(0)
        try:
            self._call("nriter", inc, rep, cap, C.byref(n))
        finally:
            self.last_report = _report(rep, min(n.value, cap))
        return self.last_report

    def nr_step(self, inc: int, nit: int):
        """One pass of NRITER's loop body (src/fasolt/Stif_sol.f90:32-77);
        returns (report line, whether NRITER would go on)."""
        r = abi.FasIterReport()
        more = C.c_int32(0)
        self._call("nr_step", inc, nit, C.byref(r), C.byref(more))
        return _report([r], 1)[0], bool(more.value)

    def nr_finish(self, inc: int) -> None:
        """NRITER's cumslip update after its loop (Stif_sol.f90:80-84)."""
        self._call("nr_finish", inc)

    def update_gptv(self) -> None:
        self._call("update_gptv")

    def do_reorient(self, inc: int, cap: int = 65536) -> list[dict]:
        ev = (abi.FasTwinEvent * cap)()
        n = C.c_int32(0)
        self._call("reorient", inc, ev, cap, C.byref(n))
        return _events(ev, min(n.value, cap))

    def increment(self, inc: int, cap: int = 128, ev_cap: int = 65536):
        """UPDATE_NODE -> NRITER -> UPDATE_GPTV -> DoReorient (when a twin
        fired): one pass of the driver loop, src/fasolt/Fasolt3.f90:38-46."""
        rep = (abi.FasIterReport * cap)()
        ev = (abi.FasTwinEvent * ev_cap)()
        n, nev = C.c_int32(0), C.c_int32(0)
        try:
            self._call("increment", inc, rep, cap, C.byref(n), ev, ev_cap, C.byref(nev))
        finally:
            self.last_report = _report(rep, min(n.value, cap))
        return self.last_report, _events(ev, min(nev.value, ev_cap))

    def constitutive(self, inc: int = 1, nit: int = 1) -> None:
        self._call("constitutive", inc, nit)

    # ---- inspection
    def pattern(self, ld: int = 96) -> np.ndarray:
        """SETPTA's `is` array, [3*nnod, ld] (== is(ld, 3*nnod)), 1-based."""
        out = np.zeros((3 * self.prob.nnod, ld), np.int32)
        self._call("get_pattern", abi.iptr(out), ld)
        return out

    def stiffness(self, ld: int = 96) -> np.ndarray:
        out = np.zeros((3 * self.prob.nnod, ld), np.float64)
        self._call("get_stiffness", abi.ptr(out), ld, 8)
        return out

    def colouring(self) -> tuple[np.ndarray, int]:
        col = np.zeros(self.prob.nnod, np.int32)
        n = C.c_int32(0)
        self._call("get_colouring", abi.iptr(col), C.byref(n))
        return col, n.value

    def tangent(self) -> np.ndarray:
        """chi(6,6,ngps) as [ngps, 6(col), 6(row)]."""
        out = np.zeros((self.prob.ngps, 6, 6), np.float64)
        self._call("get_tangent", abi.ptr(out), 8)
        return out

    def lattice_strain(self) -> np.ndarray:
        """ELASEPS for every GP: [ngps, 6] elastic strains (engineering shears)."""
        out = np.zeros((self.prob.ngps, 6), np.float64)
        if self.prefix == "fas_gpu":
            self._call("lattice_strain", abi.ptr(out), 8)
        else:
            self._call("lattice_strain", abi.ptr(out))
        return out

    def cp_ops(self) -> np.ndarray:
        out = np.zeros(self.prob.ngps, np.float64)
        self._call("get_cp_ops", out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def adjoint_forward(self, hist: "ReplayHistory") -> tuple[float, np.ndarray]:
        """The replay of `hist` from the current state: (J, final lattice
        strain q^T e q of every GP)."""
        d = hist.desc()
        J = C.c_double(0.0)
        eq = np.zeros(self.prob.ngps, np.float64)
        self._call("adjoint_forward", C.byref(d), C.byref(J), eq.ctypes.data_as(C.POINTER(C.c_double)))
        return J.value, eq

    def cp_stats(self) -> tuple[np.ndarray, np.ndarray]:
        it = np.zeros(self.prob.ngps, np.int32)
        er = np.zeros(self.prob.ngps, np.float64)
        self._call("get_cp_stats", abi.iptr(it),
                   er.ctypes.data_as(C.POINTER(C.c_double)))
        return it, er


class ReplayHistory:
    """A strain history for the adjoint replay and the objective on its end
    state, in the layouts of ``fas_replay_desc``.

    de [ninc, ngps, 6] strain increments (engineering shears), dr [ninc,
    ngps, 3] spins, dt [ninc] time increments, w / y [ngps] weight and target
    lattice strain of every GP, q the scattering direction, chk_every the
    checkpoint interval of the reverse sweep."""

    def __init__(self, de, dr, dt, w, y, q=(1.0, 0.0, 0.0), chk_every: int = 4):
        f8 = np.float64
        self.de = np.ascontiguousarray(de, f8)
        self.dr = np.ascontiguousarray(dr, f8)
        self.dt = np.ascontiguousarray(dt, f8).reshape(-1)
        self.w = np.ascontiguousarray(w, f8).reshape(-1)
        self.y = np.ascontiguousarray(y, f8).reshape(-1)
        self.q = tuple(float(v) for v in q)
        self.chk_every = int(chk_every)
        ninc, ngps = self.de.shape[0], self.de.shape[1]
        if self.de.shape != (ninc, ngps, 6) or self.dr.shape != (ninc, ngps, 3):
            raise ValueError("de must be [ninc, ngps, 6] and dr [ninc, ngps, 3]")
        if self.dt.shape != (ninc,) or self.w.shape != (ngps,) or self.y.shape != (ngps,):
            raise ValueError("dt must be [ninc], w and y [ngps]")

    @property
    def ninc(self) -> int:
        return int(self.de.shape[0])

    def desc(self) -> abi.FasReplay:
        return abi.FasReplay(self.ninc, self.chk_every, abi.ptr(self.de), abi.ptr(self.dr),
                             abi.ptr(self.dt), abi.ptr(self.w), abi.ptr(self.y),
                             (C.c_double * 3)(*self.q))


class NewtonStepper:
    """The driver loop of src/fasolt/Fasolt3.f90:38-46 advanced one global
    Newton iteration at a time, on any solver with this module's methods
    (the device solver, or the checker's).

    A step is one pass of NRITER's loop body (Stif_sol.f90:32-77), preceded
    by UPDATE_NODE when it opens an increment; when NRITER would stop, the
    step also closes the increment: NRITER's cumslip tail, UPDATE_GPTV and
    DoReorient.  Two solvers stepped from the same state take the same
    sequence of Newton iterations, whatever increments they span."""

    def __init__(self, solver, inc: int = 1):
        self.s = solver
        self.inc = inc
        self.nit = 0
        self.reports: list[dict] = []

    def step(self) -> dict:
        if self.nit == 0:
            self.s.update_node()
        self.nit += 1
        r, more = self.s.nr_step(self.inc, self.nit)
        r = dict(r, inc=self.inc, closes_increment=not more)
        self.reports.append(r)
        if not more:
            self.s.nr_finish(self.inc)
            self.s.update_gptv()
            self.s.do_reorient(self.inc)
            self.inc += 1
            self.nit = 0
        return r


def _report(rep, n) -> list[dict]:
    return [dict(nit=r.nit, sor_sweeps=r.sor_sweeps, sdx=r.sdx, sfc=r.sfc,
                 cp_err=r.cp_err, alp2=r.alp2, sor_error=r.sor_error) for r in rep[:n]]


def _events(ev, n) -> list[dict]:
    return [dict(inc=e.inc, gp=e.gp, sys=e.sys, euler_old=tuple(e.euler_old),
                 euler_new=tuple(e.euler_new)) for e in ev[:n]]


class GpuSolver(_SolverBase):
    """One problem resident on the B200 (state uploaded on construction)."""

    prefix = "fas_gpu"

    def __init__(self, prob: Problem, mode: int = abi.FAS_MODE_PLAIN, upload: bool = True):
        lib = load_library()
        mesh, matl, ctrl = prob.descriptors()
        h = C.c_void_p()
        abi.check(lib.fas_gpu_create(C.byref(mesh), C.byref(matl), C.byref(ctrl),
                                     C.c_uint32(mode), C.byref(h)), "fas_gpu_create")
        super().__init__(lib, prob, h)
        if upload:
            self.upload()

    def adjoint_grad(self, hist: ReplayHistory) -> dict:
        """J of the replay and its gradients: ``st`` [ngps, 6] (starting
        stress), ``sv`` [ngps, FAS_MAXSVS] (starting Euler angles in columns
        0-2, slip resistances from column 3), ``ampar`` [nmatl, 10] (uniform
        shift of ampar(k) over a material's systems; k = 1, 2, 3, 5 filled)."""
        d = hist.desc()
        J = C.c_double(0.0)
        ng = self.prob.ngps
        out = dict(st=np.zeros((ng, 6)), sv=np.zeros((ng, abi.FAS_MAXSVS)),
                   ampar=np.zeros((self.prob.nmatl, 10)))
        dp = C.POINTER(C.c_double)
        self._call("adjoint_grad", C.byref(d), C.byref(J), out["st"].ctypes.data_as(dp),
                   out["sv"].ctypes.data_as(dp), out["ampar"].ctypes.data_as(dp))
        out["J"] = J.value
        return out

    def profile(self, level: int) -> dict:
        """Start device-side profiling (1: counters and region time, 2: also
        per-launch phase times) or stop it (0); returns the counters gathered
        since the last start."""
        out = abi.FasProfile()
        self._call("profile", int(level), C.byref(out))
        return out.as_dict()

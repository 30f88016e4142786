"""ctypes mirror of ``include/fasolt_gpu.h``.

The structures below are byte-for-byte the C descriptors, so a
:class:`~cpfem_code_b200.problem.Problem` can be handed to the device library
(and to the CPU checker, which takes the same descriptors) without copies.
Arrays in :class:`Problem` are C-ordered with their axes reversed relative to
the Fortran declarations in ``src/fasolt/fas-com-mod.f90``, which gives the
identical memory layout: Fortran ``ln(8, nlmnt)`` is numpy ``ln[nlmnt, 8]``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

FAS_OK = 0
FAS_E_ARG = -1
FAS_E_NODEVICE = -2
FAS_E_CUDA = -3
FAS_E_ELTYPE = -4
FAS_E_NOMEM = -5
FAS_E_RANGE = -6
FAS_E_STATE = -7
FAS_E_TIMEOUT = -8
FAS_MAXSS = 60
FAS_MAXSVS = 63    # leading dimension of the adjoint's g_sv
SVLD = 63          # maxsvs, src/fasolt/fas-com-mod.f90:14
XSLD = 99          # second dimension of x_spec / f_spec (fas-com-mod.f90:30-31)

FAS_MODE_PLAIN = 0
FAS_MODE_SOR_FP32 = 1
FAS_MODE_SOR_NATURAL = 2
FAS_MODE_SOR_GRID = 4
FAS_MODE_CP_WARP = 8
FAS_MODE_SOR_TILES = 16
FAS_MODE_TANGENT_CONSISTENT = 32
FAS_MODE_CP_QUEUE = 64
FAS_MODE_GRAPH = 128
FAS_MODE_SOR_SYM = 256

#: FAFERR codes the hot path raises, with the reference's meaning.
FAFERR_TEXT = {
    903: "zero diagonal in SOR (Stif_sol.f90:184)",
    904: "SOR did not converge (Stif_sol.f90:213)",
    905: "rotation increment too large (Sig_eps.f90:58)",
    906: "strain increment too large (Sig_eps.f90:59)",
    910: "singular local Jacobian (Cpstrs.f90:102,123; crys-cons.f90:66)",
    920: "element weight below 1e-7 (Elvals.f90:103)",
    955: "stiffness row overflow (Stif_sol.f90:134)",
    987: "slip Newton error above 0.5 (crys-cons.f90:108)",
}
ABI_TEXT = {
    FAS_E_ARG: "invalid argument",
    FAS_E_NODEVICE: "no sm_100 (B200) CUDA device visible",
    FAS_E_CUDA: "CUDA runtime error",
    FAS_E_ELTYPE: "element type not implemented (only lt=12 bricks and ties)",
    FAS_E_NOMEM: "device allocation failed",
    FAS_E_RANGE: "size beyond a documented maximum",
    FAS_E_STATE: "call out of order (state not uploaded)",
    FAS_E_TIMEOUT: "a bounded device-side wait gave up (copy engine stalled)",
}

_p = C.c_void_p
_i32p = C.POINTER(C.c_int32)


class FasMesh(C.Structure):
    _fields_ = [("nlmnt", C.c_int32), ("nnod", C.c_int32), ("ngps", C.c_int32),
                ("le", _i32p), ("lt", _i32p), ("nd", _i32p), ("np", _i32p),
                ("ln", _i32p), ("ld_ln", C.c_int32),
                ("lg", _i32p), ("ld_lg", C.c_int32),
                ("ib", _i32p)]


class FasMatl(C.Structure):
    _fields_ = [("real_bytes", C.c_int32), ("nmatl", C.c_int32), ("nmpar", C.c_int32),
                ("ld_ss", C.c_int32), ("nss", _i32p),
                ("e", _p), ("ssang", _p), ("ab", _p), ("an", _p), ("ampar", _p),
                ("smatrx", _p), ("twinlim", C.c_int32), ("twinprob", C.c_double)]


class FasCtrl(C.Structure):
    _fields_ = [("real_bytes", C.c_int32), ("maxit", C.c_int32),
                ("toler", C.c_double), ("alpha", C.c_double), ("afactor", C.c_double),
                ("efix", C.c_double), ("smale", C.c_double), ("smalr", C.c_double),
                ("ninc1", C.c_int32), ("nxs", C.c_int32), ("nfs", C.c_int32),
                ("ld_xs", C.c_int32), ("tiem", _p), ("x_spec", _p), ("f_spec", _p),
                ("twin_seed", C.c_uint64)]


class FasState(C.Structure):
    _fields_ = [("real_bytes", C.c_int32), ("nsv", C.c_int32), ("ld_sv", C.c_int32),
                ("ld_slip", C.c_int32),
                ("x", _p), ("dx", _p), ("fc", _p), ("ddx", _p),
                ("eps", _p), ("dep", _p),
                ("st", _p), ("ep", _p), ("ds", _p), ("de", _p),
                ("rt", _p), ("dr", _p), ("sv", _p), ("dsv", _p),
                ("timestwinned", _i32p), ("twinsys", _i32p),
                ("srate", _p), ("cumslip", _p)]


class FasIterReport(C.Structure):
    _fields_ = [("nit", C.c_int32), ("sor_sweeps", C.c_int32),
                ("sdx", C.c_double), ("sfc", C.c_double), ("cp_err", C.c_double),
                ("alp2", C.c_double), ("sor_error", C.c_double)]


class FasProfile(C.Structure):
    _fields_ = [("ms_constitutive", C.c_double), ("ms_assembly", C.c_double),
                ("ms_sor_colour", C.c_double), ("ms_total", C.c_double),
                ("n_constitutive", C.c_int64), ("n_assembly", C.c_int64),
                ("n_sor_colour", C.c_int64), ("n_launches", C.c_int64),
                ("gp_updates", C.c_int64), ("sor_sweeps", C.c_int64),
                ("sor_bytes", C.c_double), ("assembly_bytes", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class FasReplay(C.Structure):
    _fields_ = [("ninc", C.c_int32), ("chk_every", C.c_int32),
                ("de", _p), ("dr", _p), ("dt", _p), ("w", _p), ("y", _p),
                ("q", C.c_double * 3)]


class FasTwinEvent(C.Structure):
    _fields_ = [("inc", C.c_int32), ("gp", C.c_int32), ("sys", C.c_int32), ("pad", C.c_int32),
                ("euler_old", C.c_double * 3), ("euler_new", C.c_double * 3)]


def ptr(a: np.ndarray | None):
    """Raw data pointer of a contiguous numpy array (None -> NULL)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "descriptor arrays must be C-contiguous"
    return a.ctypes.data


def iptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_i32p)


class FasError(RuntimeError):
    """A non-zero status from the C ABI.  ``code`` > 0 is the reference's
    FAFERR code (the Fortran driver would call FAFERR(code)); < 0 is an ABI
    error."""

    def __init__(self, code: int, where: str):
        self.code = int(code)
        text = FAFERR_TEXT.get(code) or ABI_TEXT.get(code) or "unknown status"
        kind = "FAFERR" if code > 0 else "ABI error"
        super().__init__(f"{where}: {kind} {code}: {text}")


def check(code: int, where: str) -> int:
    if code != 0:
        raise FasError(code, where)
    return 0


def declare(lib: C.CDLL, prefix: str) -> None:
    """Declare argument / result types of every entry point of a library
    exporting ``<prefix>_*`` with the signatures of fasolt_gpu.h."""
    H = _p
    i32 = C.c_int32
    sig = {
        "create": (i32, [C.POINTER(FasMesh), C.POINTER(FasMatl), C.POINTER(FasCtrl)]),
        "destroy": (None, [H]),
        "set_mode": (i32, [H, C.c_uint32]),
        "upload_state": (i32, [H, C.POINTER(FasState)]),
        "download_state": (i32, [H, C.POINTER(FasState)]),
        "update_node": (i32, [H]),
        "elvals": (i32, [H, i32, i32]),
        "suvals": (i32, [H, i32]),
        "facsls": (i32, [H, _i32p, C.POINTER(C.c_double)]),
        "nriter": (i32, [H, i32, C.POINTER(FasIterReport), i32, _i32p]),
        "nr_step": (i32, [H, i32, i32, C.POINTER(FasIterReport), _i32p]),
        "nr_finish": (i32, [H, i32]),
        "update_gptv": (i32, [H]),
        "reorient": (i32, [H, i32, C.POINTER(FasTwinEvent), i32, _i32p]),
        "increment": (i32, [H, i32, C.POINTER(FasIterReport), i32, _i32p,
                            C.POINTER(FasTwinEvent), i32, _i32p]),
        "get_pattern": (i32, [H, _i32p, i32]),
        "get_stiffness": (i32, [H, _p, i32, i32]),
        "get_colouring": (i32, [H, _i32p, _i32p]),
        "constitutive": (i32, [H, i32, i32]),
        "get_tangent": (i32, [H, _p, i32]),
        "get_cp_stats": (i32, [H, _i32p, C.POINTER(C.c_double)]),
        "get_cp_ops": (i32, [H, C.POINTER(C.c_double)]),
        "lattice_strain": (i32, [H, _p, i32]) if prefix == "fas_gpu" else (i32, [H, _p]),
    }
    _dp = C.POINTER(C.c_double)
    sig["adjoint_forward"] = (i32, [H, C.POINTER(FasReplay), _dp, _dp])
    if prefix == "fas_gpu":
        sig["profile"] = (i32, [H, i32, C.POINTER(FasProfile)])
        sig["adjoint_grad"] = (i32, [H, C.POINTER(FasReplay), _dp, _dp, _dp, _dp])
    for name, (res, args) in sig.items():
        fn = getattr(lib, f"{prefix}_{name}")
        fn.restype = res
        if name == "create":
            if prefix == "ora":
                args = args + [i32, C.c_uint32, C.POINTER(H)]
            else:
                args = args + [C.c_uint32, C.POINTER(H)]
        fn.argtypes = args

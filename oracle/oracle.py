"""ctypes wrapper of libfasolt_oracle.so (TEST INFRASTRUCTURE ONLY).

:class:`OracleSolver` has the same methods as the device solver, so a test
can run one problem through both and compare.  ``real_bytes=8`` is the
reference promoted to double, ``real_bytes=4`` the FP32-faithful form.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

from cpfem_code_b200 import abi
from cpfem_code_b200.problem import Problem
from cpfem_code_b200.solver import _SolverBase

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfasolt_oracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compile the checker with oracle/Makefile (g++, no GPU needed)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    else:
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return LIB_PATH


def _load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = C.CDLL(LIB_PATH)
        abi.declare(lib, "ora")
        lib.ora_set_threads.argtypes = [C.c_void_p, C.c_int32]
        lib.ora_set_threads.restype = C.c_int32
        lib.ora_facsls_limited.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_int32),
                                           C.POINTER(C.c_double)]
        lib.ora_facsls_limited.restype = C.c_int32
        for name, args, res in (
                ("ora_spower", [C.c_double, C.c_double], C.c_double),
                ("ora_fj2vom", [C.c_int32, C.POINTER(C.c_double)], C.c_double),
                ("ora_factor_solve", [C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)], C.c_int32),
                ("ora_ctmatrx", [C.c_double] * 3 + [C.POINTER(C.c_double)] * 2, None),
                ("ora_elastc", [C.POINTER(C.c_double)] * 3, None),
                ("ora_tens_rot", [C.POINTER(C.c_double)] * 3, None),
                ("ora_shape12", [C.POINTER(C.c_double)] * 2, C.c_double),
                ("ora_shape22", [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)], C.c_double),
                ("ora_shape22_table", [C.POINTER(C.c_double)], None),
                ("ora_shape_elem", [C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)], C.c_double),
                ("ora_shape21_table", [C.POINTER(C.c_double)], None),
                ("ora_shape23_table", [C.POINTER(C.c_double)], None)):
            f = getattr(lib, name)
            f.argtypes, f.restype = args, res
        _lib = lib
    return _lib


def lib() -> C.CDLL:
    return _load()


class OracleSolver(_SolverBase):
    prefix = "ora"

    def __init__(self, prob: Problem, real_bytes: int = 8, mode: int = 0,
                 threads: int = 1, upload: bool = True):
        L = _load()
        mesh, matl, ctrl = prob.descriptors()
        h = C.c_void_p()
        abi.check(L.ora_create(C.byref(mesh), C.byref(matl), C.byref(ctrl), real_bytes,
                               C.c_uint32(mode), C.byref(h)), "ora_create")
        super().__init__(L, prob, h)
        self.real_bytes = real_bytes
        L.ora_set_threads(self._h, threads)
        if upload:
            self.upload()

    def set_threads(self, n: int) -> None:
        self._lib.ora_set_threads(self._h, n)

    def facsls_limited(self, max_sweeps: int):
        s, e = C.c_int32(0), C.c_double(0.0)
        rc = self._lib.ora_facsls_limited(self._h, max_sweeps, C.byref(s), C.byref(e))
        return rc, s.value, e.value


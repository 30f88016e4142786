"""fas_gpu_facsls_noalloc against fas_gpu_facsls on the same assembled system.

fas_gpu_facsls_noalloc is the FACSLS entry point for drivers that must not
allocate device memory after set-up: its scratch is a static device array of
the library, and the call allocates nothing.  Both calls go through the C
ABI.  They run the same kernels in the same order, so the solutions agree to
rounding (RTOL) and the sweep counts are equal.  Each case makes two calls in
a row.  The second call solves with the first call's solution as its
right-hand side, because FACSLS moves ddx into the right-hand side; this also
checks that the shared control words are reset between calls.  The
allocation-free property itself is checked on a fresh handle that has never
solved: the device's free memory (cudaMemGetInfo) is the same before and
after each of two calls.  The file name sorts last, so the test also runs
after every other test in the same process; it passes when run alone as
well.
"""
import ctypes as C

import numpy as np
import pytest

from cpfem_code_b200 import GpuSolver, abi, generator
from cpfem_code_b200.solver import load_library

pytestmark = pytest.mark.gpu
RTOL = 1e-12


def _facsls_noalloc(g: GpuSolver) -> tuple[int, float]:
    fn = load_library().fas_gpu_facsls_noalloc
    fn.restype = C.c_int32
    fn.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_double)]
    sweeps, err = C.c_int32(0), C.c_double(0.0)
    abi.check(fn(g._h, C.byref(sweeps), C.byref(err)), "fas_gpu_facsls_noalloc")
    return sweeps.value, err.value


def _assembled(p, mode):
    g = GpuSolver(p.copy(), mode=mode)
    g.update_node()
    g.elvals(1, 1)
    g.suvals(1)
    return g


CASES = [((4, 4, 4), abi.FAS_MODE_PLAIN, 8),      # one-CTA solve
         ((24, 24, 24), abi.FAS_MODE_PLAIN, 8),   # colour kernels, 15,625 nodes
         ((8, 8, 8), abi.FAS_MODE_SOR_GRID, 8),   # colour kernels forced
         ((3, 3, 3), abi.FAS_MODE_PLAIN, 20),     # 81-slot rows, one CTA
         ((3, 3, 3), abi.FAS_MODE_SOR_GRID, 20),  # 81-slot colour kernels
         ((12, 12, 12), abi.FAS_MODE_PLAIN, 20),  # 81-slot colour kernels, 8,281 nodes
         ((32, 32, 32), abi.FAS_MODE_PLAIN, 20)]  # the brick20_32 workload: the most partials benchmarked


@pytest.mark.parametrize("n,mode,nodes", CASES)
def test_facsls_noalloc_matches_facsls(n, mode, nodes):
    p = generator.structured_cube(n=n, ninc=1, seed=7, nodes=nodes)
    g = _assembled(p, mode)
    try:
        start = g.download(p.copy())           # assembled right-hand side in ddx
        ref = []
        for _ in range(2):
            sweeps, _ = g.facsls()
            ref.append((sweeps, g.download(p.copy()).ddx.copy()))
        g.upload(start)                        # the same right-hand side; the matrix stays
        for k in range(2):
            sweeps, _ = _facsls_noalloc(g)
            ddx = g.download(p.copy()).ddx
            assert sweeps == ref[k][0]
            scale = np.abs(ref[k][1]).max()
            assert scale > 0
            assert np.abs(ddx - ref[k][1]).max() <= RTOL * scale
    finally:
        g.close()


@pytest.mark.parametrize("n,mode,nodes", [((24, 24, 24), abi.FAS_MODE_PLAIN, 8),
                                          ((3, 3, 3), abi.FAS_MODE_SOR_GRID, 20)])
def test_facsls_noalloc_allocates_nothing(n, mode, nodes):
    """A handle that has never solved (no CUDA graph, no lazily sized
    buffer yet): free device memory is unchanged by each of two calls, and
    the results equal fas_gpu_facsls's on a second handle."""
    import torch
    p = generator.structured_cube(n=n, ninc=1, seed=7, nodes=nodes)
    g, r = _assembled(p, mode), _assembled(p, mode)
    try:
        torch.cuda.synchronize()
        for _ in range(2):
            free0 = torch.cuda.mem_get_info()[0]
            sweeps, _ = _facsls_noalloc(g)
            torch.cuda.synchronize()
            assert torch.cuda.mem_get_info()[0] == free0
            ref_sweeps, _ = r.facsls()
            assert sweeps == ref_sweeps
            a, b = g.download(p.copy()).ddx, r.download(p.copy()).ddx
            assert np.abs(a - b).max() <= RTOL * np.abs(b).max()
    finally:
        g.close()
        r.close()

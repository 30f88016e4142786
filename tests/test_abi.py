"""The C ABI library loads and exports every entry point include/*.h
declares; without a B200 it refuses to create a problem (no CPU fallback)."""
import ctypes as C
import glob
import os
import re

import pytest

from cpfem_code_b200 import abi, build, generator
from cpfem_code_b200.solver import LIB_PATH, load_library

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        names |= set(re.findall(r"^FAS_API\s+\w+\s*\*?\s*(fas_gpu_\w+)\s*\(", open(h).read(), re.M))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "fas_gpu_create" in names and "fas_gpu_nriter" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    build.build()
    lib = C.CDLL(LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_ctypes_structs_match_header_layout(tmp_path):
    """Compile the header with the C compiler and compare every descriptor's
    size with its ctypes mirror."""
    import subprocess
    pairs = {"fas_mesh_desc": abi.FasMesh, "fas_matl_desc": abi.FasMatl,
             "fas_ctrl_desc": abi.FasCtrl, "fas_state_desc": abi.FasState,
             "fas_iter_report": abi.FasIterReport, "fas_twin_event": abi.FasTwinEvent,
             "fas_profile": abi.FasProfile}
    src = tmp_path / "sz.c"
    src.write_text('#include <stdio.h>\n#include "fasolt_gpu.h"\nint main(void){\n' +
                   "".join(f'printf("{k} %zu\\n", sizeof({k}));\n' for k in pairs) + "return 0;}\n")
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    got = dict(zip(out[0::2], map(int, out[1::2])))
    for k, cls in pairs.items():
        assert got[k] == C.sizeof(cls), k


def _has_cuda_device():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_cuda_device(), reason="a GPU is visible")
def test_create_without_device_fails_loudly():
    load_library()
    p = generator.point_batch(8)
    from cpfem_code_b200 import GpuSolver
    with pytest.raises(abi.FasError) as ei:
        GpuSolver(p)
    assert ei.value.code == abi.FAS_E_NODEVICE


def test_python_constants_match_header():
    """Every FAS_MODE_*, FAS_E_* and FAS_MAX* value of the header equals its
    name in cpfem_code_b200.abi."""
    text = open(os.path.join(ROOT, "include", "fasolt_gpu.h")).read()
    found = re.findall(r"^#define\s+(FAS_(?:MODE|E|MAX)\w*)\s+\(?(-?\d+)u?\)?", text, re.M)
    assert len(found) >= 15
    for name, val in found:
        if hasattr(abi, name):
            assert getattr(abi, name) == int(val), name
    for name, _ in found:
        if name.startswith("FAS_MODE_"):
            assert hasattr(abi, name), f"{name} has no Python mirror"

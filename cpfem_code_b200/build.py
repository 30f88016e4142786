"""Build ``cpfem_code_b200/lib/libfasgpu.so`` for sm_100a with nvcc.

``python -m cpfem_code_b200.build [--verbose]``.  The library is built in the
source tree so that it travels with the checkout; nvcc cross-compiles, so no
GPU is needed to build.  The launch shapes and scheduling options come from
``tuned.json`` (written by ``cpfem_code_b200.autotune``) when it exists, else
from the defaults in the sources.
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "lib", "libfasgpu.so")
SOURCES = ["fas_capi.cu"]
DEPS = ["fas_capi.cu", "fas_kernels.cuh", "fas_sor_tiles.cuh", "fas_device_warp.cuh", "fas_adjoint.cuh", "fas_device.cuh", "fas_flops.h", "fas_rng.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
TUNED = os.path.join(HERE, "tuned.json")


def tuned_defines() -> dict:
    """The autotuner's choice of compile-time defines (empty without tuned.json)."""
    if not os.path.exists(TUNED):
        return {}
    with open(TUNED) as f:
        return dict(json.load(f)["defines"])


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    hdr = os.path.join(HERE, "..", "include", "fasolt_gpu.h")
    deps = [os.path.join(SRC, d) for d in DEPS] + [hdr] + ([TUNED] if os.path.exists(TUNED) else [])
    return any(os.path.getmtime(p) > t for p in deps)


def build(force: bool = False, verbose: bool = False, defines: dict | None = None,
          out: str | None = None) -> str:
    """Compile the library (when stale, or always with `force`) with the
    tuned defines, or `defines` instead, into `out` (default: the library)."""
    out = out or OUT
    if out == OUT and not force and not _stale():
        return OUT
    os.makedirs(os.path.dirname(out), exist_ok=True)
    defs = tuned_defines() if defines is None else defines
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
           *[f"-D{k}={v}" for k, v in sorted(defs.items())],
           "-o", out + ".tmp", *[os.path.join(SRC, s) for s in SOURCES]]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed")
    if verbose:
        sys.stderr.write(res.stderr)
    os.replace(out + ".tmp", out)
    return out


if __name__ == "__main__":
    print(build(force=True, verbose="--verbose" in sys.argv))

"""Autotuner of the kernels' launch shapes and scheduling options.

Every knob is a set of compile-time defines, tuned on the workload whose
time it sets:

* ``sor27``: ``FAS_TMA_ROWS``, ``FAS_TMA_LPR``, ``FAS_TMA_STAGES`` (rows per
  chunk, lanes per row, ring stages of the 27-slot SOR colour kernel),
  timed by the FACSLS of the 64^3 cube's first Newton iteration;
* ``sor81``: ``FAS_TMA_ROWS81``, ``FAS_TMA_LPR81`` (the 81-slot kernel), timed
  by the FACSLS of 32^3 20-node bricks;
* ``cp``: ``FAS_WORK_DESC``, ``FAS_CP_QUEUE`` (order and device queue of the
  constitutive pass), timed by the element pass of the mixed FCC/HCP 32^3
  cube and the 2^20-point batch (geometric mean of the two ratios);
* ``sor27f32``: ``FAS_TMA_ROWS32``, ``FAS_TMA_LPR32``, ``FAS_TMA_MINB32``
  (rows per chunk, lanes per row and the CTAs per SM the register budget
  must allow, of the tuned form's FP32-matrix colour kernel), timed by the
  FP32 FACSLS of the 64^3 cube's first Newton iteration;
* ``sor81f32``: ``FAS_TMA_ROWS81_32``, ``FAS_TMA_LPR81_32`` (the FP32-matrix
  colour kernel of 81-slot rows), timed by the FP32 FACSLS of 32^3 20-node
  bricks.

The knobs act on different kernels, so library i carries candidate i of
every knob (a knob with fewer candidates repeats its last one), and one
measurement per library times every knob at once.  Builds need no GPU;
measuring does.

    python -m cpfem_code_b200.autotune build     # nvcc: lib/tune/lib_<i>.so
    python -m cpfem_code_b200.autotune measure   # on a B200: lib/tune/measure.json
    python -m cpfem_code_b200.autotune select    # tuned.json, read by build.py
"""
from __future__ import annotations

import concurrent.futures as cf
import ctypes as C
import json
import math
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
TUNE_DIR = os.path.join(HERE, "lib", "tune")
MEASURE = os.path.join(TUNE_DIR, "measure.json")
TUNED = os.path.join(HERE, "tuned.json")

KNOBS = {
    "sor27": [dict(FAS_TMA_ROWS=r, FAS_TMA_LPR=l, FAS_TMA_STAGES=st)
              for r, l, st in ((8, 4, 2), (16, 4, 2), (8, 8, 2), (8, 4, 3), (16, 8, 2))],
    "sor81": [dict(FAS_TMA_ROWS81=r, FAS_TMA_LPR81=l) for r, l in ((8, 16), (4, 16), (8, 8), (4, 32), (16, 8))],
    "cp": [dict(FAS_WORK_DESC=d, FAS_CP_QUEUE=q) for d, q in ((1, 1), (1, 0), (0, 1), (0, 0))],
    "sor27f32": [dict(FAS_TMA_ROWS32=r, FAS_TMA_LPR32=l, FAS_TMA_MINB32=m)
                 for r, l, m in ((24, 4, 1), (16, 4, 1), (32, 4, 1), (16, 8, 1), (8, 4, 1), (16, 4, 6))],
    "sor81f32": [dict(FAS_TMA_ROWS81_32=r, FAS_TMA_LPR81_32=l)
                 for r, l in ((4, 16), (8, 16), (8, 8), (4, 32), (2, 16), (16, 8))],
}


def n_libs() -> int:
    return max(len(c) for c in KNOBS.values())


def defines_of(i: int) -> dict:
    out = {}
    for cands in KNOBS.values():
        out.update(cands[min(i, len(cands) - 1)])
    return out


def lib_path(i: int) -> str:
    return os.path.join(TUNE_DIR, f"lib_{i}.so")


def build_all(jobs: int = 4) -> list[str]:
    from . import build as B
    os.makedirs(TUNE_DIR, exist_ok=True)
    with cf.ThreadPoolExecutor(jobs) as ex:
        futs = [ex.submit(B.build, True, False, defines_of(i), lib_path(i)) for i in range(n_libs())]
        return [f.result() for f in futs]


def _load(path: str):
    from . import abi, solver
    lib = C.CDLL(path)
    abi.declare(lib, "fas_gpu")
    solver._lib = lib


def _median(xs):
    xs = sorted(xs)
    return xs[len(xs) // 2]


def _solve_us(p, reps: int = 3, mode: int = 0) -> tuple[float, int]:
    """us per sweep of the FACSLS of the first Newton iteration (graphs and
    programmatic launches as the increments run it), in `mode`."""
    from .solver import GpuSolver
    g = GpuSolver(p.copy(), mode=mode)
    try:
        g.update_node()
        g.elvals(1, 1)
        g.suvals(1)
        start = g.download(p.copy()).copy()
        ts, sweeps = [], 0
        for _ in range(reps + 1):
            g.upload(start)
            g.profile(1)
            sweeps, _ = g.facsls()
            ts.append(g.profile(0)["ms_total"] * 1e3 / sweeps)
        return _median(ts[1:]), sweeps
    finally:
        g.close()


def _cp_ms(p, points: bool, reps: int = 5) -> float:
    """Constitutive-pass time: fas_gpu_constitutive on a point batch, or the
    element pass of ELVALS after one increment."""
    from .solver import GpuSolver
    g = GpuSolver(p.copy())
    try:
        if points:
            g.constitutive(1, 1)
        else:
            g.increment(1)
            g.update_node()
            g.elvals(2, 1)
        ts = []
        for _ in range(reps):
            if points:
                g.upload(p)
            g.profile(2)
            if points:
                g.constitutive(1, 1)
            else:
                g.elvals(2, 1)
            ts.append(g.profile(0)["ms_constitutive"])
        return _median(ts)
    finally:
        g.close()


def measure() -> dict:
    from . import generator
    probs = dict(cube64=generator.workload("cube64"), brick20_32=generator.workload("brick20_32"),
                 mixed32=generator.workload("mixed32"), points=generator.point_batch(1 << 20, seed=1))
    out = {}
    for i in range(n_libs()):
        _load(lib_path(i))
        try:
            us27, sw27 = _solve_us(probs["cube64"])
        except Exception as e:   # a combination the device refuses (e.g. a ring above its shared memory)
            out[str(i)] = dict(defines=defines_of(i), error=str(e))
            print(json.dumps(out[str(i)]), flush=True)
            continue
        us81, sw81 = _solve_us(probs["brick20_32"])
        us32, sw32 = _solve_us(probs["cube64"], mode=1)   # FAS_MODE_SOR_FP32
        us8132, sw8132 = _solve_us(probs["brick20_32"], mode=1)
        out[str(i)] = dict(defines=defines_of(i), cube64_sweep_us=us27, cube64_sweeps=sw27,
                           brick20_32_sweep_us=us81, brick20_32_sweeps=sw81,
                           cube64_fp32_sweep_us=us32, cube64_fp32_sweeps=sw32,
                           brick20_32_fp32_sweep_us=us8132, brick20_32_fp32_sweeps=sw8132,
                           mixed32_cp_ms=_cp_ms(probs["mixed32"], False),
                           points_cp_ms=_cp_ms(probs["points"], True))
        print(json.dumps(out[str(i)]), flush=True)
    os.makedirs(TUNE_DIR, exist_ok=True)
    with open(MEASURE, "w") as f:
        json.dump(out, f, indent=1)
    return out


def select(meas: dict | None = None, out: str = TUNED) -> dict:
    """Best candidate of every knob from the measurements, written to `out`."""
    if meas is None:
        with open(MEASURE) as f:
            meas = json.load(f)
    rows = [meas[str(i)] for i in range(n_libs())]
    inf = float("inf")
    ref = next(r for r in rows if "error" not in r)
    score = {
        "sor27": lambda r: r["cube64_sweep_us"],
        "sor81": lambda r: r["brick20_32_sweep_us"],
        "sor27f32": lambda r: r["cube64_fp32_sweep_us"],
        "sor81f32": lambda r: r.get("brick20_32_fp32_sweep_us", r["brick20_32_sweep_us"]),
        "cp": lambda r: math.sqrt(r["mixed32_cp_ms"] / ref["mixed32_cp_ms"]
                                  * r["points_cp_ms"] / ref["points_cp_ms"]),
    }
    # sweep counts do not depend on a launch shape; a candidate that changed
    # them would be wrong, not fast
    ok = [r for r in rows if "error" not in r]
    for key in ("cube64_sweeps", "brick20_32_sweeps", "cube64_fp32_sweeps", "brick20_32_fp32_sweeps"):
        assert len({r.get(key) for r in ok}) == 1, f"{key} differ between candidates"
    tuned = {"defines": {}, "measured": {}}
    for knob, cands in KNOBS.items():
        vals = [inf if "error" in rows[i] else score[knob](rows[i]) for i in range(len(cands))]
        best = min(range(len(cands)), key=lambda i: vals[i])
        tuned["defines"].update(cands[best])
        tuned["measured"][knob] = [dict(defines=cands[i], score=vals[i]) for i in range(len(cands))]
    with open(out, "w") as f:
        json.dump(tuned, f, indent=1)
        f.write("\n")
    return tuned


def main(argv: list[str]) -> int:
    step = argv[0] if argv else ""
    if step == "build":
        for p in build_all():
            print(p)
    elif step == "measure":
        measure()
    elif step == "select":
        print(json.dumps(select()["defines"]))
    else:
        print(__doc__)
        return 2
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))

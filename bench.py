#!/usr/bin/env python
"""Benchmark of the FASOLT3 increment hot path on B200.

Workload (default): the 64^3 FCC aluminium cube (262,144 one-point bricks =
GPs, 274,625 nodes, 823,875 DOF), grains of 2^3 elements with seeded
uniform-SO(3) orientations, uniaxial tension at 1e-3 strain per increment.

A *step* is one global Newton iteration of the driver loop
(src/fasolt/Fasolt3.f90:38-46): one pass of NRITER's loop body -- ELVALS,
SUVALS, the residual norm, FACSLS, the damped correction
(src/fasolt/Stif_sol.f90:32-77) -- opened by UPDATE_NODE at the start of an
increment and closed, when NRITER stops, by its cumslip tail, UPDATE_GPTV
and DoReorient.  Both arms take the SAME steps: the first K Newton
iterations of the run from the generated initial state.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload cube64|brick20_32|mixed32|brick20_10|points]

Metric: Gauss-point updates per second -- one DSTRSS evaluation of one GP in
one global Newton iteration -- over whole Newton iterations, i.e. ngps * K /
time.  `value`: device time of the K steps with the state resident in HBM
(CUDA events on the library's stream), after W warm-up steps that are then
discarded (the state is re-uploaded).  `e2e`: the same K steps through the C
ABI with the whole state copied from pinned host memory before and back
after every step.  `increments`: seconds per increment of whole increments
(plain FP64 against the tuned FP32-sweep form).  `oracle_error`: the device
path against the checker after the first CPU_STEPS steps at full size.

N > 1 (torchrun): independent replicas, one per GPU (the path is one
problem on one GPU); time is the max over ranks, value the sum of work.
`--impl reference` times the CPU restatement of the reference (oracle/) on
all host cores over the same K steps from the same initial state.

`--workload points` is the constitutive micro-benchmark (2^20 independent
FCC points): a step is one DSTRSS pass over every point.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "cube64"
# workload: (metric, description)
WORKLOADS = {
    "cube64": ("GP updates/s at 64^3 (DSTRSS evaluations per second of whole Newton iterations)",
               "64^3 FCC Al one-point bricks (262,144 GPs, 823,875 DOF), 2^3-element grains, "
               "uniaxial tension 1e-3 per increment"),
    "brick20_32": ("GP updates/s, 32^3 20-node bricks (DSTRSS evaluations per second of whole Newton iterations)",
                   "32^3 FCC Al 20-node eight-GP bricks (262,144 GPs, 421,443 DOF), 2^3-element grains, "
                   "uniaxial tension 1e-3 per increment"),
    "mixed32": ("GP updates/s, 32^3 mixed FCC/HCP (DSTRSS evaluations per second of whole Newton iterations)",
                "32^3 one-point bricks (32,768 GPs), 50/50 random HCP-Zr (30 systems incl. twins) / FCC-Al grains "
                "of 2^3 elements, uniaxial tension 1e-3 per increment"),
    "brick20_10": ("GP updates/s, 10^3 20-node bricks (DSTRSS evaluations per second of whole Newton iterations)",
                   "10^3 FCC Al 20-node eight-GP bricks (the reference sample's mesh: 8,000 GPs), "
                   "one grain per element, uniaxial tension 1e-3 per increment"),
    "diff16": ("GP-increments/s of the adjoint gradient, 16^3 FCC cube, 20 increments (replay and reverse sweep)",
               "16^3 FCC Al one-point bricks (4,096 GPs), one grain per element, 20 increments to 2 % tension; "
               "lattice-strain objective over 8 {hkl} orientation bins along the load axis; gradients with "
               "respect to h0, tau_sat, the rate exponent, the initial CRSS and all Euler angles; "
               "checkpoints every 5 increments"),
    "points": ("GP updates/s, 2^20 independent FCC points (DSTRSS evaluations per second)",
               "2^20 FCC Al material points, uniform-SO(3) orientations, Gaussian strain increments of "
               "Frobenius norm 1e-3, CRSS uniform in [tau0, 2 tau0], elastic-predictor start"),
}
METRIC, DESC = WORKLOADS[WORKLOAD]
# DRAM bytes (read + write) per FP64 colour launch at 64^3, measured with ncu
# on two launches of the profiling case and scaled per row to the mean colour
SOR_TRAFFIC_PER_LAUNCH = 81.1e6
# the same for the FP32-matrix colour kernel (profiles/k_sor_colour_tma_fp32_cube64.md)
SOR32_TRAFFIC_PER_LAUNCH = 47.3e6
CPU_STEPS = 2          # steps of the full-size checker run (cpu_baseline and oracle_error)
INC_WARM, INC_TIMED = 5, 10   # increments leg: untimed increments, then timed ones
POINTS = 1 << 20
# the tuned form: FP32-matrix sweeps with FP64 residual refinement
# (abi.FAS_MODE_SOR_FP32).  The persistent tile solve and the consistent
# tangent are measured beside it (rooflines.sor_*tiles,
# increments.plain_consistent_tangent) and left out: neither is faster, and
# the tangent moves per-point stresses by up to toler's reach.
TUNED_MODE = 1
POINTS_CPU = 1 << 15   # points of the checker's bounded sample in the point workload


def peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return dict(hbm_gbs=float(d["hbm_gbs"]), source="measured")
    except Exception:
        return dict(hbm_gbs=6650.0, source="fallback")


def fp64_peak_tflops() -> dict:
    """FP64 throughput of this GPU, measured: torch.matmul in float64 (cuBLAS
    DGEMM) on 8192^3, best of 5 by CUDA events.  The constitutive kernel's
    FP64 roofline divides by it (no FP64 figure is in MEASURED_PEAKS.json)."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return dict(tflops=2.0 * n ** 3 / best / 1e12, source="measured: torch.matmul float64 8192^3, best of 5")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return dict(sm_mhz=None, sm_max_mhz=None, reasons=["nvidia-smi unavailable"])
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for k, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(k)
        return dict(sm_mhz=float(np.median(sm)) if sm else None,
                    sm_max_mhz=float(max(smax)) if smax else None,
                    reasons=sorted(reasons), samples=len(sm))


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def init_dist(ws: int, backend: str):
    if ws <= 1:
        return None
    import datetime

    import torch.distributed as dist
    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=600))
    return dist


def reduce_max_sum(dist, t: float, work: float, device=None):
    """(max of t, sum of work) over ranks -- the only collective of the
    benchmark (replicas share nothing on the data path)."""
    if dist is None:
        return t, work
    import torch
    a = torch.tensor([t], dtype=torch.float64, device=device)
    b = torch.tensor([work], dtype=torch.float64, device=device)
    dist.all_reduce(a, op=dist.ReduceOp.MAX)
    dist.all_reduce(b, op=dist.ReduceOp.SUM)
    return float(a.item()), float(b.item())


L2_BYTES = 126e6


def l2_note(prob) -> str:
    """Whether the SOR block matrix (FP64 values and column ids, the bytes
    every sweep re-reads) exceeds the 126 MB L2."""
    slots = 81 if int(prob.nd.max(initial=8)) == 20 else 27
    rows = prob.nnod
    mb = rows * ((9 * slots + 3) // 4 * 4 * 8 + (slots + 4) // 4 * 4 * 4) / 1e6
    if mb * 1e6 > L2_BYTES:
        return f"inputs larger than L2 ({mb:.0f} MB block matrix re-read every sweep)"
    return f"block matrix ({mb:.0f} MB) fits in L2 and is not flushed: L2-resident rates"


def make_problem(name: str, ninc_needed: int = 0):
    from cpfem_code_b200 import generator
    if name == "points":
        return generator.point_batch(POINTS, seed=1)
    prob = generator.workload(name)
    if prob.ninc1 < ninc_needed:
        prob = generator.workload(name, ninc=ninc_needed)
    return prob


def step_config(prob, steps: int, reports: list[dict]) -> dict:
    """The `config` both arms print: the workload and the exact steps timed
    (identical between the arms when their Newton iterations agree)."""
    if WORKLOAD == "points":
        return {"workload": WORKLOAD, "desc": DESC, "points": prob.ngps,
                "step": "one DSTRSS pass over every point from the same inputs"}
    incs = sorted({r["inc"] for r in reports})
    return {"workload": WORKLOAD, "desc": DESC,
            "start": "the generated initial state (increment 1, nothing applied yet)",
            "step": "one global Newton iteration (NRITER loop body; UPDATE_NODE opens and "
                    "cumslip/UPDATE_GPTV/DoReorient close each increment)",
            "newton_iters": steps, "increments_touched": [incs[0], incs[-1]] if incs else None,
            "sor_sweeps": int(sum(r["sor_sweeps"] for r in reports)),
            "sor_sweeps_per_step": [int(r["sor_sweeps"]) for r in reports]}


def stress_errors(p, ref, mid_increment: bool = False) -> dict:
    """Per-point and macroscopic (mean s11) stress error of `p` against
    `ref`, relative to the largest stress and to the mean, and the nodal
    coordinate error.  Inside an increment the stress is the committed st
    plus the last Newton iteration's ds (UPDATE_GPTV has not run)."""
    s, r = (p.st + p.ds, ref.st + ref.ds) if mid_increment else (p.st, ref.st)
    return {"stress_per_point": float(np.abs(s - r).max() / np.abs(r).max()),
            "stress_macro": float(abs(s[:, 0].mean() - r[:, 0].mean()) / abs(r[:, 0].mean())),
            "x": float(np.abs(p.x - ref.x).max() / np.abs(ref.x).max())}


# ------------------------------------------------------------------ CPU leg
def cpu_steps(prob, steps: int, threads: int):
    """The checker (oracle/, the C++ restatement of the reference) on the
    host cores: `steps` Newton iterations from the state held in `prob`.
    Returns (seconds, reports, final state)."""
    from cpfem_code_b200 import NewtonStepper
    from oracle import OracleSolver
    p = prob.copy()
    o = OracleSolver(p, 8, threads=threads)
    st = NewtonStepper(o)
    t0 = time.perf_counter()
    reps = [st.step() for _ in range(steps)]
    dt = time.perf_counter() - t0
    o.download()
    o.close()
    return dt, reps, p


def cpu_points(prob, threads: int):
    """The checker's DSTRSS pass over the first POINTS_CPU points of `prob`
    (the inputs before the pass)."""
    from oracle import OracleSolver
    p = prob.first_points(POINTS_CPU)
    o = OracleSolver(p, 8, threads=threads)
    t0 = time.perf_counter()
    o.constitutive(1, 1)
    dt = time.perf_counter() - t0
    o.download()
    o.close()
    return dt, p


def run_reference(args):
    ws, rank, local = dist_env()
    dist = init_dist(ws, "gloo")
    if rank != 0:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return 0
    threads = os.cpu_count() or 1
    if WORKLOAD == "diff16":
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no adjoint, and its forward "
                          "replay needs the history of a 16^3 FE run that the host cores take about 13 minutes "
                          "to compute"}), flush=True)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return 0
    prob = make_problem(WORKLOAD)
    if WORKLOAD == "points":
        dts = []
        for _ in range(args.steps):
            dt, _ = cpu_points(prob, threads)
            dts.append(dt)
        secs = float(sum(dts))
        value = POINTS_CPU * args.steps / secs
        config = step_config(prob, args.steps, [])
        sample = f"{args.steps} DSTRSS passes over the first {POINTS_CPU} of the {prob.ngps} points"
    else:
        secs, reps, _ = cpu_steps(prob, args.steps, threads)
        value = prob.ngps * args.steps / secs
        config = step_config(prob, args.steps, reps)
        sample = (f"Newton iterations 1..{args.steps} from the generated initial state "
                  f"({config['sor_sweeps']} SOR sweeps), the same steps as the device arm times")
    line = {
        "impl": "reference", "metric": METRIC,
        "value": value, "unit": "GP-updates/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator, fs3pre semantics)",
        "config": config,
        "warmup_note": "none run: a host run has nothing to warm, and the timed steps must start "
                       "from the generated initial state like the device arm's",
        "cpu_baseline": {"value": value, "unit": "GP-updates/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "GP-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------ GPU leg
STATE_FIELDS = ("x", "dx", "fc", "ddx", "eps", "dep", "st", "ep", "ds", "de", "rt", "dr",
                "sv", "dsv", "srate", "cumslip", "timestwinned", "twinsys")


def pinned_like(prob):
    """Re-back the state arrays of `prob` with pinned host memory."""
    import torch
    for name in STATE_FIELDS:
        a = getattr(prob, name)
        t = torch.empty(a.shape, dtype=getattr(torch, str(a.dtype)), pin_memory=True)
        b = t.numpy()
        b[...] = a
        setattr(prob, name, b)
        prob.meta.setdefault("_pinned", []).append(t)


def moved_bytes(prob, ns: int) -> int:
    """Bytes one upload (or download) moves: the nodal vectors and the used
    columns of every GP field."""
    nsv = 3 + ns
    per_gp = 8 * (2 + 24 + 6 + 2 * nsv + 2 * ns) + 8
    return 4 * 3 * prob.nnod * 8 + prob.ngps * per_gp


def _state_arrays(p):
    return {n: getattr(p, n).copy() for n in ("x", "dx", "st", "ds", "sv", "ep", "cumslip")}


AD_INC, AD_CHK = 4, 2


def run_adjoint(g, prob, start, de, dr, dt):
    """Time one replay and one replay-with-gradients over every GP (wall
    clock around the synchronous calls, the history's upload included)."""
    from cpfem_code_b200 import ReplayHistory, abi
    hist = ReplayHistory(np.repeat(de[None], AD_INC, 0), np.repeat(dr[None], AD_INC, 0), np.full(AD_INC, dt),
                         np.full(prob.ngps, 1.0 / prob.ngps), np.zeros(prob.ngps), q=(1.0, 0.0, 0.0),
                         chk_every=AD_CHK)
    g.upload(start)
    try:
        g.adjoint_forward(hist)   # warm-up (buffers)
        t0 = time.perf_counter()
        J, _ = g.adjoint_forward(hist)
        tf = time.perf_counter() - t0
        t0 = time.perf_counter()
        g.adjoint_grad(hist)
        tg = time.perf_counter() - t0
    except abi.FasError as e:
        return {"error": str(e)}
    n = prob.ngps * AD_INC
    return {"history": f"{AD_INC} increments per GP, each the last timed increment's strain increment "
                       f"and spin, from the state at the start of the increments leg; checkpoints every {AD_CHK}",
            "objective": "sum over GPs of (lattice strain along x)^2 / (2 ngps)", "J": J,
            "forward_s": tf, "grad_s": tg, "gp_increments_per_s_forward": n / tf,
            "gp_increments_per_s_grad": n / tg}


def timed_steps(g, start, steps: int, mode: int, level: int = 1):
    """`steps` Newton iterations from `start` on the device (state resident),
    one event pair around the region; returns (profile, reports)."""
    from cpfem_code_b200 import NewtonStepper
    g.upload(start)
    g.set_mode(mode)
    st = NewtonStepper(g)
    if level:
        g.profile(level)
    reps = [st.step() for _ in range(steps)]
    prof = g.profile(0) if level else None
    return prof, reps


def run_increments(g, prob, start, ninc_warm: int, ninc_timed: int):
    """Seconds per whole increment, plain FP64 against the tuned form (FP32
    SOR sweeps with FP64 residual refinement), over the same increments from
    the same state (the state after `ninc_warm` increments)."""
    from cpfem_code_b200 import abi
    g.upload(start)
    g.set_mode(abi.FAS_MODE_PLAIN)
    for i in range(1, ninc_warm + 1):
        g.increment(i)
    s0 = prob.copy()
    g.download(s0)
    incs = list(range(ninc_warm + 1, ninc_warm + ninc_timed + 1))
    out, ends = {}, {}
    legs = [("plain", abi.FAS_MODE_PLAIN), ("tuned", TUNED_MODE),
            ("plain_consistent_tangent", abi.FAS_MODE_TANGENT_CONSISTENT),
            ("plain_graph", abi.FAS_MODE_GRAPH), ("tuned_graph", TUNED_MODE | abi.FAS_MODE_GRAPH),
            ("tuned_sym", TUNED_MODE | abi.FAS_MODE_SOR_SYM)]
    for tag, mode in legs:
        t = s0.copy()
        g.upload(t)
        g.set_mode(mode)
        g.profile(1)
        nit = 0
        for i in incs:
            rep, _ = g.increment(i)
            nit += len(rep)
        prof = g.profile(0)
        g.download(t)
        ends[tag] = t
        g.profile(2)                  # one more increment with per-phase events
        g.upload(s0)
        g.increment(incs[0])
        ph = g.profile(0)
        out[tag] = {"s_per_increment": prof["ms_total"] / 1e3 / len(incs), "newton_iters": nit,
                    "ms_constitutive_first_increment": ph["ms_constitutive"],
                    "sor_sweeps": int(prof["sor_sweeps"]),
                    "gp_updates_per_s": prob.ngps * nit / (prof["ms_total"] / 1e3)}
    g.set_mode(abi.FAS_MODE_PLAIN)
    e = stress_errors(ends["tuned"], ends["plain"])
    out["increments"] = [incs[0], incs[-1]]
    out["tuned"]["mode"] = "FP32-matrix SOR sweeps with FP64 residual refinement every 16 sweeps"
    out["plain_consistent_tangent"]["mode"] = "plain FP64 with the consistent tangent (Newton counts of both tangents)"
    out["speedup_tuned_vs_plain_s_per_increment"] = out["plain"]["s_per_increment"] / out["tuned"]["s_per_increment"]
    out["tuned_vs_plain_error"] = e
    out["consistent_tangent_vs_plain_error"] = stress_errors(ends["plain_consistent_tangent"], ends["plain"])
    out["plain_graph"]["mode"] = "plain FP64, each increment's NRITER as one CUDA graph (conditional while nodes)"
    out["plain_graph"]["same_result_as_plain"] = all(
        np.array_equal(getattr(ends["plain_graph"], k), getattr(ends["plain"], k)) for k in _state_arrays(s0))
    out["speedup_graph_vs_plain_s_per_increment"] = (out["plain"]["s_per_increment"]
                                                     / out["plain_graph"]["s_per_increment"])
    out["tuned_graph"]["mode"] = "the tuned form with each increment's NRITER as one CUDA graph"
    out["tuned_graph"]["same_result_as_tuned"] = all(
        np.array_equal(getattr(ends["tuned_graph"], k), getattr(ends["tuned"], k)) for k in _state_arrays(s0))
    out["tuned_sym"]["mode"] = ("the tuned form on symmetric FP32 rows (each off-diagonal block streamed once, "
                                "transposed products pushed by vector atomic adds); no effect on 20-node rows")
    out["speedup_tuned_sym_vs_plain_s_per_increment"] = (out["plain"]["s_per_increment"]
                                                         / out["tuned_sym"]["s_per_increment"])
    out["tuned_sym_vs_plain_error"] = stress_errors(ends["tuned_sym"], ends["plain"])
    return out, s0, ends["plain"]


def run_gpu(args):
    import torch

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = init_dist(ws, "nccl")
    dev = torch.device("cuda", local)
    if WORKLOAD == "points":
        return run_gpu_points(args, ws, rank, local, dist, dev)
    if WORKLOAD == "diff16":
        return run_gpu_diff16(args, ws, rank, local, dist, dev)
    from cpfem_code_b200 import GpuSolver, NewtonStepper, abi

    prob = make_problem(WORKLOAD, INC_WARM + INC_TIMED + 2)
    start = prob.copy()
    g = GpuSolver(prob, upload=False)

    # ---- warm-up: W steps from the initial state, then discarded
    g.profile(1)
    g.upload(start)
    st = NewtonStepper(g)
    for _ in range(args.warmup):
        st.step()
    launches_before = int(g.profile(0)["n_launches"])

    # ---- timed: K steps from the initial state, state resident in HBM
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    t0 = time.perf_counter()
    prof, reps = timed_steps(g, start, args.steps, abi.FAS_MODE_PLAIN)
    wall = time.perf_counter() - t0
    torch.cuda.synchronize()
    clk = clocks.stop()
    dev_s = prof["ms_total"] / 1e3
    t_max, work = reduce_max_sum(dist, dev_s, float(prob.ngps * args.steps), dev)
    value = work / t_max
    resident = prob.copy()
    g.download(resident)
    resident_end = _state_arrays(resident)

    # ---- e2e: the same steps through the C ABI, state from pinned host memory
    e2e_s, deterministic = 0.0, None
    if not args.no_e2e:
        host = start.copy()
        pinned_like(host)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        st = NewtonStepper(g)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            g.upload(host)
            st.step()
            g.download(host)
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
        deterministic = all(np.array_equal(v, getattr(host, k)) for k, v in resident_end.items())
    te, work_e = reduce_max_sum(dist, e2e_s, float(prob.ngps * args.steps), dev)

    # ---- whole increments: plain FP64 against the tuned form
    incr, s_inc, plain_end = None, None, None
    if not args.no_increments:
        incr, s_inc, plain_end = run_increments(g, prob, start, INC_WARM, INC_TIMED)

    # ---- adjoint: every GP replays the last timed increment's strain
    # increment and spin AD_INC times
    adjoint = None
    if not args.no_adjoint and s_inc is not None:
        adjoint = run_adjoint(g, prob, s_inc, plain_end.de, plain_end.dr,
                              float(prob.tiem[INC_WARM + INC_TIMED - 1]))

    # ---- the dominant kernel as the steps run it: one FACSLS solve (CUDA
    # graph, programmatic launches) of the first step, colour kernels and
    # stopping tests under one event pair; the same for the FP32 sweeps;
    # the constitutive pass of one step with per-phase events
    roof = None
    if rank == 0:
        roof = rooflines(g, start, prob)

    if rank == 0:
        pk = peaks()
        line = {
            "metric": METRIC,
            "value": value, "unit": "GP-updates/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator, fs3pre semantics)",
            "config": step_config(prob, args.steps, reps),
            "parallelism": f"replicas{ws}",
            "l2": l2_note(prob),
            "wall_s": wall,
            "gpu_launches": int(prof["n_launches"]),
            "launches_before_timed": launches_before,
            "roofline": roof["sor"] if roof else None,
            "rooflines": roof,
            "clocks": clk,
            "e2e": {"value": work_e / te if te > 0 else None, "unit": "GP-updates/s",
                    "h2d_bytes_per_step": moved_bytes(prob, int(prob.nss.max())),
                    "d2h_bytes_per_step": moved_bytes(prob, int(prob.nss.max())),
                    "same_result_as_resident_run": deterministic},
            "increments": incr,
            "adjoint": adjoint,
        }
        if ws == 1 and not args.no_cpu:
            # the checker from the same initial state over the first
            # CPU_STEPS steps: the host-core baseline, and the full-size
            # error of the device path (plain and tuned) against it
            threads = os.cpu_count() or 1
            secs, reps_c, pc = cpu_steps(start, CPU_STEPS, threads)
            line["cpu_baseline"] = {
                "value": prob.ngps * CPU_STEPS / secs, "unit": "GP-updates/s", "cores": threads,
                "kind": "port",
                "sample": f"Newton iterations 1..{CPU_STEPS} from the generated initial state "
                          f"({sum(r['sor_sweeps'] for r in reps_c)} SOR sweeps) by the C++ restatement, "
                          f"{secs:.1f} s"}
            errs = {}
            for tag, mode in (("plain", abi.FAS_MODE_PLAIN), ("tuned", TUNED_MODE),
                              ("tuned_sym", TUNED_MODE | abi.FAS_MODE_SOR_SYM)):
                q = prob.copy()
                _, rg = timed_steps(g, start, CPU_STEPS, mode, level=0)
                g.download(q)
                errs[tag] = dict(stress_errors(q, pc, mid_increment=not reps_c[-1]["closes_increment"]),
                                 same_sweeps=[r["sor_sweeps"] for r in rg] == [r["sor_sweeps"] for r in reps_c])
            g.set_mode(abi.FAS_MODE_PLAIN)
            line["oracle_error"] = dict(errs, after=f"{CPU_STEPS} Newton iterations from the initial state, "
                                                    "against the FP64 checker in the same SOR order")
        print(json.dumps(line), flush=True)
        del pk
    g.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def rooflines(g, start, prob) -> dict:
    """Achieved rates of the dominant kernels against the measured peaks.

    * SOR colour kernels (FP64 and the tuned FP32 copy): algorithmic bytes of
      one whole FACSLS solve -- the first step's -- over its device time with
      the CUDA graph and programmatic launches the steps use (per-launch
      event pairs would serialise the overlapped launches).  `launch_ms` is
      that time per colour launch, so launches x launch_ms is the solve.
    * k_elem (constitutive pass): the algorithmic FP64 operations counted per
      GP (fas_flops.h) over its per-launch event time, against measured DGEMM.
    """
    from cpfem_code_b200 import abi
    pk = peaks()
    out = {}
    kernels = {"sor": "k_sor_colour_tma<double,27,4>", "sor_fp32": "k_sor_colour_tma<float,27,4>",
               "sor_tiles": "k_sor_tiles<double>", "sor_fp32_tiles": "k_sor_tiles<float>",
               "sor_fp32_sym": "k_sor_colour_tma<float,15,8,true>"}
    for tag, mode in (("sor", abi.FAS_MODE_PLAIN), ("sor_fp32", abi.FAS_MODE_SOR_FP32),
                      ("sor_tiles", abi.FAS_MODE_SOR_TILES),
                      ("sor_fp32_tiles", abi.FAS_MODE_SOR_FP32 | abi.FAS_MODE_SOR_TILES),
                      ("sor_fp32_sym", abi.FAS_MODE_SOR_FP32 | abi.FAS_MODE_SOR_SYM)):
        g.upload(start)
        g.set_mode(mode)
        g.update_node()
        g.elvals(1, 1)
        g.suvals(1)
        g.profile(1)
        g.facsls()
        p = g.profile(0)
        secs = p["ms_total"] / 1e3
        ach = p["sor_bytes"] / secs / 1e9
        nl = max(int(p["n_sor_colour"]), 1)
        out[tag] = {"kernel": kernels[tag],
                    "bound": "hbm", "achieved": ach, "peak": pk["hbm_gbs"], "unit": "GB/s",
                    "frac": ach / pk["hbm_gbs"], "peak_source": pk["source"],
                    "traffic": (SOR_TRAFFIC_PER_LAUNCH if tag == "sor" else
                                SOR32_TRAFFIC_PER_LAUNCH if tag == "sor_fp32" else None)
                    if WORKLOAD == "cube64" else None,
                    "bytes_per_launch": p["sor_bytes"] / nl, "launch_ms": p["ms_total"] / nl,
                    "launches": nl, "sweeps": int(p["sor_sweeps"]),
                    "timed": "one FACSLS solve of Newton iteration 1 of increment 1 (CUDA graph, programmatic "
                             "launches, stopping tests included) under one event pair"}
    g.set_mode(abi.FAS_MODE_PLAIN)
    # the constitutive pass of a plastic Newton iteration: step 3 from the start
    from cpfem_code_b200 import NewtonStepper
    g.upload(start)
    st = NewtonStepper(g)
    st.step()
    st.step()
    g.profile(2)
    st.step()
    p = g.profile(0)
    ops = float(g.cp_ops().sum())
    fp = fp64_peak_tflops()
    if p["ms_constitutive"] > 0:
        ach = ops / (p["ms_constitutive"] / 1e3) / 1e12
        out["constitutive"] = {"kernel": "k_elem<12>", "bound": "fp64", "achieved": ach, "peak": fp["tflops"],
                               "unit": "TFLOP/s", "frac": ach / fp["tflops"], "peak_source": fp["source"],
                               "gp_updates_per_s": p["gp_updates"] / (p["ms_constitutive"] / 1e3),
                               "timed": "per-launch events of the constitutive pass of Newton iteration 3"}
    return out


DIFF_INC, DIFF_CHK = 20, 5
DIFF_BINS = ((1, 1, 1), (2, 0, 0), (2, 2, 0), (3, 1, 1), (3, 3, 1), (4, 2, 0), (4, 2, 2), (5, 3, 1))


def diff16_history(g, prob):
    """The 16^3 run's strain history: every increment on the device (the
    plain path), each GP's converged strain increment and spin recorded
    before UPDATE_GPTV commits it."""
    from cpfem_code_b200 import ReplayHistory, calibration
    start = prob.copy()
    de, dr = [], []
    for inc in range(1, DIFF_INC + 1):
        g.update_node()
        g.nriter(inc)
        q = g.download(prob.copy())
        de.append(q.de.copy())
        dr.append(q.dr.copy())
        g.update_gptv()
        g.do_reorient(inc)
    euler = start.sv[:, :3]
    w = np.zeros(prob.ngps)
    for hkl in DIFF_BINS:
        w += calibration.bin_weights(euler, calibration.cubic_family(hkl), (1.0, 0.0, 0.0), 5.0)
    hist = ReplayHistory(np.stack(de), np.stack(dr), prob.tiem[:DIFF_INC], w / len(DIFF_BINS),
                         np.zeros(prob.ngps), q=(1.0, 0.0, 0.0), chk_every=DIFF_CHK)
    return start, hist


def run_gpu_diff16(args, ws, rank, local, dist, dev):
    """Configuration 3: adjoint gradients of a lattice-strain objective over
    the 16^3 cube's 20 increments.  A step is one gradient evaluation
    (fas_gpu_adjoint_grad: the replay of every GP's recorded history with
    checkpoints every 5 increments, then the reverse sweep)."""
    import torch

    from cpfem_code_b200 import GpuSolver, generator
    prob = generator.workload("cube16")
    g = GpuSolver(prob)
    start, hist = diff16_history(g, prob)
    g.upload(start)
    for _ in range(args.warmup):
        g.adjoint_grad(hist)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    g.profile(1)
    for _ in range(args.steps):
        out = g.adjoint_grad(hist)
    prof = g.profile(0)
    clk = clocks.stop()
    work = float(prob.ngps * DIFF_INC * args.steps)
    t_max, work = reduce_max_sum(dist, prof["ms_total"] / 1e3, work, dev)
    # e2e: the history uploaded from host memory every step (the call copies it)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        g.upload(start)
        g.adjoint_grad(hist)
    torch.cuda.synchronize()
    te, work_e = reduce_max_sum(dist, time.perf_counter() - t0, float(prob.ngps * DIFF_INC * args.steps), dev)
    line = None
    if rank == 0:
        # central differences (relative step 1e-6) of J in h0 (ampar(2)) and
        # in a uniform shift of every initial CRSS, against the gradients
        fd = {}
        h0 = float(prob.ampar[0, 0, 1])
        for name, setter, gval in (
                ("h0", lambda p, d: p.ampar[:, :, 1].__iadd__(d), out["ampar"][0, 1]),
                ("crss", lambda p, d: p.sv[:, 3:15].__iadd__(d), out["sv"][:, 3:15].sum())):
            step = 1e-6 * (h0 if name == "h0" else float(start.sv[:, 3:15].mean()))
            J = []
            for sgn in (1.0, -1.0):
                p = start.copy()
                setter(p, sgn * step)
                gg = GpuSolver(p)
                J.append(gg.adjoint_forward(hist)[0])
                gg.close()
            d = (J[0] - J[1]) / (2 * step)
            fd[name] = {"adjoint": float(gval), "central_difference": d,
                        "rel_diff": abs(float(gval) - d) / max(abs(d), 1e-300)}
        line = {
            "metric": METRIC, "value": work / t_max, "unit": "GP-increments/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator, fs3pre semantics); history recorded from the 16^3 FE run",
            "config": {"workload": WORKLOAD, "desc": DESC, "gps": prob.ngps, "increments": DIFF_INC,
                       "checkpoint_every": DIFF_CHK, "bins": [list(b) for b in DIFF_BINS],
                       "step": "one fas_gpu_adjoint_grad call (forward replay with checkpoints + reverse sweep)"},
            "parallelism": f"replicas{ws}", "gpu_launches": int(prof["n_launches"]),
            "J": out["J"], "finite_difference_check": fd,
            "roofline": None,
            "roofline_note": "the reverse kernel is bound by local-memory spills (profiles/k_replay_adj_points16k.md)",
            "clocks": clk,
            "e2e": {"value": work_e / te, "unit": "GP-increments/s",
                    "h2d_bytes_per_step": int(hist.de.nbytes + hist.dr.nbytes + hist.w.nbytes + hist.y.nbytes),
                    "d2h_bytes_per_step": int(prob.ngps * (6 + 63) * 8 + 10 * 8 * prob.nmatl)},
        }
        if ws == 1 and not args.no_cpu:
            from oracle import OracleSolver
            o = OracleSolver(start.copy(), 8, threads=os.cpu_count() or 1)
            t0 = time.perf_counter()
            o.adjoint_forward(hist)
            dt = time.perf_counter() - t0
            o.close()
            line["cpu_baseline"] = {"value": prob.ngps * DIFF_INC / dt, "unit": "GP-increments/s",
                                    "cores": os.cpu_count() or 1, "kind": "port",
                                    "sample": "the checker's forward replay of the same history (no reverse sweep: "
                                              f"the checker has none), {dt:.2f} s"}
        print(json.dumps(line), flush=True)
    g.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_gpu_points(args, ws, rank, local, dist, dev):
    """The constitutive micro-benchmark: every step is one DSTRSS pass over
    2^20 points from the same inputs (re-uploaded between steps, outside
    the per-launch event pair)."""
    import torch

    from cpfem_code_b200 import GpuSolver
    prob = make_problem("points")
    start = prob.copy()
    g = GpuSolver(prob)
    for _ in range(args.warmup):
        g.upload(start)
        g.constitutive(1, 1)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    ms, launches, ops = 0.0, 0, 0.0
    for _ in range(args.steps):
        g.upload(start)
        g.profile(2)
        g.constitutive(1, 1)
        p = g.profile(0)
        ms += p["ms_constitutive"]
        launches += int(p["n_launches"])
    ops = float(g.cp_ops().sum())
    clk = clocks.stop()
    t_max, work = reduce_max_sum(dist, ms / 1e3, float(prob.ngps * args.steps), dev)
    value = work / t_max
    # e2e: inputs from pinned host memory, outputs back, every step
    host = start.copy()
    pinned_like(host)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        g.upload(host)
        g.constitutive(1, 1)
        g.download(host)
    torch.cuda.synchronize()
    e2e = time.perf_counter() - t0
    te, work_e = reduce_max_sum(dist, e2e, float(prob.ngps * args.steps), dev)
    # the batched persistent kernel on the same points: a grid of the CTAs
    # that reside at once, every warp taking the next 32 points of the
    # work-sorted order from a device queue (FAS_MODE_CP_QUEUE)
    from cpfem_code_b200 import abi
    g.set_mode(abi.FAS_MODE_CP_QUEUE)
    for _ in range(args.warmup):
        g.upload(start)
        g.constitutive(1, 1)
    qms = 0.0
    for _ in range(args.steps):
        g.upload(start)
        g.profile(2)
        g.constitutive(1, 1)
        qms += g.profile(0)["ms_constitutive"]
    qprob = start.copy()
    g.download(qprob)
    g.set_mode(abi.FAS_MODE_PLAIN)
    if rank == 0:
        fp = fp64_peak_tflops()
        ach = ops / (ms / 1e3 / args.steps) / 1e12
        g.upload(start)
        g.constitutive(1, 1)
        g.download(prob)
        line = {
            "metric": METRIC, "value": value, "unit": "GP-updates/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
            "config": step_config(prob, args.steps, []), "parallelism": f"replicas{ws}",
            "l2": "inputs (about 1 KB of state per point, 1 GB in all) larger than L2",
            "gpu_launches": launches,
            "roofline": {"kernel": "k_points<12>", "bound": "fp64", "achieved": ach, "peak": fp["tflops"],
                         "unit": "TFLOP/s", "frac": ach / fp["tflops"], "peak_source": fp["source"],
                         "traffic": None},
            "clocks": clk,
            "e2e": {"value": work_e / te, "unit": "GP-updates/s",
                    "h2d_bytes_per_step": moved_bytes(prob, 12), "d2h_bytes_per_step": moved_bytes(prob, 12)},
            "persistent": {"value": prob.ngps * args.steps / (qms / 1e3), "unit": "GP-updates/s",
                           "ms_per_pass": qms / args.steps, "plain_ms_per_pass": ms / args.steps,
                           "same_result_as_plain": bool(np.array_equal(qprob.ds, prob.ds)
                                                        and np.array_equal(qprob.dsv, prob.dsv)),
                           "mode": "batched persistent kernel: resident CTAs only, warps take the next 32 "
                                   "points of the work-sorted order from a device queue"},
        }
        if ws == 1 and not args.no_cpu:
            secs, pc = cpu_points(start, os.cpu_count() or 1)
            line["cpu_baseline"] = {"value": POINTS_CPU / secs, "unit": "GP-updates/s",
                                    "cores": os.cpu_count() or 1, "kind": "port",
                                    "sample": f"one DSTRSS pass over the first {POINTS_CPU} points"}
            n = POINTS_CPU
            ds_g, ds_o = prob.ds[:n], pc.ds
            line["oracle_error"] = {"stress_per_point": float(np.abs(ds_g - ds_o).max() / np.abs(ds_o).max()),
                                    "points_compared": n}
        print(json.dumps(line), flush=True)
    g.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_case(args) -> int:
    """Small single-purpose runs for profiling (one GPU, a few launches):

    * ``--case facsls``: UPDATE_NODE, ELVALS, SUVALS and one FACSLS solve of
      the workload's first Newton iteration, in ``--mode``;
    * ``--case adjoint``: the adjoint replay with gradients on ``--points``
      independent FCC points (4 increments, checkpoints every 2);
    * ``--case points``: ``--reps`` DSTRSS passes over ``--points`` points;
    * ``--case sweeps``: microseconds per sweep of the first FACSLS of n^3
      cubes on every solve path (one CTA, colour kernels, tiles; FP64 and
      FP32, and FP32 on symmetric rows), one JSON line per size.
    """
    from cpfem_code_b200 import GpuSolver, ReplayHistory, generator
    if args.case == "facsls":
        p = make_problem(WORKLOAD)
        g = GpuSolver(p, mode=args.mode)
        g.update_node()
        g.elvals(1, 1)
        g.suvals(1)
        sweeps, err = g.facsls()
        print(f"{WORKLOAD}: FACSLS {sweeps} sweeps, error {err:.3e}", flush=True)
    elif args.case == "adjoint":
        n = args.points
        p = generator.point_batch(n, seed=1)
        rng = np.random.default_rng(2)
        de = np.stack([p.de * (1.0 + 0.2 * rng.standard_normal(p.de.shape)) for _ in range(4)])
        dr = 2e-4 * rng.standard_normal((4, n, 3))
        h = ReplayHistory(de, dr, np.full(4, p.tiem[0]), np.ones(n), np.zeros(n), chk_every=2)
        g = GpuSolver(p)
        out = g.adjoint_grad(h)
        print(f"adjoint: {n} points x 4 increments, J {out['J']:.4e}", flush=True)
    elif args.case == "sweeps":
        # us per sweep of the first FACSLS of n^3 cubes on each solve path
        from cpfem_code_b200 import abi
        paths = {"one_cta": 0, "colour": abi.FAS_MODE_SOR_GRID,
                 "tiles": abi.FAS_MODE_SOR_GRID | abi.FAS_MODE_SOR_TILES,
                 "tiles_fp32": abi.FAS_MODE_SOR_GRID | abi.FAS_MODE_SOR_TILES | abi.FAS_MODE_SOR_FP32,
                 "colour_fp32": abi.FAS_MODE_SOR_GRID | abi.FAS_MODE_SOR_FP32,
                 "colour_fp32_sym": abi.FAS_MODE_SOR_GRID | abi.FAS_MODE_SOR_FP32 | abi.FAS_MODE_SOR_SYM}
        for n in (2, 4, 8, 12, 16, 20, 24, 32, 40, 48, 64):
            p = generator.cube_config(n=n, ninc=1, grain=1, seed=n)
            row = {"n": n, "nodes": p.nnod}
            for tag, mode in paths.items():
                if tag == "one_cta" and p.nnod > 256:   # above it mode 0 is the grid path
                    continue
                g = GpuSolver(p.copy(), mode=mode)
                g.update_node()
                g.elvals(1, 1)
                g.suvals(1)
                start = g.download(p.copy())
                g.facsls()                 # warm-up (graphs, buffers)
                g.upload(start)
                g.profile(1)
                sw, _ = g.facsls()
                pr = g.profile(0)
                row[tag] = round(1e3 * pr["ms_total"] / max(sw, 1), 2)
                row["sweeps"] = sw
                g.close()
            print(json.dumps(row), flush=True)
        return 0
    else:
        p = generator.point_batch(args.points, seed=1)
        g = GpuSolver(p.copy(), mode=args.mode)
        for _ in range(args.reps):
            g.upload(p)
            g.constitutive(1, 1)
        print(f"points: {args.points} x {args.reps} DSTRSS passes", flush=True)
    g.close()
    return 0


def main():
    global WORKLOAD, METRIC, DESC
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline and full-size oracle error")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer (e2e) leg")
    ap.add_argument("--no-increments", action="store_true", help="skip the whole-increment (plain vs tuned) leg")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint (replay gradients) leg")
    ap.add_argument("--workload", default=WORKLOAD, choices=list(WORKLOADS),
                    help="the headline 64^3 workload (default), another mesh, or the point batch")
    ap.add_argument("--case", default=None, choices=["facsls", "adjoint", "points", "sweeps"],
                    help="a small profiling run instead of the benchmark (see run_case)")
    ap.add_argument("--mode", type=int, default=0, help="FAS_MODE_* mask of --case facsls / points")
    ap.add_argument("--points", type=int, default=1 << 14, help="points of --case adjoint / points")
    ap.add_argument("--reps", type=int, default=2, help="passes of --case points")
    args = ap.parse_args()
    WORKLOAD = args.workload
    METRIC, DESC = WORKLOADS[WORKLOAD]
    if args.case:
        return run_case(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())

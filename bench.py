#!/usr/bin/env python
"""Benchmark of the FASOLT3 increment hot path on B200.

Workload: the 64^3 FCC aluminium cube (262,144 one-point bricks = GPs,
274,625 nodes, 823,875 DOF), grains of 2^3 elements with seeded uniform-SO(3)
orientations, uniaxial tension at 1e-3 strain per increment.  A *step* is one
increment of the driver loop: UPDATE_NODE -> NRITER -> UPDATE_GPTV ->
DoReorient.  W untimed increments, then K timed ones.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Metric: Gauss-point updates per second -- one DSTRSS evaluation of one GP in
one global Newton iteration -- over the whole increment (elements, assembly,
SOR, norms, commit), i.e. ngps * Newton iterations / time.  The seconds per
increment are reported beside it.  `value` is device time of the timed
increments with all inputs resident in HBM (CUDA events on the library's
stream); `e2e` replays the same increments from the same start state through
the C ABI with the whole state copied from pinned host memory before and
back after every increment.

N > 1 (torchrun): independent replicas, one per GPU (the path is one
problem on one GPU); time is the max over ranks, value the sum of work.
`--impl reference` times the CPU restatement of the reference on the host
cores instead (each step one complete Newton iteration of increment 1).
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
METRIC = "GP updates/s at 64^3 (DSTRSS evaluations per second of whole Newton iterations)"
SOR_TRAFFIC_PER_LAUNCH = 81.1e6   # DRAM bytes per colour launch, measured with ncu at 64^3
DESC = ("64^3 FCC Al one-point bricks (262,144 GPs, 823,875 DOF), 2^3-element grains, "
        "uniaxial tension 1e-3 per increment")
# other workloads (--workload): (metric, description); no ncu traffic figure
OTHER_WORKLOADS = {
    "brick20_32": ("GP updates/s, 32^3 20-node bricks (DSTRSS evaluations per second of whole Newton iterations)",
                   "32^3 FCC Al 20-node eight-GP bricks (262,144 GPs, 421,443 DOF), 2^3-element grains, "
                   "uniaxial tension 1e-3 per increment"),
    "mixed32": ("GP updates/s, 32^3 mixed FCC/HCP (DSTRSS evaluations per second of whole Newton iterations)",
                "32^3 one-point bricks (32,768 GPs), 50/50 random HCP-Zr (30 systems incl. twins) / FCC-Al grains "
                "of 2^3 elements, uniaxial tension 1e-3 per increment"),
    "brick20_10": ("GP updates/s, 10^3 20-node bricks (DSTRSS evaluations per second of whole Newton iterations)",
                   "10^3 FCC Al 20-node eight-GP bricks (the reference sample's mesh: 8,000 GPs), "
                   "one grain per element, uniaxial tension 1e-3 per increment"),
}


def peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return dict(hbm_gbs=float(d["hbm_gbs"]), source="measured")
    except Exception:
        return dict(hbm_gbs=6650.0, source="fallback")


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


# ------------------------------------------------------------------ CPU leg
def cpu_sample(prob, inc: int, warm_iters: int, timed_iters: int, threads: int) -> dict:
    """The checker (oracle/, the C++ restatement of the reference) on the
    host cores: complete Newton iterations of increment `inc` of the
    workload, starting from the state held in `prob`."""
    from oracle import OracleSolver
    o = OracleSolver(prob.copy(), 8, threads=threads)
    o.update_node()
    nit = 0
    for _ in range(warm_iters):
        nit += 1
        o.nr_step(inc, nit)
    t0 = time.perf_counter()
    sweeps = 0
    for _ in range(timed_iters):
        nit += 1
        r, more = o.nr_step(inc, nit)
        sweeps += r["sor_sweeps"]
    dt = time.perf_counter() - t0
    o.close()
    return dict(value=prob.ngps * timed_iters / dt, seconds=dt, iters=timed_iters, sweeps=sweeps,
                first_iter=warm_iters + 1)


def run_reference(args):
    ws, rank, local = dist_env()
    dist = init_dist(ws, "gloo")
    if rank != 0:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return 0
    from cpfem_code_b200 import generator
    prob = generator.workload(WORKLOAD)
    threads = os.cpu_count() or 1
    # iterations 1-2 of increment 1 are elastic (dx and ds start at zero);
    # the warm-up covers at least those
    s = cpu_sample(prob, 1, max(args.warmup, 2), args.steps, threads)
    line = {
        "impl": "reference", "metric": METRIC,
        "value": s["value"], "unit": "GP-updates/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * s["seconds"] / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator, fs3pre semantics)",
        "config": {"workload": WORKLOAD, "desc": DESC, "step": "one complete Newton iteration of increment 1"},
        "cpu_baseline": {"value": s["value"], "unit": "GP-updates/s", "cores": threads, "kind": "port",
                         "sample": f"Newton iterations {s['first_iter']}..{s['first_iter'] + s['iters'] - 1} "
                                   f"of increment 1 ({s['sweeps']} SOR sweeps) on {threads} threads"},
        "e2e": {"value": s["value"], "unit": "GP-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------ GPU leg
def pinned_like(prob):
    """Re-back the state arrays of `prob` with pinned host memory."""
    import torch
    for name in ("x", "dx", "fc", "ddx", "eps", "dep", "st", "ep", "ds", "de", "rt", "dr",
                 "sv", "dsv", "srate", "cumslip", "timestwinned", "twinsys"):
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
    return {n: getattr(p, n).copy() for n in ("x", "dx", "st", "sv", "ep", "ds", "cumslip")}


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
                       f"and spin, from the state before the timed increments; checkpoints every {AD_CHK}",
            "objective": "sum over GPs of (lattice strain along x)^2 / (2 ngps)", "J": J,
            "forward_s": tf, "grad_s": tg, "gp_increments_per_s_forward": n / tf,
            "gp_increments_per_s_grad": n / tg}


def run_gpu(args):
    import torch

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = init_dist(ws, "nccl")
    dev = torch.device("cuda", local)
    from cpfem_code_b200 import GpuSolver, abi, generator

    prob = generator.workload(WORKLOAD)
    ninc_needed = args.warmup + args.steps + 2
    if prob.ninc1 < ninc_needed:
        prob = generator.workload(WORKLOAD, ninc=ninc_needed)
    g = GpuSolver(prob, upload=False)
    g.profile(1)           # counts this library's launches before the timed region
    g.upload()
    inc = 0
    for _ in range(args.warmup):
        inc += 1
        g.increment(inc)
    # the state at the start of the timed increments, kept on the host so the
    # e2e and tuned legs replay exactly the same increments
    g.download()
    launches_before = int(g.profile(0)["n_launches"])
    start = prob.copy()
    inc0 = inc
    incs = list(range(inc0 + 1, inc0 + args.steps + 1))

    # ---- plain FP64, inputs resident in HBM: one event pair around the region
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    g.profile(1)
    nit = sweeps = 0
    t0 = time.perf_counter()
    for i in incs:
        rep, _ = g.increment(i)
        nit += len(rep)
        sweeps += sum(r["sor_sweeps"] for r in rep)
    prof = g.profile(0)
    wall = time.perf_counter() - t0
    torch.cuda.synchronize()
    clk = clocks.stop()
    dev_s = prof["ms_total"] / 1e3
    t_max, work = reduce_max_sum(dist, dev_s, float(prob.ngps * nit), dev)
    value = work / t_max
    g.download()
    plain_end = _state_arrays(prob)
    last_de, last_dr = prob.de.copy(), prob.dr.copy()   # the last timed increment's strain and spin

    # ---- e2e: the same increments through the ABI, state from pinned host memory
    nit_e, e2e_s, deterministic = 0, 0.0, None
    if not args.no_e2e:
        host = start.copy()
        pinned_like(host)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        for i in incs:
            g.upload(host)
            rep, _ = g.increment(i)
            g.download(host)
            nit_e += len(rep)
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
        deterministic = all(np.array_equal(v, getattr(host, k)) for k, v in plain_end.items())
    te, work_e = reduce_max_sum(dist, e2e_s, float(prob.ngps * nit_e), dev)

    # ---- adjoint: every GP replays the last timed increment's strain
    # increment and spin AD_INC times from the state at the start of the
    # timed increments; the objective and its gradients (fas_gpu_adjoint_grad)
    adjoint = None
    if not args.no_adjoint:
        adjoint = run_adjoint(g, prob, start, last_de, last_dr, float(prob.tiem[incs[-1] - 1]))

    # ---- tuned form: FP32 SOR sweeps with FP64 residual refinement
    tuned = None
    if not args.no_tuned:
        t = start.copy()
        g.upload(t)
        g.set_mode(abi.FAS_MODE_SOR_FP32)
        torch.cuda.synchronize()
        g.profile(1)
        nit_t = 0
        for i in incs:
            rep, _ = g.increment(i)
            nit_t += len(rep)
        prof_t = g.profile(0)
        g.set_mode(abi.FAS_MODE_PLAIN)
        g.download(t)
        st_ref, st_t = plain_end["st"], t.st
        tt, work_t = reduce_max_sum(dist, prof_t["ms_total"] / 1e3, float(prob.ngps * nit_t), dev)
        tuned = {"mode": "FP32-matrix SOR sweeps, FP64 residual refinement every 16 sweeps",
                 "value": work_t / tt, "s_per_increment": tt / args.steps, "newton_iters": nit_t,
                 "sor_sweeps": int(prof_t["sor_sweeps"]),
                 "speedup_vs_plain_s_per_increment": (t_max / args.steps) / (tt / args.steps),
                 "stress_err_per_point": float(np.abs(st_t - st_ref).max() / np.abs(st_ref).max()),
                 "stress_err_macro": float(abs(st_t[:, 0].mean() - st_ref[:, 0].mean())
                                           / abs(st_ref[:, 0].mean())),
                 "err_reference": "plain FP64 GPU path (equal to the FP64 checker to ~1e-15)"}

    # ---- per-kernel CUDA-event timing of one more increment (roofline)
    k = start.copy()
    g.upload(k)
    torch.cuda.synchronize()
    g.profile(2)
    g.increment(incs[0])
    prof_k = g.profile(0)

    # ---- one FACSLS solve as the increments run it (CUDA graph, programmatic
    # launches): colour kernels and stopping tests together, one event pair
    k = start.copy()
    g.upload(k)
    g.update_node()
    g.elvals(incs[0], 1)
    g.suvals(incs[0])
    torch.cuda.synchronize()
    g.profile(1)
    g.facsls()
    prof_s = g.profile(0)

    if rank == 0:
        pk = peaks()
        achieved = (prof_k["sor_bytes"] / (prof_k["ms_sor_colour"] / 1e3) / 1e9
                    if prof_k["ms_sor_colour"] else 0.0)
        launch_ms = prof_k["ms_sor_colour"] / max(prof_k["n_sor_colour"], 1)
        line = {
            "metric": METRIC,
            "value": value, "unit": "GP-updates/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator, fs3pre semantics)",
            "config": {"workload": WORKLOAD, "desc": DESC, "parallelism": f"replicas{ws}",
                       "increments": [incs[0], incs[-1]], "newton_iters": nit, "sor_sweeps": sweeps,
                       "l2": l2_note(prob)},
            "s_per_increment": t_max / args.steps,
            "wall_s": wall,
            "gpu_launches": int(prof["n_launches"]),
            "launches_before_timed": launches_before,
            "phases_ms_profiled_increment": {
                "constitutive": prof_k["ms_constitutive"], "assembly": prof_k["ms_assembly"],
                "sor_colour": prof_k["ms_sor_colour"], "total": prof_k["ms_total"]},
            "constitutive_gp_updates_per_s": prof_k["gp_updates"] / (prof_k["ms_constitutive"] / 1e3)
            if prof_k["ms_constitutive"] else None,
            "roofline": {"kernel": "k_sor_colour_tma", "bound": "hbm", "achieved": achieved,
                         "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": achieved / pk["hbm_gbs"],
                         "peak_source": pk["source"],
                         # ncu dram__bytes_read.sum + dram__bytes_write.sum of two colour
                         # launches of the same workload, scaled per row to the mean colour
                         # (ncu flushes the caches before every replay, so the solution
                         # vector is re-read from DRAM there)
                         "traffic": SOR_TRAFFIC_PER_LAUNCH,
                         "launch_ms": launch_ms,
                         "bytes_per_launch": prof_k["sor_bytes"] / max(prof_k["n_sor_colour"], 1),
                         "timed": f"CUDA events around every launch of increment {incs[0]}",
                         "achieved_solve": prof_s["sor_bytes"] / (prof_s["ms_total"] / 1e3) / 1e9,
                         "frac_solve": prof_s["sor_bytes"] / (prof_s["ms_total"] / 1e3) / 1e9 / pk["hbm_gbs"],
                         "solve": (f"one FACSLS of Newton iteration 1 of increment {incs[0]}: "
                                   f"{int(prof_s['sor_sweeps'])} sweeps, {prof_s['ms_total']:.2f} ms "
                                   "with its stopping tests, graph and programmatic launches")},
            "clocks": clk,
            "e2e": {"value": work_e / te if te > 0 else None, "unit": "GP-updates/s",
                    "h2d_bytes_per_step": moved_bytes(prob, int(prob.nss.max())),
                    "d2h_bytes_per_step": moved_bytes(prob, int(prob.nss.max())),
                    "s_per_increment": te / args.steps if te > 0 else None,
                    "newton_iters": nit_e, "increments": [incs[0], incs[-1]],
                    "same_result_as_resident_run": deterministic},
            "tuned": tuned,
            "adjoint": adjoint,
        }
        if ws == 1 and not args.no_cpu:
            # plastic state at the end of the timed increments: time the first
            # Newton iteration of the next increment on the host cores
            # `prob` still holds the whole state downloaded after the timed run
            s = cpu_sample(prob, incs[-1] + 1, 0, 1, os.cpu_count() or 1)
            line["cpu_baseline"] = {
                "value": s["value"], "unit": "GP-updates/s", "cores": os.cpu_count() or 1,
                "kind": "port",
                "sample": f"Newton iteration 1 of increment {incs[-1] + 1} ({s['sweeps']} SOR sweeps) "
                          f"by the C++ restatement from the same state, {s['seconds']:.1f} s"}
        print(json.dumps(line), flush=True)
    g.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    global WORKLOAD, METRIC, DESC, SOR_TRAFFIC_PER_LAUNCH
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer (e2e) leg")
    ap.add_argument("--no-tuned", action="store_true", help="skip the tuned-form (FP32 SOR) leg")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint (replay gradients) leg")
    ap.add_argument("--workload", default=WORKLOAD, choices=[WORKLOAD, *OTHER_WORKLOADS],
                    help="the headline 64^3 workload (default) or a 20-node brick mesh")
    args = ap.parse_args()
    if args.workload != WORKLOAD:
        WORKLOAD = args.workload
        METRIC, DESC = OTHER_WORKLOADS[WORKLOAD]
        SOR_TRAFFIC_PER_LAUNCH = None
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())

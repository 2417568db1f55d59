#!/usr/bin/env python
"""bench.py -- particle-steps/s of the Stokes-limit midpoint step on B200.

Workload (default): the single large instance of the benchmark set, 128^3
periodic cells (dx = 1), 65,536 particles as 4,096 bead-spring chains of 16
beads (k = 10, r0 = 1), soft repulsion eps = 1, rc = 1.5, eta = 1, kT = 0.01,
dt = 0.005, 4-point kernel; noise drawn on the device.  Inputs are seeded
synthetic data (there is no dataset).

One step = one full midpoint step (noise, 2 x (cell list, forces, spread,
FFT Stokes solve), RFD drift spreads, predictor and corrector).  `value` is
device time (CUDA events on the library's stream), L2 flushed between timed
steps with a 256 MiB write.  `e2e` is the same metric through the C ABI with
the step's input positions copied from pinned host memory and the new
positions read back every step.

Multi-GPU: one process per GPU, each an independent replica (the path has no
exchange step); value = all particle-steps / max-over-ranks time.
`--impl reference`: the FP64 CPU implementation of the same step on the
host's cores (the reference's CUDA build does not compile with CUDA 12).
"""
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

WORKLOAD = "plain_128"


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default=WORKLOAD)
    p.add_argument("--cpu-seconds", type=float, default=20.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    return p.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------------ clocks --
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 8:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if r[4 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


# ---------------------------------------------------------- algorithmic bytes
def stage_bytes(name, P):
    """Algorithmic DRAM bytes of one launch of a stage (FP32 fields, FP64
    particle state, materialised FP32 noise, int64 fixed-point spread grid)."""
    nc, npart, k = P["nc"], P["np"], P["kernel"]
    spec = 3 * 8 * (P["mx"] // 2 + 1) * P["my"] * P["mz"]
    touched = 3 * 8 * min(P["nc"], k ** 3 * npart)
    return {
        "noise": 4 * (12 * nc + 9 * npart),
        "cells": 40 * npart + 12 * P["mN"],
        "forces": 52 * npart + 4 * P["mN"],
        "grid_zero": 24 * nc,
        "spread": 48 * npart + 2 * touched,
        # force spread + the drift test (reference mode: the drift spreads
        # cancel and are skipped except at stencil changes)
        "spread_rfd": 48 * npart + 2 * touched + 36 * npart,
        # int64 field read + cleared, mean noise of the two solves, W written
        "wbuild": 24 * nc + 24 * nc + 36 * nc + 12 * nc,
        "plane_fwd": 12 * nc + spec,               # W read, half spectrum written
        "plane_inv": spec + 12 * nc,
        "xfwd": 24 * nc + 36 * nc + spec,
        "yfft": 2 * spec,
        "zsolve": 2 * spec,
        "xinv": spec + 12 * nc,
        "interp_update": 72 * npart + min(12 * nc, 12 * k ** 3 * npart),
        "counter": 8,
    }.get(name, 0)


# --------------------------------------------------------------- cpu side ---
def cpu_run(workload, seconds, threads=None):
    """Time the FP64 CPU implementation (oracle) on a bounded sample."""
    from oracle import oracle_py as O
    from fluam_b200 import workloads as W
    w = W.WORKLOADS[workload]
    m, L = w["cells"], w["box"]
    if w["chains"]:
        q, bi, bj = W.chains(w["chains"], w["beads"], L, 1, w["r0"])
    else:
        q, bi, bj = W.uniform(w["n"], L, 1), None, None
    o = O.Oracle(m, m, m, L, L, L, q, eta=w["eta"], kT=w["kT"], dt=w["dt"], cutoff=w["rc"],
                 kernel=w["kernel"], pair=O.PAIR_SOFT, soft_epsilon=w["eps"], seed=1)
    if bi is not None:
        o.set_bonds(bi, bj, np.full(len(bi), w["k"]), np.full(len(bi), w["r0"]))
    o.step(1)  # warm-up (page faults, thread pool)
    n = 0
    t0 = time.perf_counter()
    while True:
        o.step(1)
        n += 1
        el = time.perf_counter() - t0
        if el >= seconds or (n >= 2 and el * (n + 1) / n > 3 * seconds):
            break
    npart = q.shape[1]
    return {"value": npart * n / el, "unit": "particle-steps/s", "cores": O.num_threads(),
            "kind": "port",
            "sample": f"{n} steps of {workload} ({m}^3, {npart} particles), FP64 oracle, "
                      f"{el:.1f} s, OpenMP {O.num_threads()} threads"}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    per = max(args.cpu_seconds / max(args.steps, 1), 1.0)
    per = min(per, args.cpu_seconds)
    r = cpu_run(args.workload, per * max(1, min(args.steps, 3)))
    line = {
        "metric": "particle-steps/s", "value": r["value"], "unit": "particle-steps/s",
        "impl": "reference", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": True, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args.workload),
        "cpu_baseline": {"value": r["value"], "unit": r["unit"], "cores": r["cores"],
                         "kind": r["kind"], "sample": r["sample"]},
        "e2e": {"value": r["value"], "unit": r["unit"], "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": "the reference's CUDA build does not compile with CUDA 12 (legacy texture "
                "references); this arm times the FP64 CPU restatement of its step",
    }
    print(json.dumps(line), flush=True)
    return 0


def aggregate(local_times, dist=None, device=None):
    """Max over ranks of each local time (ms or s), as floats; the replicas
    do not exchange data, so this is the only collective of a run."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return [float(x) for x in local_times]
    import torch
    t = torch.tensor([float(x) for x in local_times], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def replica_seed(rank, base=1):
    """Each rank runs its own replica of the workload: same sizes, own seed."""
    return base + rank


def workload_config(name):
    from fluam_b200 import workloads as W
    w = W.WORKLOADS[name]
    return {"workload": f"{name}: {w['cells']}^3 periodic cells dx=1, {w['n']} particles"
                        + (f" ({w['chains']} chains x {w['beads']} beads, k={w['k']}, r0={w['r0']})"
                           if w["chains"] else " uniform")
                        + f", soft repulsion eps={w['eps']} rc={w['rc']}, {w['kernel']}-pt kernel,"
                          f" eta={w['eta']} kT={w['kT']} dt={w['dt']}",
            "cells": w["cells"], "np": w["n"], "kernel": w["kernel"],
            "fields": "fp32", "positions": "fp64", "spread": "int64 fixed point 2^-40",
            "l2": "flushed between timed steps (256 MiB write)"}


# -------------------------------------------------------------- GPU side ---
def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    from fluam_b200 import StokesLimit, workloads
    cfg, q, bonds = workloads.build(args.workload, seed=replica_seed(rank))
    cfg.device = local
    sim = StokesLimit(cfg, q)
    if bonds is not None:
        sim.load_bonds(*bonds)
    npart = q.shape[1]
    stream = torch.cuda.ExternalStream(sim.L.fsl_stream(sim.h))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    sim.step(max(args.warmup, 3))
    sim.sync()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()

    def timed_pass(k):
        e0 = [torch.cuda.Event(enable_timing=True) for _ in range(k)]
        e1 = [torch.cuda.Event(enable_timing=True) for _ in range(k)]
        for i in range(k):
            flush.fill_(float(i))
            torch.cuda.synchronize()
            e0[i].record(stream)
            sim.step(1)
            e1[i].record(stream)
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in zip(e0, e1))

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    total_ms = timed_pass(args.steps)            # pass A: the headline number
    sim.profile(True)                            # pass B: per-stage events
    sim.step(1)
    sim.sync()
    sim.profile(True)
    prof_ms = timed_pass(args.steps)
    stages = sim.profile_read()
    sim.profile(False)
    clk = clocks.stop()
    sim.sync()
    st = sim.status()

    # e2e through the C ABI with pinned host buffers
    hq = torch.empty((3, npart), dtype=torch.float64).pin_memory()
    hq.copy_(torch.from_numpy(sim.positions()))
    import ctypes
    qp = ctypes.cast(hq.data_ptr(), ctypes.POINTER(ctypes.c_double))
    ke = max(10, args.steps // 4)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(ke):
        sim.L.fsl_set_positions(sim.h, qp)
        sim.L.fsl_step(sim.h, 1)
        sim.L.fsl_get_positions(sim.h, qp)
    e2e_s = time.perf_counter() - t0
    sim.sync()

    t_max, e2e_max = aggregate([total_ms, e2e_s], dist, device="cuda")
    if dist:
        dist.barrier()

    if rank == 0:
        hbm, peak_kind = peaks()
        P = {"nc": cfg.mx * cfg.my * cfg.mz, "np": npart, "kernel": cfg.kernel, "mx": cfg.mx,
             "my": cfg.my, "mz": cfg.mz,
             "mN": int(np.prod(sim.neighbor_grid()))}
        dom = max(stages.items(), key=lambda kv: kv[1]["total_ms"])
        dname, dv = dom
        avg_ms = dv["total_ms"] / max(dv["launches"], 1)
        abytes = stage_bytes(dname, P)
        achieved = abytes / (avg_ms * 1e-3) / 1e9
        traffic = None  # DRAM bytes of one launch from the committed ncu capture
        try:
            with open(os.path.join(ROOT, "profiles", "traffic_%s.json" % args.workload.replace("plain_", "plain"))) as f:
                tr = json.load(f)
            if dname in tr["stages"]:
                traffic = tr["stages"][dname]["dram_bytes"]
        except (OSError, KeyError, ValueError):
            traffic = None
        cpu = None
        if not args.no_cpu_baseline:
            try:
                cpu = cpu_run(args.workload, args.cpu_seconds)
            except Exception as e:  # reported, not fatal
                cpu = {"value": None, "unit": "particle-steps/s", "cores": 0, "kind": "port",
                       "sample": f"failed: {e}"}
        value = world * npart * args.steps / (t_max * 1e-3)
        line = {
            "metric": "particle-steps/s", "value": value, "unit": "particle-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(workload_config(args.workload),
                           parallelism=f"replicas{world}" if world > 1 else "single"),
            "grid_cell_updates_per_s": world * P["nc"] * args.steps / (t_max * 1e-3),
            "e2e": {"value": world * npart * ke / e2e_max, "unit": "particle-steps/s",
                    "h2d_bytes_per_step": 24 * npart, "d2h_bytes_per_step": 24 * npart},
            "roofline": {"bound": "hbm", "kernel": dname, "achieved": achieved, "peak": hbm,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": traffic, "algorithmic_bytes_per_launch": abytes,
                         "avg_launch_ms": avg_ms},
            "stages_ms_per_step": {k: v["total_ms"] / args.steps for k, v in sorted(stages.items())},
            "profiled_ms_per_step": prof_ms / args.steps,
            "cpu_baseline": cpu,
            "clocks": clk,
            "gpu_launches": st["launches_per_step"] * args.steps,
        }
        print(json.dumps(line), flush=True)
    sim.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

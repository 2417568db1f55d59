"""Precision study of the three fluid-side forms at scale.

TEST INFRASTRUCTURE: compares the CUDA path's precision forms with each other
and with the FP64 oracle (oracle/); it is not part of the library.

Workload (defaults): periodic 256^3 grid, dx = 1, N = 1,000,000 particles at
seeded uniform random positions, 3-point kernel, eta = 1, kT = 0.01,
dt = 0.002, soft repulsion eps = 1, rc = 1.5, 200 steps.  Forms:
  (a) FIXED64      FP32 fields, 64-bit fixed-point spreading (default);
  (b) FLOAT_ATOMIC FP32 fields, FP32 atomic spreading;
  (c) FP64         every fluid quantity in FP64 on the GPU.

1. Oracle pin: for the first K steps, every form is stepped from the oracle's
   state (teacher forcing: same positions, same step index, so the same
   noise) and its displacement, forces and fluid velocity are compared with
   the oracle's.
2. Per-step errors over the whole run: form (c) advances the reference
   trajectory; at every step forms (a) and (b) start from its state and their
   displacement and velocity are compared with its result.  Every
   --oracle-every steps the oracle also takes that step from the same state,
   and all three forms are compared with it, so the oracle pins the forms
   along the whole run (an oracle step at 256^3 / 10^6 particles takes some
   seconds on the host's cores).
3. Reproducibility: every form runs the whole run twice from the same start
   (graph replay); the final positions are compared bit for bit.

Error norms: rel_inf = max|x - ref| / max|ref|, rel_l2 = ||x - ref|| / ||ref||.

    python tests/precision_study.py --json out.json --md out.md
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (ROOT, HERE):
    if p not in sys.path:
        sys.path.insert(0, p)

FORMS = {0: "fixed64", 1: "float_atomic", 2: "fp64"}


def rel_inf(a, b):
    d = np.abs(b).max()
    return float(np.abs(a - b).max() / (d if d > 0 else 1.0))


def rel_l2(a, b):
    d = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (d if d > 0 else 1.0))


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--cells", type=int, default=256)
    ap.add_argument("--np", type=int, default=1_000_000)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--oracle-steps", type=int, default=2)
    ap.add_argument("--oracle-every", type=int, default=10,
                    help="compare every k-th step of the run with the oracle (0: none)")
    ap.add_argument("--v-every", type=int, default=10, help="compare the velocity fields every k steps")
    ap.add_argument("--dt", type=float, default=0.002)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--json", default=None)
    ap.add_argument("--md", default=None)
    a = ap.parse_args(argv)

    import fluam_b200 as fsl
    from fluam_b200 import _lib
    from helpers import uniform_positions
    from oracle import oracle_py as oracle
    _lib.load()
    oracle._load()

    m = a.cells
    L = (float(m),) * 3
    q0 = uniform_positions(a.np, L, a.seed)
    params = dict(eta=1.0, kT=0.01, dt=a.dt, cutoff=1.5, kernel=3)

    def gpu(prec):
        cfg = fsl.make_config((m, m, m), L, pair=fsl.PAIR_SOFT, seed=a.seed, precision=prec, **params)
        return fsl.StokesLimit(cfg, q0)

    t_start = time.time()
    inst = {p: gpu(p) for p in FORMS}
    for g in inst.values():
        g.set_graph(False)

    def teacher_step(g, q, t, with_v=True):
        g.set_positions(q)
        g.set_step(t)
        g.step(1)
        g.sync()
        return g.positions(), g.forces(), (g.velocity64() if with_v else None)

    report = {"workload": {"cells": [m, m, m], "np": a.np, "steps": a.steps, "dt": a.dt,
                           "kernel": 3, "eta": 1.0, "kT": 0.01, "pair": "soft eps=1 rc=1.5",
                           "seed": a.seed},
              "norms": "rel_inf = max|x-ref|/max|ref|; rel_l2 = ||x-ref||/||ref||"}

    # 1. oracle pin
    pin = []
    if a.oracle_steps > 0:
        o = oracle.Oracle(m, m, m, L[0], L[1], L[2], q0, pair=oracle.PAIR_SOFT, seed=a.seed,
                          **{k: params[k] for k in ("eta", "kT", "dt", "cutoff", "kernel")})
        for t in range(a.oracle_steps):
            q = o.positions()
            o.t = t
            t0 = time.time()
            o.step(1)
            t_orc = time.time() - t0
            qo, Fo, vo = o.positions(), o.forces(), o.velocity()
            row = {"step": t, "oracle_seconds": t_orc}
            for p, name in FORMS.items():
                qg, Fg, vg = teacher_step(inst[p], q, t)
                row[name] = {"dq_rel_inf": rel_inf(qg - q, qo - q), "dq_rel_l2": rel_l2(qg - q, qo - q),
                             "F_rel_inf": rel_inf(Fg, Fo), "v_rel_inf": rel_inf(vg, vo),
                             "v_rel_l2": rel_l2(vg, vo)}
            pin.append(row)
            print("oracle pin", json.dumps(row), flush=True)
    report["oracle_pin"] = pin
    o = None
    if a.oracle_every > 0:
        o = oracle.Oracle(m, m, m, L[0], L[1], L[2], q0, pair=oracle.PAIR_SOFT, seed=a.seed,
                          **{k: params[k] for k in ("eta", "kT", "dt", "cutoff", "kernel")})

    # 2. per-step errors of (a), (b) against the FP64 form's trajectory
    per = {"fixed64": [], "float_atomic": []}
    along = []  # every --oracle-every steps: all forms against the oracle
    q = q0.copy()
    for t in range(a.steps):
        orc = o is not None and t % a.oracle_every == 0
        wv = t % a.v_every == 0 or orc
        qc, Fc, vc = teacher_step(inst[2], q, t, wv)
        got = {2: (qc, Fc, vc)}
        for p in (0, 1):
            qg, Fg, vg = teacher_step(inst[p], q, t, wv)
            got[p] = (qg, Fg, vg)
            per[FORMS[p]].append([rel_inf(qg - q, qc - q), rel_l2(qg - q, qc - q),
                                  rel_inf(vg, vc) if wv else np.nan, rel_l2(vg, vc) if wv else np.nan])
        if orc:
            o.set_positions(q)
            o.t = t
            t0 = time.time()
            o.step(1)
            t_orc = time.time() - t0
            qo, Fo, vo = o.positions(), o.forces(), o.velocity()
            row = {"step": t, "oracle_seconds": t_orc}
            for p, name in FORMS.items():
                qg, Fg, vg = got[p]
                row[name] = {"dq_rel_inf": rel_inf(qg - q, qo - q), "F_rel_inf": rel_inf(Fg, Fo),
                             "v_rel_inf": rel_inf(vg, vo)}
            along.append(row)
            print("oracle along", json.dumps(row), flush=True)
        q = qc
        if t % 20 == 0:
            print("step", t, {k: v[-1] for k, v in per.items()}, flush=True)
    summ = {}
    for k, rows in per.items():
        r = np.array(rows)
        summ[k] = {"dq_rel_inf_max": float(r[:, 0].max()), "dq_rel_inf_median": float(np.median(r[:, 0])),
                   "dq_rel_l2_max": float(r[:, 1].max()), "v_rel_inf_max": float(np.nanmax(r[:, 2])),
                   "v_rel_inf_median": float(np.nanmedian(r[:, 2])), "v_rel_l2_max": float(np.nanmax(r[:, 3]))}
    report["per_step_vs_fp64_form"] = summ
    report["oracle_along_run"] = along
    report["oracle_every"] = a.oracle_every
    report["per_step_rows"] = {k: [[None if np.isnan(x) else x for x in row] for row in v]
                               for k, v in per.items()}
    report["velocity_every"] = a.v_every
    report["final_drift_fp64_form"] = float(np.abs(q - q0).max())

    # 3. reproducibility: two free runs with graph replay per form
    repro = {}
    for p, name in FORMS.items():
        outs = []
        for _ in range(2):
            g = inst[p]
            g.set_positions(q0)
            g.set_step(0)
            g.set_graph(True)
            t0 = time.time()
            g.step(a.steps)
            g.sync()
            outs.append((g.positions(), time.time() - t0))
        same = bool(np.array_equal(outs[0][0], outs[1][0]))
        repro[name] = {"bit_identical": same, "max_abs_diff": float(np.abs(outs[0][0] - outs[1][0]).max()),
                       "seconds_per_run": outs[1][1]}
        print("repro", name, repro[name], flush=True)
    report["reproducibility"] = repro
    report["wall_seconds"] = time.time() - t_start
    for g in inst.values():
        g.close()

    if a.json:
        with open(a.json, "w") as f:
            json.dump(report, f, indent=1)
    if a.md:
        with open(a.md, "w") as f:
            f.write(markdown(report))
    return report


def markdown(r):
    w = r["workload"]
    s = [f"# Precision study: {w['cells'][0]}^3 grid, {w['np']:,} particles, {w['steps']} steps\n",
         f"3-point kernel, eta {w['eta']}, kT {w['kT']}, dt {w['dt']}, {w['pair']}, seed {w['seed']}. "
         f"{r['norms']}.\n"]
    if r["oracle_pin"]:
        s.append("\n## Against the FP64 oracle (teacher forced, first steps)\n")
        s.append("| step | form | dq rel_inf | dq rel_l2 | F rel_inf | v rel_inf | v rel_l2 |\n|---|---|---|---|---|---|---|\n")
        for row in r["oracle_pin"]:
            for f in FORMS.values():
                e = row[f]
                s.append(f"| {row['step']} | {f} | {e['dq_rel_inf']:.2e} | {e['dq_rel_l2']:.2e} | "
                         f"{e['F_rel_inf']:.2e} | {e['v_rel_inf']:.2e} | {e['v_rel_l2']:.2e} |\n")
    if r.get("oracle_along_run"):
        s.append(f"\n## Against the FP64 oracle along the run (every {r['oracle_every']} steps of the "
                 "FP64 form's trajectory, teacher forced)\n")
        s.append("| form | steps compared | dq rel_inf max | dq rel_inf median | F rel_inf max | v rel_inf max |\n"
                 "|---|---|---|---|---|---|\n")
        for f in FORMS.values():
            dq = [row[f]["dq_rel_inf"] for row in r["oracle_along_run"]]
            fr = [row[f]["F_rel_inf"] for row in r["oracle_along_run"]]
            vv = [row[f]["v_rel_inf"] for row in r["oracle_along_run"]]
            s.append(f"| {f} | {len(dq)} | {max(dq):.2e} | {float(np.median(dq)):.2e} | {max(fr):.2e} | "
                     f"{max(vv):.2e} |\n")
    s.append("\n## Every step against the FP64 form's trajectory (teacher forced; velocity fields "
             f"every {r['velocity_every']} steps)\n")
    s.append("| form | dq rel_inf max | dq rel_inf median | dq rel_l2 max | v rel_inf max | v rel_inf median | v rel_l2 max |\n|---|---|---|---|---|---|---|\n")
    for f, e in r["per_step_vs_fp64_form"].items():
        s.append(f"| {f} | {e['dq_rel_inf_max']:.2e} | {e['dq_rel_inf_median']:.2e} | {e['dq_rel_l2_max']:.2e} | "
                 f"{e['v_rel_inf_max']:.2e} | {e['v_rel_inf_median']:.2e} | {e['v_rel_l2_max']:.2e} |\n")
    s.append("\n## Run-to-run reproducibility (two free runs, graph replay)\n")
    s.append("| form | bit identical | max abs diff of final positions | seconds per run |\n|---|---|---|---|\n")
    for f, e in r["reproducibility"].items():
        s.append(f"| {f} | {e['bit_identical']} | {e['max_abs_diff']:.2e} | {e['seconds_per_run']:.2f} |\n")
    return "".join(s)


if __name__ == "__main__":
    main()

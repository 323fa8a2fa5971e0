"""Autotuner of the step kernel's launch configuration.

For a workload (topologies, tis_params, temperatures) it times tis_step on
the GPU for every valid configuration of

* CTAs per replica: 1, or 2 (a thread-block cluster; mixed precision, no
  periodic box, no Ewald, >= 64 beads);
* threads per CTA: 128, 256, 512, and 1024 for one mixed-precision CTA
  (the cluster kernel runs 512);
* threads per bead in the force gather: the per-replica rule, 1, 2, 4, 8;
* for two CTAs, whether the noise is drawn in the bonded sweep or in the
  update;
* for batches of different sizes, the launch order (as given, or largest
  first),
* for one CTA, the schedule of the bonded sweep: item chunks dealt to the
  warps in turn, warps taking chunks from a shared counter (longest kinds
  first), or a longest-first deal made once per launch (the cluster kernel
  always deals them in turn),

keeps the fastest, and writes it as a row of the table that tis_init reads
(tuned_launch.tsv next to libtis_b200.so; one row per workload key:
largest replica, replicas, precision, electrostatics, periodic box, rebuild
rule).  Every configuration computes the same forces up to the summation
order of each bead's sum, so the choice is a speed choice only.  The
neighbour rebuild rule (Verlet skin or a fixed cadence) is part of the
model the caller sets; the tuner times the workload as given.

    python -m tis_b200.autotune --workload c1 c3 c3skin c3fp64 c4 c4skin [--out PATH]
"""
from __future__ import annotations

import argparse
import itertools
import json
import os
import statistics

import numpy as np

HEADER = ("# nmp nlane precision i_ele periodic skin | threads group ctas noise_sweep order sweep | "
          "replica-steps/s measured by tis_b200.autotune\n")


def table_path() -> str:
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned_launch.tsv")


def workload_key(systems, par, nrep):
    return (max(int(s["nmp"]) for s in systems), int(sum(nrep)), int(par.get("precision", 0)),
            int(par.get("i_ele", 0)), int(par.get("i_periodic", 0)), int(par.get("n_step_neighbor", 10) <= 0))


def candidates(systems, par, nrep):
    """Every valid launch configuration of the workload."""
    mixed = par.get("precision", 0) == 1
    pair_ok = (mixed and not par.get("i_periodic", 0) and par.get("i_ele", 0) != 2
               and min(int(s["nmp"]) for s in systems) >= 64)
    uneven = len({int(s["nmp"]) for s in systems}) > 1
    out = []
    for ctas in ([1, 2] if pair_ok else [1]):
        threads = [512] if ctas == 2 else ([128, 256, 512] + ([1024] if mixed else []))
        sweeps = [1, 2] if ctas == 2 else [1]
        orders = [1, 2] if uneven else [1]
        for t, g, nz, o, sw in itertools.product(threads, [0, 1, 2, 4, 8], sweeps, orders, [1] if ctas == 2 else [1, 2, 3]):
            out.append(dict(launch_ctas=ctas, launch_threads=t, launch_group=g, launch_noise_sweep=nz,
                            launch_order=o, launch_sweep=sw))
    return out


def time_config(systems, par, temps, nrep, cfg, steps, reps):
    """Median replica-steps/s of `reps` launches of `steps` MD steps."""
    from .engine import Engine, TisError
    try:
        eng = Engine(systems, dict(par, **cfg), temps, nrep=nrep)
    except TisError:
        return None
    try:
        eng.set_state(np.vstack([np.tile(s["xyz"], (r, 1)) for s, r in zip(systems, nrep)]))
        eng.time_integral_pre()
        eng.step(min(steps, 200))
        rates = []
        for _ in range(reps):
            eng.step(steps)
            rates.append(eng.nlane * steps / (eng.last_step_ms() * 1e-3))
        return statistics.median(rates)
    except TisError:
        return None
    finally:
        eng.close()


def tune(systems, par, temps, nrep, steps=500, reps=3):
    """(best configuration, its rate, every configuration's rate)."""
    results = []
    for cfg in candidates(systems, par, nrep):
        r = time_config(systems, par, temps, nrep, cfg, steps, reps)
        if r is not None:
            results.append((cfg, r))
    best = max(results, key=lambda x: x[1])
    return best[0], best[1], results


def format_row(key, cfg, rate):
    return ("%d %d %d %d %d %d %d %d %d %d %d %d %.6g\n" %
            (key + (cfg["launch_threads"], cfg["launch_group"], cfg["launch_ctas"], cfg["launch_noise_sweep"],
                    cfg["launch_order"], cfg["launch_sweep"], rate)))


def merge_rows(path, rows):
    """Writes rows {key: line} into the table, replacing rows of the same key."""
    keep = {}
    if os.path.exists(path):
        for line in open(path):
            if line.startswith("#") or not line.strip():
                continue
            keep[tuple(int(v) for v in line.split()[:6])] = line
    keep.update(rows)
    with open(path, "w") as f:
        f.write(HEADER)
        for k in sorted(keep):
            f.write(keep[k])


def _workload(name):
    from . import synth
    if name == "c1":
        systems, par, temps = synth.workload_c1()
        return systems, par, temps, [1]
    if name in ("c3", "c3skin", "c3fp64"):
        systems, par, temps = synth.workload_c3()
        if name == "c3skin":
            par = dict(par, n_step_neighbor=0)
        if name == "c3fp64":
            par = dict(par, precision=0)
        return systems, par, temps, [len(temps)]
    if name in ("c4", "c4skin"):
        systems, par, temps = synth.workload_c4()
        if name == "c4skin":
            par = dict(par, n_step_neighbor=0)
        return systems, par, temps, [1] * len(systems)
    if name in ("c2", "c2skin"):
        systems, par, temps = synth.workload_c2()
        if name == "c2skin":
            par = dict(par, n_step_neighbor=0)
        return systems, par, temps, [1]
    raise ValueError(name)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", nargs="+", default=["c1", "c3", "c3skin", "c3fp64", "c4", "c4skin"])
    ap.add_argument("--out", default=table_path())
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args()
    rows, report = {}, {}
    for name in args.workload:
        systems, par, temps, nrep = _workload(name)
        steps = args.steps if name != "c2" else max(1, args.steps // 50)
        cfg, rate, results = tune(systems, par, temps, nrep, steps, args.reps)
        key = workload_key(systems, par, nrep)
        rows[key] = format_row(key, cfg, rate)
        ranked = sorted(results, key=lambda x: -x[1])
        report[name] = {"key": key, "best": cfg, "rate": rate, "configs": len(results),
                        "top": [(c, r) for c, r in ranked[:5]], "worst": ranked[-1]}
        print(json.dumps({name: report[name]}), flush=True)
    merge_rows(args.out, rows)


if __name__ == "__main__":
    main()

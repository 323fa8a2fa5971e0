#!/usr/bin/env python
"""Benchmark: replica-steps/s of the batched mixed-precision DT15 path on B200.

Workload (default, --workload c3): 64-replica temperature replica exchange of
one 76-nt DT15 chain (227 beads), Debye-Hueckel at 100 mM, geometric ladder
280-400 K, Langevin dt 0.05, the Verlet-skin rebuild (neigh_margin 8 A), an
exchange attempt every 1000 steps.  One bench *step* is one exchange period:
1000 MD steps of all 64 replicas plus the exchange (energies at own and
partner temperature, Metropolis, label swap, velocity rescale), recorded
once as a CUDA graph (tis_run) and replayed.  value = replica-steps/s of the
whole job (all ranks).  Inputs are synthetic (seeded random-walk chains).

Other fields: e2e (same metric through the C-ABI with host buffers, state
copied in from pinned host memory and out every step), the plain FP64
single-system path (65-bead chain, one replica) as the denominator of the
batched/plain ratio, the roofline of the dominant kernel (lane_kernel<float>)
and the CPU restatement timed on the host cores.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "replica-steps/s: batched FP32 vs plain FP64 on 1 B200, force rel err<1e-5"
UNIT = "replica-steps/s"
PERIOD = 1000


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3", choices=["c3", "c4", "c2", "c5"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--period", type=int, default=None, help="MD steps per bench step (C3: exchange period)")
    ap.add_argument("--precision", type=int, default=None, choices=[0, 1],
                    help="override the workload's arithmetic (0 FP64, 1 mixed)")
    ap.add_argument("--ref-sample", type=int, default=None,
                    help="reference arm: MD steps per replica in one timed step (default: the CPU leg's sample)")
    ap.add_argument("--refine", action="store_true",
                    help="C5: refine the mixed-precision correlated noise once per step (tis_params.hi_refine)")
    ap.add_argument("--neighbor", default=None, choices=["cadence", "skin"],
                    help="neighbour rebuild rule: every 10 steps, or the reference's Verlet skin (neigh_margin "
                         "8 A, time_integral.F90:57-93); default: the cadence where the workload's "
                         "configuration fixes one (C1), else the skin rule")
    ap.add_argument("--quick", action="store_true",
                    help="device timing only (no CPU leg, e2e or plain path): small profiling runs")
    return ap.parse_args()


def neighbor_rule(args):
    """The rebuild rule of the run: --neighbor, else the cadence where the
    workload's configuration fixes one (C1: every 10 steps), else the
    reference's own rule, the Verlet skin.  With the 8 A margin both rules
    keep every pair within the force cutoffs in the lists, so the forces
    differ only by the rounding of the summation order (pairs beyond a
    cutoff add zero); the number of rebuilds is what differs."""
    if args.neighbor:
        return args.neighbor
    return "cadence" if args.workload == "c1" else "skin"


def apply_rule(par, rule):
    if rule == "skin":
        par["n_step_neighbor"] = 0
    return par


RULE_TEXT = {"skin": "Verlet-skin rebuild (neigh_margin 8 A, the reference's rule)",
             "cadence": "rebuild every 10 steps"}


def workload(name):
    from tis_b200 import synth
    if name == "c3":
        systems, par, temps = synth.workload_c3()
        nrep = [len(temps)]
        desc = ("C3: 64-replica temperature REMD of a 76-nt DT15 chain (227 beads), 20 random stem "
                "hbond pairs, Debye-Hueckel 100 mM, ladder 280-400 K, Langevin dt 0.05 tau, "
                "friction 0.5/tau, exchange every 1000 steps")
    elif name == "c4":
        systems, par, temps = synth.workload_c4()
        nrep = [1] * len(systems)
        desc = ("C4: 256 independent DT15 chains, lengths log-uniform 20-400 nt, 30% of residues in "
                "hbond pairs, Debye-Hueckel 150 mM, 300 K, Langevin dt 0.05 tau")
    elif name == "c2":
        systems, par, temps = synth.workload_c2()
        nrep = [1]
        desc = ("C2: 51-nt DT15 chain + 590 ions (Mg 5 mM, K 150 mM, Cl to neutrality) in a 150 A periodic "
                "box, Ewald alpha 0.05, r_c 20 A, |h| <= 10 (4168 k), FP32 forces, 300 K")
    else:
        systems, par, temps = synth.workload_c5()
        nrep = [1] * len(systems)
        desc = ("C5: 32 bead chains, N uniform 100-1000, FENE bonds, WCA between all non-bonded pairs, "
                "Brownian dynamics with the Rotne-Prager tensor (radius 2 A) and its Cholesky factor "
                "refreshed every 10 steps, dt 0.01")
    return systems, par, temps, nrep, desc


# MD steps per bench step, by workload (C3: one exchange period)
PERIODS = {"c3": PERIOD, "c4": PERIOD, "c2": 100, "c5": 10}


def algorithmic_bytes(systems, nrep, exv_pairs, ele_pairs):
    """Bytes per replica-step: 144N (x, v, a FP64 read+write) + 40N (per-bead
    parameters) + 8 per exv and ele pair + 24 per bond + 28 per angle + 84 per
    stack + 128 per hbond (the per-unit figures of the measurement plan)."""
    total = 0.0
    lane = 0
    for s, r in zip(systems, nrep):
        for _ in range(r):
            N = s["nmp"]
            total += (184 * N + 8 * exv_pairs[lane] + 8 * ele_pairs[lane] + 24 * s["nbd"] + 28 * s["nba"]
                      + 84 * s["nst"] + 128 * s["nhb"])
            lane += 1
    return total / lane


def bdhi_bytes(systems, every, mixed):
    """Algorithmic bytes per chain-step of the Brownian-HI path, n = 3N:
    the two matrix-vector products read D (n^2) and the lower half of L
    (n(n+1)/2), FP32 copies in mixed precision, FP64 otherwise; every `every`
    steps the refresh writes D and tril(D), and the blocked Cholesky reads
    and writes the FP64 trailing tiles once per update launch (64 x 64
    tiles; mixed precision updates two panels per launch)."""
    tot = 0.0
    for s in systems:
        n = 3 * s["nmp"]
        T = (n + 63) // 64
        esz = 4 if mixed else 8
        gemv = esz * (n * n + n * (n + 1) / 2)
        tiles = 0
        if mixed:
            for k in range(0, T - 1, 2):
                tiles += T - k - 1                                   # narrow: column tile k + 1
                m = T - k - 2
                tiles += m * (m + 1) // 2                            # wide: tiles right of panel k + 1
        else:
            for k in range(T - 1):
                m = T - k - 1
                tiles += m * (m + 1) // 2
        refresh = esz * n * n + 8 * n * (n + 1) / 2 + 16.0 * 4096 * tiles
        tot += gemv + refresh / every
    return tot / len(systems)


# ------------------------------------------------------------------ CPU leg
def _fleet_worker(jobs, nsteps, variant, barrier, cmd, res):
    """One host process: sets up its share of the replicas once (not timed),
    then for every command steps all of them nsteps after a barrier that
    every process passes together, and reports its start and end times."""
    import numpy as np
    from oracle import oracle as om
    orcs, noise = [], {}
    for sysd, par, T, seed in jobs:
        o = om.Oracle(sysd, dict(par, precision=0), [T], variant=variant)
        o.set_state(sysd["xyz"][None])
        if o.nmp not in noise:
            noise[o.nmp] = np.random.default_rng(seed).normal(size=(nsteps + 1, 1, o.nmp, 3))
        o.set_noise(noise[o.nmp])
        o.time_integral_pre()
        orcs.append(o)
    res.put(("ready", len(orcs)))
    while True:
        n = cmd.get()
        if n is None:
            break
        for o in orcs:
            o.set_noise(noise[o.nmp][1:])
        barrier.wait()
        t0 = time.perf_counter()
        for o in orcs:
            o.step(n)
        t1 = time.perf_counter()
        res.put((t0, t1))


class CpuFleet:
    """The CPU restatement of the path on the host cores: one process per
    core, each owning a fixed share of the replicas (largest first, to the
    least loaded process), set up once.  A pass steps every replica n MD
    steps; its rate is replica-steps over the wall time from the first
    process's start to the last one's end (perf_counter is one clock for
    every process of the host)."""

    def __init__(self, systems, par, temps, nrep, nsteps, variant):
        import multiprocessing as mp
        reps = []
        lane = 0
        for s, r in zip(systems, nrep):
            for _ in range(r):
                reps.append((s, par, temps[lane], 1000 + lane))
                lane += 1
        self.nrep = len(reps)
        self.cores = max(1, min(os.cpu_count() or 1, self.nrep))
        load = [0.0] * self.cores
        share = [[] for _ in range(self.cores)]
        for job in sorted(reps, key=lambda j: -j[0]["nmp"]):
            k = load.index(min(load))
            share[k].append(job)
            load[k] += job[0]["nmp"]
        ctx = mp.get_context("spawn")
        self.barrier = ctx.Barrier(self.cores)
        self.cmd = [ctx.Queue() for _ in range(self.cores)]
        self.res = ctx.Queue()
        self.nsteps = nsteps
        self.procs = [ctx.Process(target=_fleet_worker, args=(share[k], nsteps, variant, self.barrier,
                                                              self.cmd[k], self.res), daemon=True)
                      for k in range(self.cores)]
        for p in self.procs:
            p.start()
        for _ in range(self.cores):
            self.res.get()

    def run(self, n):
        n = min(n, self.nsteps)
        for q in self.cmd:
            q.put(n)
        spans = [self.res.get() for _ in range(self.cores)]
        wall = max(t1 for _, t1 in spans) - min(t0 for t0, _ in spans)
        return self.nrep * n / wall

    def close(self):
        for q in self.cmd:
            q.put(None)
        for p in self.procs:
            p.join(timeout=30)


def cpu_variant():
    """The -O3 -march=native copy built on this host, else the checker build."""
    from oracle import oracle as om
    return ("native", "-O3 -march=native -ffp-contract=off") if om.build_native() else ("checker", "-O2 -ffp-contract=off")


CPU_SAMPLE = {"c3": 2000, "c4": 1000, "c2": 20, "c5": 10}


# ------------------------------------------------------------------ clocks
class Clocks:
    def __init__(self, gpu_index=0):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-i", str(gpu_index), "-lms", "100"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        # wait for the first sample so that the timed region is covered
        t0 = time.time()
        while self.p is not None and time.time() - t0 < 5.0:
            if os.path.getsize(self.f.name) > 0:
                break
            time.sleep(0.05)

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(x, dist, device):
    """The largest value over all ranks (the slowest rank's device time)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank, world, total_ms):
    """Whole-job rate: units every rank processed / the max-over-ranks time."""
    return units_per_rank * world / (total_ms * 1e-3)


def profiled_traffic():
    """DRAM bytes per lane_kernel launch at the bench size, from the committed
    ncu summary (dram__bytes_read.sum + dram__bytes_write.sum), or None."""
    import re
    path = os.path.join(ROOT, "profiles", "lane_kernel_c3_launches.md")
    try:
        m = re.search(r"traffic per launch \| ([\d,]+) B", open(path).read())
        return int(m.group(1).replace(",", "")) if m else None
    except OSError:
        return None


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------------ arms
def run_reference(args, rank, world):
    """The reference's CPU implementation of the path (the C++ restatement:
    no Fortran compiler exists on this image or the GPU host), all host
    cores, one process per core, on a bounded sample of the workload.  Under
    several ranks every rank joins a gloo group and rank 0 alone runs."""
    joined = 1
    if world > 1:
        import datetime
        import torch
        import torch.distributed as tdist
        tdist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        t = torch.ones(1)
        tdist.all_reduce(t)
        joined = int(t.item())
    if rank == 0:
        systems, par, temps, nrep, desc = workload(args.workload)
        apply_rule(par, neighbor_rule(args))
        sample = args.ref_sample or CPU_SAMPLE[args.workload]
        variant, flags = cpu_variant()
        fleet = CpuFleet(systems, par, temps, nrep, sample, variant)
        for _ in range(max(args.warmup, 0)):
            fleet.run(min(sample, 100))
        vals = [fleet.run(sample) for _ in range(args.steps)]
        fleet.close()
        value = statistics.median(vals)
        nlane = sum(nrep)
        line = {
            "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "ranks_joined": joined,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": nlane * sample / value * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded random-walk DT15 chains)",
            "config": {"workload": desc, "neighbor_rule": RULE_TEXT[neighbor_rule(args)],
                       "parallelism": f"{fleet.cores} host processes"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": fleet.cores, "kind": "port",
                             "sample": f"{nlane} replicas x {sample} MD steps per step, median of {args.steps} "
                                       f"(C++ FP64 restatement built {flags}; no Fortran compiler on this "
                                       "image or the GPU host)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as tdist
        tdist.barrier()
        tdist.destroy_process_group()


def run_ours(args, rank, world, local_rank):
    import numpy as np
    cpu_line = None
    period_len = args.period or PERIODS[args.workload]
    if args.workload != "c3":
        args.no_plain = True
    if args.quick:
        args.no_cpu_baseline = True
        args.no_plain = True
    if rank == 0 and not args.no_cpu_baseline:
        # CPU leg first, in spawned processes, before this process touches the
        # GPU; timed exactly as the reference arm times it
        systems, par, temps, nrep, _ = workload(args.workload)
        apply_rule(par, neighbor_rule(args))
        sample = CPU_SAMPLE[args.workload]
        variant, flags = cpu_variant()
        fleet = CpuFleet(systems, par, temps, nrep, sample, variant)
        fleet.run(min(sample, 100))
        v = statistics.median([fleet.run(sample) for _ in range(3)])
        fleet.close()
        cpu_line = {"value": v, "unit": UNIT, "cores": fleet.cores, "kind": "port",
                    "sample": f"{sum(nrep)} replicas x {sample} MD steps, median of 3 after a warm pass "
                              f"(C++ FP64 restatement of the reference loops built {flags}, one process per core)"}
    import torch
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    from tis_b200.engine import Engine

    systems, par, temps, nrep, desc = workload(args.workload)
    apply_rule(par, neighbor_rule(args))
    if args.precision is not None:
        par["precision"] = args.precision
    if args.refine:
        par["hi_refine"] = 1
    remd = args.workload == "c3"
    ladder = None
    if remd and world > 1:
        # one ladder of 64 replicas per GPU, split over the ranks: noise is
        # keyed by the global replica (one seed for all), and each exchange
        # all-gathers replica_energy(2, .) over NCCL (tis_b200.remd)
        from tis_b200 import remd as rx
        from tis_b200 import synth
        nall = len(temps) * world
        tall = synth.temperature_ladder(nall, 280.0, 400.0)
        first, count = rx.ladder_share(nall, world, rank)
        temps = tall[first - 1:first - 1 + count]
        nrep = [count]
        par = dict(par, seed=1234)
        eng = Engine(systems, par, temps, nrep=nrep, ladder=(tall, first))
        ladder = rx.LadderExchange(eng, nall, dist, "cuda")
        desc += f"; the {nall}-replica ladder (280-400 K) split over {world} GPUs, exchanges all-gather energies"
    else:
        par = dict(par, seed=1234 + rank)
        eng = Engine(systems, par, temps, nrep=nrep)
    x0 = np.vstack([np.tile(s["xyz"], (r, 1)) for s, r in zip(systems, nrep)])
    eng.set_state(x0)
    # set-up, outside the timed steps: time_integral_pre (the first list build
    # of every replica, its forces and accelerations), reported apart
    eng.timer_start()
    eng.time_integral_pre()
    first_build_ms = eng.timer_stop()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MiB > 126 MB L2

    def period():
        if ladder is not None:
            eng.step(period_len)
            ladder.exchange()
        elif remd:
            eng.run(1, period_len)          # the period's kernels as one recorded CUDA graph
        else:
            eng.step(period_len)

    for _ in range(args.warmup):
        period()
    nlane = eng.nlane
    if args.workload == "c5":
        bytes_per_rs = bdhi_bytes(systems, par["n_step_hydro"], par.get("precision", 0) == 1)
    else:
        # pair counts for the algorithmic bytes
        exv = [len(eng.exv_list(i + 1)) for i in range(nlane)]
        ele = [len(eng.ele_list(i + 1)[0]) for i in range(nlane)]
        bytes_per_rs = algorithmic_bytes(systems, nrep, exv, ele)

    if dist:
        dist.barrier()
    clocks = Clocks(local_rank) if rank == 0 else None
    times, kern = [], []
    launches0 = eng.launch_count()
    for _ in range(args.steps):
        flush.zero_()                       # L2 flush between timed steps (outside the timed region)
        torch.cuda.synchronize()
        eng.timer_start()
        period()
        times.append(eng.timer_stop())
        kern.append(eng.last_step_ms())
    torch.cuda.synchronize()
    launches = eng.launch_count() - launches0
    ck = clocks.stop() if clocks else None
    total_ms = max_over_ranks(sum(times), dist, "cuda")
    if dist:
        dist.barrier()
    rs_rank = nlane * period_len * args.steps
    rs = rs_rank * world
    value = aggregate_rate(rs_rank, world, total_ms)

    # e2e: host buffers through the C-ABI, copies inside the timed region
    xh, vh, ah = (torch.empty((eng.nbead, 3), dtype=torch.float64).pin_memory() for _ in range(3))
    x, v, a = eng.get_state()
    xh.numpy()[:] = x; vh.numpy()[:] = v; ah.numpy()[:] = a
    e2e_ms = []
    for _ in range(0 if args.quick else args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        eng.timer_start()
        eng.set_state(xh.numpy(), vh.numpy(), ah.numpy())
        period()
        xo, vo, ao = eng.get_state()
        e2e_ms.append(eng.timer_stop())
        xh.numpy()[:] = xo; vh.numpy()[:] = vo; ah.numpy()[:] = ao
    e2e_value = None   # not measured in --quick runs
    if e2e_ms:
        e2e_total = max_over_ranks(sum(e2e_ms), dist, "cuda")
        e2e_value = aggregate_rate(rs_rank, world, e2e_total)
    nbytes = 3 * eng.nbead * 3 * 8

    # C3 under the other neighbour rule, the same periods (no exchange kernel
    # differences): the headline uses neighbor_rule(args)
    other_rule = None
    if remd and ladder is None and not args.quick:
        alt = dict(par, n_step_neighbor=0 if par["n_step_neighbor"] > 0 else 10)
        e2 = Engine(systems, alt, temps, nrep=nrep)
        e2.set_state(x0)
        e2.time_integral_pre()
        for _ in range(args.warmup):
            e2.run(1, period_len)
        t2 = []
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e2.timer_start()
            e2.run(1, period_len)
            t2.append(e2.timer_stop())
        other_rule = {"rule": RULE_TEXT["skin" if alt["n_step_neighbor"] <= 0 else "cadence"],
                      "value": nlane * period_len * args.steps / (sum(t2) * 1e-3), "unit": UNIT,
                      "n_rebuild_per_replica_step": e2.status()["n_rebuild"] / (nlane * period_len * (args.steps + args.warmup))}
        e2.close()

    plain = None
    if rank == 0 and not args.no_plain:
        from tis_b200 import synth
        s1, p1, t1 = synth.workload_c1()
        pe = Engine(s1, dict(p1, precision=0), t1)
        pe.set_state(s1[0]["xyz"])
        pe.time_integral_pre()
        pe.step(2000)
        n_plain = 20000
        pe.timer_start()
        pe.step(n_plain)
        pms = pe.timer_stop()
        plain = {"value": n_plain / (pms * 1e-3), "unit": "steps/s",
                 "config": "C1: 22-nt DT15 chain (65 beads), one replica, FP64 forces and state, DH 150 mM, 300 K",
                 "batched_over_plain": value / world / (n_plain / (pms * 1e-3))}
        pe.close()

    if rank == 0:
        peak, src = peaks()
        kern_ms = statistics.mean(kern)
        achieved = bytes_per_rs * nlane * period_len / (kern_ms * 1e-3) / 1e9
        if args.workload == "c5":
            dtype = ("f64 state and forces; Cholesky trailing updates on tcgen05 tensor cores in split TF32 "
                     "(3 products, f32 accumulation), f64 diagonal and panel tiles; f32 D and L in the step"
                     if par.get("precision", 0) == 1 else "f64")
        else:
            dtype = "f32 forces, f64 accumulation and state" if par.get("precision", 1) == 1 else "f64"
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": dtype,
            "data": "synthetic (seeded random-walk DT15 chains, reference parameter tables)",
            "config": {"workload": desc, "replicas_per_gpu": nlane, "beads_per_replica": int(systems[0]["nmp"]),
                       "md_steps_per_step": period_len, "l2": "flushed between timed steps (256 MiB write)",
                       "neighbor_rule": RULE_TEXT[neighbor_rule(args)],
                       "parallelism": (f"ladder split, {nlane} replicas per GPU, NCCL all-gather at exchanges"
                                       if ladder is not None else f"replicas only, {nlane} lanes per GPU")},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": profiled_traffic() if (args.workload == "c3" and period_len == PERIOD) else None,
                         "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum, one launch "
                                            "(profiles/lane_kernel_c3_launches.md)") if args.workload == "c3"
                                           else "not captured for this workload",
                         "kernel": ("Brownian-HI step: bd_update_kernel matrix-vector products + Cholesky refresh "
                                    "(chol_update_tc_kernel dominant)" if args.workload == "c5"
                                    else "lane_kernel<float>"), "peak_source": src,
                         "bytes_per_replica_step": bytes_per_rs,
                         "note": ("time-averaged over whole refresh periods; achieved counts the algorithmic "
                                  "HBM bytes of the step and of the amortised refresh" if args.workload == "c5" else
                                  "state stays in shared memory across the 1000-step launch; frac > 1 is on-chip reuse")},
            "cpu_baseline": cpu_line,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes},
            "gpu_launches": launches,
            "clocks": ck,
            "plain_fp64": plain,
            "other_neighbor_rule": other_rule,
            "first_build": {"ms": first_build_ms, "what": "time_integral_pre: first neighbour lists, forces and "
                                                          "accelerations of every replica (not in the timed steps)"},
            "status": eng.status(),
        }
        print(json.dumps(line), flush=True)
    eng.close()
    if dist:
        dist.destroy_process_group()


def free_port():
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: relaunch this command under torch.distributed.run
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
               "--master-addr", "127.0.0.1", "--master-port", str(free_port()), os.path.abspath(__file__)]
        sys.exit(subprocess.call(cmd + sys.argv[1:]))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()

"""Host-side logic on CPU: synthetic workload generators (sizes of the
measurement plan), the bench contract helpers, the reference arm's JSON line,
and the multi-rank timing reduction over world_size 2 gloo ranks."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from tis_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


@pytest.mark.parametrize("n", [5, 22, 76])
def test_chain_sizes(n):
    s = synth.dt15_chain(n, 1)
    # linear-S chain of n nt: N = 3n-1, 3n-2 bonds, 4n-5 angles, n-3 consecutive stacks
    assert s["nmp"] == 3 * n - 1
    assert s["nbd"] == 3 * n - 2
    assert s["nba"] == 4 * n - 5
    assert s["nst"] == n - 3
    assert s["ncharge"] == n - 1


def test_workload_shapes():
    sys1, par1, t1 = synth.workload_c1()
    assert sys1[0]["nmp"] == 65 and sys1[0]["nhb"] > 0 and t1 == [300.0]
    sys3, par3, t3 = synth.workload_c3()
    assert sys3[0]["nmp"] == 227 and len(t3) == 64 and par3["precision"] == 1
    ratio = np.array(t3[1:]) / np.array(t3[:-1])
    assert np.allclose(ratio, (400.0 / 280.0) ** (1 / 63))
    assert t3[0] == pytest.approx(280.0) and t3[-1] == pytest.approx(400.0)


def test_generators_are_seeded():
    a = synth.dt15_chain(30, 9)
    b = synth.dt15_chain(30, 9)
    c = synth.dt15_chain(30, 10)
    assert np.array_equal(a["xyz"], b["xyz"]) and a["seq"] == b["seq"]
    assert not np.array_equal(a["xyz"], c["xyz"])


def test_algorithmic_bytes():
    s = synth.dt15_chain(10, 1)
    got = bench.algorithmic_bytes([s], [2], [100, 120], [30, 10])
    base = 184 * s["nmp"] + 24 * s["nbd"] + 28 * s["nba"] + 84 * s["nst"] + 128 * s["nhb"]
    assert got == pytest.approx(base + 8 * (110 + 20))


def test_aggregate_rate_is_whole_job():
    assert bench.aggregate_rate(1000, 4, 2000.0) == pytest.approx(2000.0)
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # each rank times its own independent replicas; the job takes the slowest rank
        t = bench.max_over_ranks(10.0 + rank, dist, "cpu")
        v = bench.aggregate_rate(64 * 1000, world, t)
        q.put((rank, t, v))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, t, v in res:
        assert t == 11.0
        assert v == pytest.approx(2 * 64 * 1000 / 11e-3)


def test_reference_arm_prints_contract_line():
    env = dict(os.environ, PYTHONPATH=ROOT)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "0", "--ref-sample", "5"],
                         check=True, capture_output=True, text=True, timeout=600, env=env).stdout
    line = json.loads(out.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0


def test_bench_gpus_2_spawns_two_ranks():
    """bench.py --gpus 2 without a launcher relaunches itself as two ranks
    (torch.distributed.run); the reference arm joins them in a gloo group and
    rank 0 alone prints the line."""
    env = dict(os.environ, PYTHONPATH=ROOT)
    env.pop("WORLD_SIZE", None)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                          "--steps", "1", "--warmup", "0", "--ref-sample", "5"],
                         check=True, capture_output=True, text=True, timeout=600, env=env).stdout
    lines = [json.loads(x) for x in out.strip().splitlines() if x.startswith("{")]
    assert len(lines) == 1
    assert lines[0]["n_gpus"] == 2 and lines[0]["ranks_joined"] == 2


def test_cpu_fleet_times_only_the_steps():
    """The CPU leg's processes set up their replicas before the timed passes;
    a pass of n steps reports the replica-steps over its wall time."""
    s, par, temps = synth.workload_c1()
    fleet = bench.CpuFleet(s * 1, par, temps * 3, [3], 40, "checker")
    try:
        assert fleet.cores == min(os.cpu_count() or 1, 3)
        r1 = fleet.run(20)
        r2 = fleet.run(40)
        assert r1 > 0 and r2 > 0
    finally:
        fleet.close()

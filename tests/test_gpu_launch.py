"""Launch configurations of the step kernel (tis_params.launch_*, the tuned
table tis_b200/autotune.py writes, the environment overrides): the source of
the configuration in use, and forces and trajectories that stay within the
parity tolerances for every configuration, against the oracle.  The
configurations differ only in the summation order of each bead's force."""
import os

import numpy as np
import pytest

from tis_b200 import autotune, synth
from tis_b200.engine import Engine
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def test_table_caller_and_environment(tis_lib, tmp_path, monkeypatch):
    systems, par, temps = synth.workload_c1()
    key = autotune.workload_key(systems, par, [1])
    table = tmp_path / "t.tsv"
    cfg = dict(launch_threads=256, launch_group=4, launch_ctas=1, launch_noise_sweep=1, launch_order=1,
               launch_sweep=2)
    autotune.merge_rows(str(table), {key: autotune.format_row(key, cfg, 1.0)})
    eng = Engine(systems, dict(par, launch_table=str(table)), temps)
    st = eng.status()
    assert (st["launch_source"], st["threads_per_cta"], st["group"], st["sweep"]) == (1, 256, 4, 2)
    eng.close()
    # a row without the sweep column leaves the schedule to the built-in rule
    old = tmp_path / "old.tsv"
    old.write_text(" ".join(str(v) for v in key) + " 256 4 1 1 1 1.0\n")
    eng = Engine(systems, dict(par, launch_table=str(old)), temps)
    st = eng.status()
    assert (st["launch_source"], st["threads_per_cta"], st["sweep"]) == (1, 256, 1)
    eng.close()
    eng = Engine(systems, dict(par, launch_table=str(table), launch_threads=128), temps)
    st = eng.status()
    assert (st["launch_source"], st["threads_per_cta"], st["group"]) == (2, 128, 4)
    eng.close()
    monkeypatch.setenv("TIS_GROUP", "2")
    eng = Engine(systems, dict(par, launch_table=str(table)), temps)
    assert (eng.status()["launch_source"], eng.status()["group"]) == (2, 2)
    eng.close()
    monkeypatch.delenv("TIS_GROUP")
    eng = Engine(systems, dict(par, launch_table=str(tmp_path / "absent.tsv")), temps)
    assert eng.status()["launch_source"] == 0
    eng.close()


@pytest.mark.parametrize("cfg", [dict(launch_threads=128, launch_group=1), dict(launch_threads=256, launch_group=8),
                                 dict(launch_threads=1024, launch_group=2), dict(launch_ctas=2, launch_group=4,
                                                                                 launch_noise_sweep=2),
                                 dict(launch_threads=512, launch_sweep=2), dict(launch_threads=1024, launch_sweep=2),
                                 dict(launch_threads=512, launch_sweep=3)])
def test_configurations_keep_parity(tis_lib, cfg):
    systems, par, ladder = synth.workload_c3()
    s = systems[0]
    temps = list(ladder[::16])
    nrep, n, nsteps = len(temps), s["nmp"], 25
    eng = Engine([s], dict(par, **cfg), temps, nrep=[nrep])
    noise = np.random.default_rng(3).normal(size=(nsteps + 1, nrep * n, 3))
    eng.set_state(np.tile(s["xyz"], (nrep, 1)))
    eng.set_noise(noise)
    eng.time_integral_pre()
    eng.step(nsteps)
    x, _, _ = eng.get_state()
    orc = Oracle(s, dict(par, precision=0), temps)
    orc.set_state(np.tile(s["xyz"], (nrep, 1, 1)))
    orc.set_noise(noise.reshape(nsteps + 1, nrep, n, 3))
    orc.time_integral_pre()
    orc.step(nsteps)
    assert np.abs(x - orc.get_state()[0].reshape(-1, 3)).max() < 1e-4
    eng.close()


def test_largest_first_order_on_uneven_batch(tis_lib):
    """Batches launch their largest replicas first; the order changes which
    SM runs a replica, not its numbers."""
    systems = [synth.set_friction(synth.dt15_chain(k, 100 + k, hb_fraction=0.3), 0.5) for k in (9, 41, 23, 60)]
    par = synth.dt15_params(ionic_strength=0.15, precision=1)
    out = []
    for order in (1, 2):
        eng = Engine(systems, dict(par, launch_order=order), [300.0] * 4, nrep=[1] * 4)
        assert eng.status()["lane_order"] == order
        eng.set_state(np.vstack([s["xyz"] for s in systems]))
        eng.time_integral_pre()
        eng.step(30)
        out.append(eng.get_state()[0])
        eng.close()
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("threads", [512, 1024])
def test_sweep_schedules_agree_bitwise(tis_lib, threads):
    """The three schedules of the bonded sweep (chunks dealt in turn, taken
    from a shared counter, dealt longest first) hand the same item chunks to
    different warps: every item is computed the same way and every bead's
    sum keeps its order, so the trajectories are bitwise equal."""
    systems, par, ladder = synth.workload_c3()
    s = systems[0]
    temps = list(ladder[::8])
    out = []
    for sweep in (1, 2, 3):
        eng = Engine([s], dict(par, launch_ctas=1, launch_threads=threads, launch_sweep=sweep), temps,
                     nrep=[len(temps)])
        assert eng.status()["sweep"] == sweep
        eng.set_state(np.tile(s["xyz"], (len(temps), 1)))
        eng.time_integral_pre()
        eng.step(200)
        out.append(eng.get_state())
        eng.close()
    for other in out[1:]:
        for a, b in zip(out[0], other):
            assert np.array_equal(a, b)


def test_two_cta_layout_that_does_not_fit_runs_on_one_cta(tis_lib):
    """The largest C4 chain (1,193 beads): its two-CTA layout (each CTA keeps
    every bead's positions plus the next-step copies) needs more than the
    227 KB of shared memory a CTA may use, so the context runs it on one CTA
    even when two are asked for, and the steps run."""
    systems, par, _ = synth.workload_c4()
    s = max(systems, key=lambda x: x["nmp"])
    assert s["nmp"] == 1193
    for cfg in ({}, {"launch_ctas": 2}):
        eng = Engine([s], dict(par, n_step_neighbor=0, **cfg), [300.0])
        assert eng.status()["ctas_per_lane"] == 1
        eng.set_state(s["xyz"])
        assert eng.time_integral_pre() >= 0
        assert eng.run(1, 20, exchange=False) >= 0
        x, _, _ = eng.get_state()
        assert np.isfinite(x).all()
        eng.close()

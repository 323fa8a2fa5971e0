"""tis_run: the time-integral loop of mloop_simulator (mloop_simulator.F90:
123-150) with the replica exchange of time_integral_post
(time_integral_post.F90:275-363), one period recorded as a CUDA graph and
replayed.  The graph replays the same kernels with the same arguments as
the per-call path (tis_step + tis_replica_exchange with counter-based
uniforms), so the two runs must agree bit for bit: positions, velocities,
accelerations, labels, step counters and rebuild records.  Checked on the
64-replica C3 ensemble (both rebuild rules, FP64 one CTA per replica and
mixed two-CTA clusters), a replayed graph, a re-recorded one (another
period length), an uneven batch without exchanges, an Ewald box, and the
refusals.
"""
import numpy as np
import pytest

from tis_b200 import synth
from tis_b200.engine import Engine, TisError

pytestmark = pytest.mark.gpu

TIS_E_ARG, TIS_E_UNSUPPORTED = -1, -7


def c3_engine(precision, pair, skin):
    systems, par, temps = synth.workload_c3()
    par = dict(par, precision=precision, launch_ctas=2 if pair else 1,
               n_step_neighbor=0 if skin else 10)
    eng = Engine(systems, par, temps, nrep=[len(temps)])
    assert eng.status()["ctas_per_lane"] == (2 if pair else 1)
    eng.set_state(np.tile(systems[0]["xyz"], (len(temps), 1)))
    assert eng.time_integral_pre() >= 0
    return eng


def snapshot(eng):
    x, v, a = eng.get_state()
    return x, v, a, eng.labels(), eng.steps(), [eng.rebuild_info(k + 1) for k in range(eng.nlane)]


def assert_same(s1, s2):
    for u, w in zip(s1[:3], s2[:3]):
        assert np.array_equal(u, w)
    assert np.array_equal(s1[3], s2[3])
    assert np.array_equal(s1[4], s2[4])
    assert s1[5] == s2[5]


@pytest.mark.parametrize("precision,pair,skin", [(0, False, True), (1, True, True), (1, True, False)])
def test_run_matches_step_and_exchange(tis_lib, precision, pair, skin):
    a = c3_engine(precision, pair, skin)   # per call
    b = c3_engine(precision, pair, skin)   # recorded graph
    for nper, nstep in ((3, 200), (2, 200), (2, 70)):   # record, replay, record again
        l0a, l0b = a.launch_count(), b.launch_count()
        for _ in range(nper):
            assert a.step(nstep) >= 0
            a.replica_exchange(count=False)
        assert b.run(nper, nstep) >= 0
        assert a.launch_count() - l0a == b.launch_count() - l0b
        assert_same(snapshot(a), snapshot(b))
    # some exchanges were accepted, so the labels moved
    assert not np.array_equal(a.labels(), np.arange(1, a.nlane + 1))
    a.close()
    b.close()


def test_run_batch_without_exchange(tis_lib):
    systems, par, temps = synth.workload_c4(nchain=12)
    par = dict(par, n_step_neighbor=0)
    engs = []
    for _ in range(2):
        e = Engine(systems, par, temps)
        e.set_state(np.vstack([s["xyz"] for s in systems]))
        assert e.time_integral_pre() >= 0
        engs.append(e)
    a, b = engs
    for _ in range(3):
        assert a.step(150) >= 0
    assert b.run(3, 150, exchange=False) >= 0
    assert_same(snapshot(a), snapshot(b))
    # a batch of several topologies has no temperature ladder to exchange
    with pytest.raises(TisError) as ei:
        b.run(1, 10, exchange=True)
    assert ei.value.code == TIS_E_UNSUPPORTED
    a.close()
    b.close()


def test_run_ewald(tis_lib):
    systems, par, temps = synth.workload_c2()
    par = dict(par, n_step_neighbor=0)
    engs = []
    for _ in range(2):
        e = Engine(systems, par, temps)
        e.set_state(systems[0]["xyz"])
        assert e.time_integral_pre() >= 0
        engs.append(e)
    a, b = engs
    for _ in range(2):
        assert a.step(20) >= 0
    assert b.run(2, 20, exchange=False) >= 0
    assert_same(snapshot(a), snapshot(b))
    a.close()
    b.close()


def test_run_refusals(tis_lib):
    eng = c3_engine(1, True, True)
    n = eng.nlane * eng.systems[0]["nmp"]
    with pytest.raises(TisError) as ei:
        eng.run(1, 0)
    assert ei.value.code == TIS_E_ARG
    eng.set_noise(np.zeros((4, n, 3)))
    with pytest.raises(TisError) as ei:
        eng.run(1, 4)
    assert ei.value.code == TIS_E_UNSUPPORTED
    eng.set_noise(None)
    assert eng.run(1, 4) >= 0
    eng.close()
    systems, par, temps = synth.workload_c5(nchain=2)
    bd = Engine(systems, par, temps)
    with pytest.raises(TisError) as ei:
        bd.run(1, 10, exchange=False)
    assert ei.value.code == TIS_E_UNSUPPORTED
    bd.close()

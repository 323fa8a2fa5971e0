"""The reference's only live neighbour-list rule, the Verlet skin
(time_integral.F90:57-93; a fixed cadence is refused at
setp_md_info.F90:474-476): a replica rebuilds its lists when the two largest
displacements since its last rebuild add up to more than neigh_margin, and
then clears the displacements.  GPU against the oracle with the noise
injected identically, through the C-ABI, on the 227-bead C3 chain.

Checked: the step of every rebuild of every replica (one-step calls), the
rebuild count and last rebuild step after one long launch, the long launch
against the one-step calls (bit-exact), lists after the run (bit-exact,
FP64), and positions: FP64 1e-8 A, mixed 1e-4 A (1e-2 A after the 1,500
steps of the 64-replica run, where the dynamics has amplified the mixed
path's force differences).  One CTA per replica and
the two-CTA cluster are both run.  A margin of 2 A makes the rule fire every
~85 steps; the default 8 A fires about once per 1,300 steps, which the
64-replica run covers.
"""
import numpy as np
import pytest

from tis_b200 import synth
from tis_b200.engine import Engine
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

POS_TOL = {0: 1e-8, 1: 1e-4}


def engine(system, par, temps, pair):
    eng = Engine([system], dict(par, launch_ctas=2 if pair else 1), temps, nrep=[len(temps)])
    assert eng.status()["ctas_per_lane"] == (2 if pair else 1)
    return eng


def skin_setup(margin, precision, nrep):
    systems, par, temps = synth.workload_c3()
    s = systems[0]
    par = dict(par, precision=precision, n_step_neighbor=0, neigh_margin=margin)
    temps = list(temps[::max(1, len(temps) // nrep)])[:nrep]
    return s, par, temps


def rebuild_table(obj, nrep):
    return [obj.rebuild_info(k + 1) for k in range(nrep)]


@pytest.mark.parametrize("precision,pair", [(0, False), (1, False), (1, True)])
def test_skin_rebuild_steps_match_oracle(tis_lib, precision, pair):
    nsteps, nrep = 300, 4
    s, par, temps = skin_setup(2.0, precision, nrep)
    noise = np.random.default_rng(21).normal(size=(nsteps + 1, nrep * s["nmp"], 3))
    x0 = np.tile(s["xyz"], (nrep, 1))
    # one launch of nsteps
    eng = engine(s, par, temps, pair)
    eng.set_state(x0)
    eng.set_noise(noise)
    assert eng.time_integral_pre() >= 0
    assert eng.step(nsteps) >= 0
    x_long, v_long, _ = eng.get_state()
    long_info = rebuild_table(eng, nrep)
    eng.close()
    # one-step calls, recording the step of every rebuild
    eng = engine(s, par, temps, pair)
    eng.set_state(x0)
    orc = Oracle(s, dict(par, precision=0), temps)
    orc.set_state(x0.reshape(nrep, -1, 3))
    gpu_steps = [[] for _ in range(nrep)]
    orc_steps = [[] for _ in range(nrep)]
    for k in range(nsteps + 1):
        eng.set_noise(noise[k:k + 1])
        orc.set_noise(noise[k:k + 1].reshape(1, nrep, s["nmp"], 3))
        if k == 0:
            assert eng.time_integral_pre() >= 0
            assert orc.time_integral_pre() == 0
            g0, o0 = rebuild_table(eng, nrep), rebuild_table(orc, nrep)
            continue
        eng.step(1)
        orc.step(1)
        for r, (g, o) in enumerate(zip(rebuild_table(eng, nrep), rebuild_table(orc, nrep))):
            if g[0] != (g0[r][0] + len(gpu_steps[r])):
                gpu_steps[r].append(g[1])
            if o[0] != (o0[r][0] + len(orc_steps[r])):
                orc_steps[r].append(o[1])
    assert gpu_steps == orc_steps
    assert all(len(v) >= 2 for v in gpu_steps), gpu_steps     # the rule fired several times
    x, v, _ = eng.get_state()
    xr, vr, _ = orc.get_state()
    assert np.abs(x - xr.reshape(-1, 3)).max() < POS_TOL[precision]
    # the long launch is the same computation as the one-step calls
    assert np.array_equal(x_long, x) and np.array_equal(v_long, v)
    assert long_info == rebuild_table(eng, nrep) == rebuild_table(orc, nrep)
    if precision == 0:
        # lists of the last rebuild, from the same positions
        for r in range(nrep):
            assert np.array_equal(eng.exv_list(r + 1), orc.exv_list(r + 1))
            assert np.array_equal(eng.ele_list(r + 1)[0], orc.ele_list(r + 1)[0])
    eng.close()


@pytest.mark.parametrize("precision,pair", [(0, False), (1, True)])
def test_skin_default_margin_64_replicas(tis_lib, precision, pair):
    """The C3 ensemble (64 replicas, 280-400 K) with the default 8 A margin,
    1,500 steps in launches of 500: per-replica rebuild counts and steps and
    the positions against the oracle."""
    nsteps, chunk, nrep = 1500, 500, 64
    s, par, temps = skin_setup(8.0, precision, nrep)
    eng = engine(s, par, temps, pair)
    orc = Oracle(s, dict(par, precision=0), temps)
    x0 = np.tile(s["xyz"], (nrep, 1))
    eng.set_state(x0)
    orc.set_state(x0.reshape(nrep, -1, 3))
    rng = np.random.default_rng(8)
    for c in range(nsteps // chunk):
        noise = rng.normal(size=(chunk + (1 if c == 0 else 0), nrep * s["nmp"], 3))
        eng.set_noise(noise)
        orc.set_noise(noise.reshape(noise.shape[0], nrep, s["nmp"], 3))
        if c == 0:
            eng.time_integral_pre()
            orc.time_integral_pre()
        eng.step(chunk)
        orc.step(chunk)
    g, o = rebuild_table(eng, nrep), rebuild_table(orc, nrep)
    assert g == o
    assert sum(n for n, _ in g) - nrep >= 32     # skin rebuilds beyond time_integral_pre's
    x, _, _ = eng.get_state()
    xr, _, _ = orc.get_state()
    # over 1,500 steps the dynamics amplifies the mixed path's ~1e-7 relative
    # force differences (measured up to ~1e-3 A on one of the 64 replicas);
    # the rebuild records above are the point of this test
    tol = POS_TOL[0] if precision == 0 else 1e-2
    assert np.abs(x - xr.reshape(-1, 3)).max() < tol
    eng.close()


@pytest.mark.parametrize("pair", [False, True])
def test_time_integral_exchange_flags(tis_lib, pair):
    """tis_time_integral: replicas stop at their exchange step and set their
    flag (time_integral.F90:134,460-465); each replica's state equals the
    same replica stepped exactly that far (counter-based noise is keyed by
    replica and step, so the other replicas do not matter)."""
    systems, par, temps = synth.workload_c3()
    s = systems[0]
    temps = list(temps[::16])
    nrep = len(temps)
    x0 = np.tile(s["xyz"], (nrep, 1))
    stops = np.array([5, 8, 8, 12], dtype=np.int64)
    eng = engine(s, par, temps, pair)
    eng.set_state(x0)
    eng.time_integral_pre()
    flags = np.zeros(nrep, dtype=np.int32)
    flags[2] = 1                                   # waits from the start
    eng.time_integral(20, flags, stops)
    assert list(flags) == [1, 1, 1, 1]
    assert list(eng.steps()) == [5, 8, 0, 12]
    xa, va, _ = eng.get_state()
    eng.close()
    ref = engine(s, par, temps, pair)
    ref.set_state(x0)
    ref.time_integral_pre()
    xb0, _, _ = ref.get_state()
    n = s["nmp"]
    lane = lambda a, r: a[r * n:(r + 1) * n]
    assert np.array_equal(lane(xa, 2), lane(xb0, 2))
    done = 0
    for r, stop in ((0, 5), (1, 8), (3, 12)):
        ref.step(stop - done)
        done = stop
        xb, vb, _ = ref.get_state()
        assert np.array_equal(lane(xa, r), lane(xb, r)), r
        assert np.array_equal(lane(va, r), lane(vb, r)), r
    ref.close()

"""Parity at the benched sizes, through the C-ABI, against the oracle.

* C3 (64 replicas of the 227-bead chain, 280-400 K): after one exchange
  period run exactly as the bench runs it (counter-based noise, 1,000 steps,
  an exchange on the device), the next step rebuilds the lists inside the
  step kernel (one CTA per replica, FP64 and mixed, and the two-CTA cluster):
  every replica's exv and ele lists (pairs, order, coef_ele) are bit-exact
  with the oracle's from the same positions, and the step's forces (read
  back as m a with the noise of that step set to zero) agree with the
  oracle's on the same positions and lists: FP64 relative 1e-9, mixed 1e-5
  of max(|F_i|, median |F|).
* C3, 1,000 steps with injected noise and an exchange with injected
  uniforms at step 500: labels equal, positions FP64 1e-10 A, mixed 1e-4 A;
  DE_MAX clamp counts equal in FP64 and within 10 % (or 2) in mixed
  precision, whose FP32 forces can fall either side of the clamp.
* C4 (256 chains, 20-400 nt): lists of every chain bit-exact and forces of
  every chain within the tolerances above (FP64: the chains up to 1,100
  beads; larger ones do not fit one CTA's shared memory in FP64 and are
  refused).  Chains above 512 beads keep their bit matrices in global
  memory.
"""
import numpy as np
import pytest

from tis_b200 import synth
from tis_b200.engine import Engine
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

FORCE_TOL = {0: 1e-9, 1: 1e-5}


def rel_force_err(f, ref):
    mag = np.linalg.norm(ref, axis=1)
    den = np.maximum(mag, np.median(mag))
    return np.max(np.linalg.norm(f - ref, axis=1) / den)


def engine(systems, par, temps, nrep, pair):
    eng = Engine(systems, dict(par, launch_ctas=2 if pair else 1), temps, nrep=nrep)
    return eng


@pytest.mark.parametrize("precision,pair", [(0, False), (1, False), (1, True)])
def test_c3_lists_and_forces_every_replica(tis_lib, precision, pair):
    systems, par, ladder = synth.workload_c3()
    s = systems[0]
    par = dict(par, precision=precision)
    nrep, n = len(ladder), s["nmp"]
    eng = engine(systems, par, ladder, [nrep], pair)
    assert eng.status()["ctas_per_lane"] == (2 if pair else 1)
    eng.set_state(np.tile(s["xyz"], (nrep, 1)))
    eng.time_integral_pre()
    eng.step(1000)
    eng.replica_exchange(count=False)
    x0, _, _ = eng.get_state()
    labels = eng.labels()
    eng.set_noise(np.zeros((1, nrep * n, 3)))
    assert eng.step(1) >= 0                       # step 1001 rebuilds (cadence 10)
    x1, _, a1 = eng.get_state()
    temps = [ladder[lab - 1] for lab in labels]
    orc = Oracle(s, dict(par, precision=0), temps)
    orc.set_state(x0.reshape(nrep, n, 3))
    orc.neighbor()
    orc.set_state(x1.reshape(nrep, n, 3))         # the step's forces use the lists of x0
    mass = np.asarray(s["cmass"], dtype=np.float64)[:, None]
    worst = 0.0
    for r in range(nrep):
        assert np.array_equal(eng.exv_list(r + 1), orc.exv_list(r + 1)), r
        gl, gc = eng.ele_list(r + 1)
        ol, oc = orc.ele_list(r + 1)
        assert np.array_equal(gl, ol) and np.array_equal(gc, oc), r
        fr, _ = orc.force(r + 1)
        f = a1[r * n:(r + 1) * n] * mass
        worst = max(worst, rel_force_err(f, fr))
    assert worst < FORCE_TOL[precision], worst
    eng.close()


@pytest.mark.parametrize("precision,pair", [(0, False), (1, True)])
def test_c3_trajectory_1000_steps_with_exchange(tis_lib, precision, pair):
    systems, par, ladder = synth.workload_c3()
    s = systems[0]
    par = dict(par, precision=precision)
    nrep, n = len(ladder), s["nmp"]
    eng = engine(systems, par, ladder, [nrep], pair)
    orc = Oracle(s, dict(par, precision=0), ladder)
    x0 = np.tile(s["xyz"], (nrep, 1))
    eng.set_state(x0)
    orc.set_state(x0.reshape(nrep, n, 3))
    rng = np.random.default_rng(17)
    chunk = 100
    for c in range(10):
        noise = rng.normal(size=(chunk + (1 if c == 0 else 0), nrep * n, 3))
        eng.set_noise(noise)
        orc.set_noise(noise.reshape(noise.shape[0], nrep, n, 3))
        if c == 0:
            eng.time_integral_pre()
            orc.time_integral_pre()
        eng.step(chunk)
        orc.step(chunk)
        if c == 4:
            u = rng.uniform(size=nrep)
            assert eng.replica_exchange(u) == orc.replica_exchange(u)
            assert np.array_equal(eng.labels(), orc.labels())
    x, v, _ = eng.get_state()
    xr, vr, _ = orc.get_state()
    tol = 1e-10 if precision == 0 else 1e-4
    assert np.abs(x - xr.reshape(-1, 3)).max() < tol
    assert np.abs(v - vr.reshape(-1, 3)).max() < 10 * tol
    g, o = eng.status()["n_clamp"], orc.nclamp()
    if precision == 0:
        assert g == o
    else:
        assert abs(g - o) <= max(2, 0.1 * o), (g, o)
    eng.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_c4_every_chain(tis_lib, precision):
    systems, par, temps = synth.workload_c4()
    if precision == 0:
        # an FP64 replica keeps its state in one CTA's shared memory: the
        # library refuses chains above ~1,100 beads (TIS_E_UNSUPPORTED)
        keep = [k for k, s in enumerate(systems) if s["nmp"] <= 1100]
        systems, temps = [systems[k] for k in keep], [temps[k] for k in keep]
    par = dict(par, precision=precision)
    assert max(s["nmp"] for s in systems) > 512       # global-memory bit matrices
    eng = Engine(systems, par, temps, nrep=[1] * len(systems))
    eng.set_state(np.vstack([s["xyz"] for s in systems]))
    eng.neighbor()
    worst = 0.0
    for k, s in enumerate(systems):
        orc = Oracle(s, dict(par, precision=0), [temps[k]])
        orc.set_state(s["xyz"][None])
        orc.neighbor()
        assert np.array_equal(eng.exv_list(k + 1), orc.exv_list()), k
        gl, gc = eng.ele_list(k + 1)
        ol, oc = orc.ele_list()
        assert np.array_equal(gl, ol) and np.array_equal(gc, oc), k
        assert np.array_equal(eng.hb_list(k + 1), orc.hb_list()), k
        f, _ = eng.force(k + 1)
        fr, _ = orc.force()
        err = rel_force_err(f, fr)
        if err > worst:
            mag = np.linalg.norm(fr, axis=1)
            b = int(np.argmax(np.linalg.norm(f - fr, axis=1) / np.maximum(mag, np.median(mag))))
            where = (k, s["nmp"], b, float(mag[b]), float(np.median(mag)))
            worst = err
        orc.close()
    assert worst < FORCE_TOL[precision], (worst, "chain, beads, bead, |F|, median |F|", where)
    eng.close()

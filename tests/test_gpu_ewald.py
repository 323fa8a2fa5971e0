"""Ewald electrostatics on the GPU (force_ele_coulomb_ewld.F90, mloop_ewld.F90)
against the CPU restatement, through the C-ABI.

Two systems: a small neutral box (40 A, alpha 0.2, |h| <= 8) and the
explicit-ion workload (51-nt chain + 590 ions in a 150 A box, alpha 0.05,
r_c 20 A, |h| <= 10: 4168 k vectors).  Tolerances as in the other parity
tests: lists bit-exact; FP64 forces and energies relative 1e-9; mixed
forces 1e-5 of max(|F_i|, median |F|); trajectories with injected noise
FP64 1e-8 A, mixed 1e-4 A.
"""
import numpy as np
import pytest

from tis_b200 import synth
from tis_b200.engine import Engine
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def rel_force_err(f, ref):
    mag = np.linalg.norm(ref, axis=1)
    den = np.maximum(mag, np.median(mag))
    return np.max(np.linalg.norm(f - ref, axis=1) / den)


def small_box():
    s = synth.set_friction(synth.dt15_chain(12, 3, stem=3), 0.5)
    s = synth.add_ions(s, 40.0, {"Mg": 2, "K": 10, "Cl": 3}, 9, clash=5.0)
    par = synth.dt15_params(i_periodic=1, psize=(40.0, 40.0, 40.0), i_ele=2, ewld_alpha=0.2, ewld_hmax=8.0,
                            cutoff_ele=19.9)
    return s, par


def c2_box():
    systems, par, _ = synth.workload_c2()
    return systems[0], par


SYSTEMS = {"small": small_box, "c2": c2_box}


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", list(SYSTEMS))
def test_ewald_lists_forces_energy(tis_lib, name, precision):
    s, par = SYSTEMS[name]()
    par = dict(par, precision=precision)
    eng = Engine([s], par, [300.0])
    orc = Oracle(s, dict(par, precision=0), [300.0])
    eng.set_state(s["xyz"])
    orc.set_state(s["xyz"][None])
    eng.neighbor()
    orc.neighbor()
    assert np.array_equal(eng.exv_list(), orc.exv_list())
    ge, gc = eng.ele_list()
    oe, oc = orc.ele_list()
    assert np.array_equal(ge, oe) and len(oe) > 0
    f, _ = eng.force()
    fr, _ = orc.force()
    err = rel_force_err(f, fr)
    assert err < (1e-9 if precision == 0 else 1e-5), err
    # the reciprocal part alone is a sizeable share of the electrostatic force
    fe = orc.force_term("ewald")
    assert np.abs(fe).max() > 1e-3
    if precision == 0:
        e = eng.energy()
        er = orc.energy(reuse_hb=True)
        assert abs(e[7] - er[7]) <= 1e-9 * max(1.0, abs(er[7]))
        assert np.allclose(e, er, rtol=1e-9, atol=1e-9)
    eng.close()


@pytest.mark.parametrize("precision,tol", [(0, 1e-8), (1, 1e-4)])
def test_ewald_trajectory_injected_noise(tis_lib, precision, tol):
    s, par = small_box()
    par = dict(par, precision=precision)
    nsteps = 12
    eng = Engine([s], par, [300.0])
    orc = Oracle(s, dict(par, precision=0), [300.0])
    eng.set_state(s["xyz"])
    orc.set_state(s["xyz"][None])
    noise = np.random.default_rng(21).normal(size=(nsteps + 1, s["nmp"], 3))
    eng.set_noise(noise)
    orc.set_noise(noise.reshape(nsteps + 1, 1, s["nmp"], 3))
    assert eng.time_integral_pre() >= 0
    assert orc.time_integral_pre() == 0
    eng.step(nsteps)
    orc.step(nsteps)
    x, v, a = eng.get_state()
    xr, vr, ar = orc.get_state()
    assert np.abs(x - xr.reshape(-1, 3)).max() < tol
    assert np.abs(v - vr.reshape(-1, 3)).max() < 10 * tol
    eng.close()


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("skin", [False, True])
def test_ewald_long_call_equals_one_step_calls(tis_lib, precision, skin):
    """A call of n steps runs the x update of each next step in the launch of
    the forces; it must give the one-step calls' state bit for bit (with
    the skin rule: through several rebuilds)."""
    s, par = c2_box()
    par = dict(par, precision=precision, n_step_neighbor=0 if skin else 10, neigh_margin=2.0 if skin else 8.0)
    nsteps = 60
    out = []
    for calls in ([nsteps], [1] * nsteps):
        eng = Engine([s], par, [300.0])
        eng.set_state(s["xyz"])
        assert eng.time_integral_pre() >= 0
        for n in calls:
            assert eng.step(n) >= 0
        out.append(eng.get_state() + (eng.get_pxyz(), eng.rebuild_info(1)))
        eng.close()
    for u, w in zip(out[0][:4], out[1][:4]):
        assert np.array_equal(u, w)
    assert out[0][4] == out[1][4]
    if skin:
        assert out[0][4][0] >= 3


def test_ewald_rejects_non_cubic_box(tis_lib):
    from tis_b200.engine import TisError
    s, par = small_box()
    par = dict(par, psize=(40.0, 40.0, 41.0))
    with pytest.raises(TisError):
        Engine([s], par, [300.0])

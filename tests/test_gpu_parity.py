"""Parity of the CUDA path (through the C-ABI) against the CPU restatement of
the reference (oracle/), on seeded synthetic DT15 systems.

Tolerances:
* neighbour lists: bit-exact (pairs, order, mirror index, coef_ele);
* FP64 path forces / energies: relative 1e-9 (different summation order and
  CUDA vs glibc transcendentals);
* mixed path (FP32 terms, FP64 accumulation): per-bead force error
  <= 1e-5 * max(|F_ref,i|, median_i |F_ref,i|);
* trajectories with injected noise: FP64 1e-8 A after 20 steps, mixed 1e-4 A.
"""
import numpy as np
import pytest

from tis_b200 import synth
from tis_b200.engine import Engine
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

FORCE_TOL_MIXED = 1e-5
FORCE_TOL_FP64 = 1e-9


def rel_force_err(f, ref):
    mag = np.linalg.norm(ref, axis=1)
    den = np.maximum(mag, np.median(mag))
    return np.max(np.linalg.norm(f - ref, axis=1) / den)


def c1_system(seed=1):
    return synth.set_friction(synth.dt15_chain(22, seed, stem=6), 0.5)


def hairpin(seed=1, n=22, stem=6):
    s = synth.set_friction(synth.dt15_chain(n, seed, stem=stem), 0.5)
    return synth.hairpin_coords(s, stem, seed=seed)


def dense(seed=5, n=30):
    return synth.set_friction(synth.dt15_chain(n, seed, min_dist=2.6, confine=10.0), 0.5)


def ninfo_hairpin():
    """tests/golden/hairpin_tertiary.{cg.pdb,ninfo} read through
    tis_b200.ninfo: tertiary stacks, 'T' hydrogen bonds, an ion unit."""
    import os
    from tis_b200 import ninfo
    g = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "hairpin_tertiary")
    return ninfo.load(g + ".cg.pdb", g + ".ninfo", i_fric=0, fric_const=0.5)


def periodic_ions(seed=7):
    s = synth.set_friction(synth.dt15_chain(12, seed, stem=3), 0.5)
    s = synth.add_ions(s, 40.0, {"Mg": 2, "K": 12, "Cl": 5}, seed + 1, clash=4.0)
    return s


SYSTEMS = {
    "c1_walk": (c1_system, {}),
    "hairpin_tertiary": (synth.hairpin_tertiary, {}),
    "ninfo_hairpin": (ninfo_hairpin, {}),
    # DT19 semi-explicit Mg: NHT19 exv rules, Manning charges, Mg-P table
    "dt19_mg": (synth.dt19_mg_system, dict(_base=synth.dt19_params, i_periodic=1, psize=(80.0, 80.0, 80.0),
                                           ionic_strength=0.1)),
    "hairpin_coulomb": (hairpin, dict(i_ele=3, cutoff_ele=60.0)),
    "hairpin": (hairpin, {}),
    "dense": (dense, {}),
    "periodic_ions": (periodic_ions, dict(i_periodic=1, psize=(40.0, 40.0, 40.0))),
}


def make_pair(name, precision, nrep=1, temps=None, **over):
    fn, extra = SYSTEMS[name]
    s = fn()
    extra = dict(extra)
    base = extra.pop("_base", synth.dt15_params)
    kw = dict(ionic_strength=0.15, precision=precision)
    kw.update(extra)
    kw.update(over)
    par = base(**kw)
    temps = temps or [300.0] * nrep
    eng = Engine([s], par, temps, nrep=[nrep])
    orc = Oracle(s, par, temps)
    x = np.tile(s["xyz"], (nrep, 1))
    eng.set_state(x)
    orc.set_state(x.reshape(nrep, -1, 3))
    return s, par, eng, orc


@pytest.mark.parametrize("name", list(SYSTEMS))
def test_neighbor_lists_bit_exact(tis_lib, name):
    s, par, eng, orc = make_pair(name, 0)
    eng.neighbor()
    orc.neighbor()
    ge, oe = eng.exv_list(), orc.exv_list()
    assert ge.shape == oe.shape and len(oe) > 0
    assert np.array_equal(ge, oe)
    gl, gc = eng.ele_list()
    ol, oc = orc.ele_list()
    assert np.array_equal(gl, ol)
    assert np.array_equal(gc, oc)      # bit-exact coef_ele
    assert np.array_equal(eng.hb_list(), orc.hb_list())
    if par["i_periodic"]:
        assert np.array_equal(eng.get_pxyz(), orc.get_pxyz().reshape(-1, 3))


@pytest.mark.parametrize("name", list(SYSTEMS))
def test_force_fp64(tis_lib, name):
    s, par, eng, orc = make_pair(name, 0)
    eng.neighbor(); orc.neighbor()
    f, _ = eng.force()
    fr, _ = orc.force()
    assert rel_force_err(f, fr) < FORCE_TOL_FP64
    # Newton's third law holds pair by pair: total force ~ 0
    assert np.abs(f.sum(axis=0)).max() < 1e-8 * max(1.0, np.abs(fr).max())


@pytest.mark.parametrize("name", list(SYSTEMS))
def test_force_mixed(tis_lib, name):
    s, par, eng, orc = make_pair(name, 1)
    eng.neighbor(); orc.neighbor()
    f, _ = eng.force()
    fr, _ = orc.force()
    err = rel_force_err(f, fr)
    assert err < FORCE_TOL_MIXED, err


@pytest.mark.parametrize("name", ["c1_walk", "hairpin", "dense", "hairpin_tertiary", "hairpin_coulomb",
                                  "ninfo_hairpin", "dt19_mg"])
def test_energy_fp64(tis_lib, name):
    s, par, eng, orc = make_pair(name, 0)
    eng.neighbor(); orc.neighbor()
    eng.force(); orc.force()
    e = eng.energy()
    er = orc.energy(reuse_hb=True)
    if name == "ninfo_hairpin":
        assert er[20 - 1] < 0.0 and er[17 - 1] < 0.0   # both secondary and tertiary bonds formed
    for k in (1, 3, 4, 8, 16, 17, 18, 19, 20):
        assert abs(e[k - 1] - er[k - 1]) <= 1e-9 * max(1.0, abs(er[k - 1])), (k, e[k - 1], er[k - 1])


@pytest.mark.parametrize("precision,tol", [(0, 1e-8), (1, 1e-4)])
def test_trajectory_injected_noise(tis_lib, precision, tol):
    nrep, nsteps = 3, 20
    s, par, eng, orc = make_pair("hairpin", precision, nrep=nrep, temps=[290.0, 300.0, 310.0])
    rng = np.random.default_rng(11)
    noise = rng.normal(size=(nsteps + 1, nrep * s["nmp"], 3))
    eng.set_noise(noise)
    orc.set_noise(noise.reshape(nsteps + 1, nrep, s["nmp"], 3))
    assert eng.time_integral_pre() >= 0
    assert orc.time_integral_pre() == 0
    eng.step(nsteps)
    orc.step(nsteps)
    x, v, a = eng.get_state()
    xr, vr, ar = orc.get_state()
    assert np.abs(x - xr.reshape(-1, 3)).max() < tol
    assert np.abs(v - vr.reshape(-1, 3)).max() < 10 * tol


def test_hbond_valence_pruning(tis_lib):
    s = synth.duplicate_hbonds(hairpin(seed=3), seed=4)
    par = synth.dt15_params(ionic_strength=0.15, precision=0)
    eng = Engine([s], par, [300.0])
    orc = Oracle(s, par, [300.0])
    eng.set_state(s["xyz"]); orc.set_state(s["xyz"][None])
    u = np.random.default_rng(5).uniform(1e-6, 1.0, size=(1, 4096))
    eng.set_noise(np.zeros((1, s["nmp"], 3)), u)
    orc.set_noise(np.zeros((1, 1, s["nmp"], 3)), u)
    eng.neighbor(); orc.neighbor()
    f, _ = eng.force()
    fr, _ = orc.force()
    st, _ = orc.hb_status()
    assert 0 < st.sum() < len(st)      # pruning removed some, not all
    assert rel_force_err(f, fr) < FORCE_TOL_FP64


def test_replica_exchange(tis_lib):
    nrep = 8
    temps = synth.temperature_ladder(nrep, 280.0, 400.0)
    s, par, eng, orc = make_pair("hairpin", 0, nrep=nrep, temps=temps)
    rng = np.random.default_rng(3)
    noise = rng.normal(size=(11, nrep * s["nmp"], 3))
    eng.set_noise(noise)
    orc.set_noise(noise.reshape(11, nrep, s["nmp"], 3))
    eng.time_integral_pre(); orc.time_integral_pre()
    eng.step(10); orc.step(10)
    for k in range(4):
        u = rng.uniform(size=nrep)
        na = eng.replica_exchange(u)
        nb = orc.replica_exchange(u)
        assert na == nb
        assert np.array_equal(eng.labels(), orc.labels())
    x, v, _ = eng.get_state()
    xr, vr, _ = orc.get_state()
    assert np.abs(v - vr.reshape(-1, 3)).max() < 1e-8


def test_replica_exchange_without_host_wait(tis_lib):
    """Exchanges that do not ask for the accept count stay on the device
    (counter-based uniforms, no host wait): labels and velocities equal those
    of the same run that reads the count after every exchange."""
    nrep = 8
    temps = synth.temperature_ladder(nrep, 280.0, 400.0)
    runs = []
    for count in (True, False):
        s, par, eng, orc = make_pair("hairpin", 1, nrep=nrep, temps=temps)
        eng.time_integral_pre()
        nacc = 0
        for k in range(6):
            eng.step(20)
            r = eng.replica_exchange(count=count)
            nacc += r or 0
        x, v, _ = eng.get_state()
        runs.append((eng.labels(), v, nacc))
        eng.close()
    assert np.array_equal(runs[0][0], runs[1][0])
    assert np.array_equal(runs[0][1], runs[1][1])
    assert runs[0][2] > 0   # the ladder makes some swaps happen


def test_uneven_batch(tis_lib):
    systems = [synth.set_friction(synth.dt15_chain(n, 100 + n, hb_fraction=0.3), 0.5) for n in (9, 23, 41)]
    par = synth.dt15_params(ionic_strength=0.15, precision=1)
    eng = Engine(systems, par, [300.0] * 3)
    eng.set_state(np.vstack([s["xyz"] for s in systems]))
    eng.neighbor()
    for k, s in enumerate(systems):
        orc = Oracle(s, par, [300.0])
        orc.set_state(s["xyz"][None])
        orc.neighbor()
        assert np.array_equal(eng.exv_list(k + 1), orc.exv_list())
        f, _ = eng.force(k + 1)
        fr, _ = orc.force()
        assert rel_force_err(f, fr) < FORCE_TOL_MIXED

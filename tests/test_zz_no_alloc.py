"""tis_force_sumup_static: neighbour lists and forces for caller-owned device
arrays, with all scratch in the library's fixed static device array.  Callers
whose device memory is held by their own pool allocator, or that must not
grow device memory once running, use it instead of tis_force_sumup.

Checked on two calls in a row on different replicas of different sizes (a
second call that saw the first call's leftovers would differ):
* against the allocating path (tis_set_state + tis_neighbor +
  tis_force_sumup) on the same coordinates, and against the oracle;
* the context's own lists and state are the same before and after;
* free device memory (cudaMemGetInfo) does not change across a call;
* a sticky error flag left in the context by an earlier call does not make
  the static call fail;
* a Brownian-HI context is refused before any launch.
Tolerances are the force parity tests': FP64 relative 1e-9, mixed 1e-5 of
max(|F_i|, median |F|).  This file is collected last so that a run that
stops at the first failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from tis_b200 import synth
from tis_b200.engine import Engine, TisError
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

TOL = {0: 1e-9, 1: 1e-5}
TIS_E_UNSUPPORTED = -7
TIS_E_NOISE_EXHAUSTED = -6


def rel_force_err(f, ref):
    mag = np.linalg.norm(ref, axis=1)
    den = np.maximum(mag, np.median(mag))
    return np.max(np.linalg.norm(f - ref, axis=1) / den)


def two_systems(periodic):
    if periodic:
        s = synth.set_friction(synth.dt15_chain(12, 7, stem=3), 0.5)
        s = synth.add_ions(s, 40.0, {"Mg": 2, "K": 12, "Cl": 5}, 8, clash=4.0)
        extra = dict(i_periodic=1, psize=(40.0, 40.0, 40.0))
        return [s], [2], extra
    a = synth.hairpin_coords(synth.set_friction(synth.dt15_chain(22, 1, stem=6), 0.5), 6, seed=1)
    b = synth.set_friction(synth.dt15_chain(30, 5, min_dist=2.6, confine=10.0), 0.5)
    return [a, b], [1, 1], {}


def static_force(eng, irep, xyz, free_check=False):
    """One call through the C-ABI; with free_check, also the device's free
    memory just before and just after it."""
    import torch
    n = eng.lane_nmp[irep - 1]
    x = torch.tensor(np.ascontiguousarray(xyz, dtype=np.float64).reshape(n, 3), device="cuda:0")
    f = torch.full((n, 3), float("nan"), dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0] if free_check else None
    rc = eng.L.tis_force_sumup_static(eng.h, irep, C.c_void_p(x.data_ptr()), C.c_void_p(f.data_ptr()))
    free1 = torch.cuda.mem_get_info()[0] if free_check else None
    if rc < 0:
        raise TisError(rc, eng.L.tis_last_error(eng.h).decode())
    out = f.cpu().numpy()
    return (out, rc, free0, free1) if free_check else (out, rc)


def context_snapshot(eng):
    lists = []
    for irep in range(1, eng.nlane + 1):
        el, ec = eng.ele_list(irep)
        lists.append((eng.exv_list(irep), el, ec, eng.hb_list(irep)))
    return eng.get_state(), lists, eng.status()


@pytest.mark.parametrize("periodic", [False, True])
@pytest.mark.parametrize("precision", [0, 1])
def test_static_matches_force_sumup(tis_lib, precision, periodic):
    systems, nrep, extra = two_systems(periodic)
    par = synth.dt15_params(ionic_strength=0.15, precision=precision, **extra)
    temps = [300.0, 330.0]
    eng = Engine(systems, par, temps, nrep=nrep)
    rng = np.random.default_rng(11)
    xs = []
    for k in range(eng.nlane):
        s = systems[k] if len(systems) > 1 else systems[0]
        xs.append(s["xyz"] + rng.normal(0.0, 0.05, s["xyz"].shape))
    # the context holds other coordinates and lists of its own
    eng.set_state(np.concatenate([x + 0.3 for x in xs]))
    eng.neighbor()
    before = context_snapshot(eng)
    # two calls in a row, the larger replica first; the second also checks
    # that no device memory is taken (the first one has loaded the kernels)
    got = {2: static_force(eng, 2, xs[1])}
    f1, rc1, free0, free1 = static_force(eng, 1, xs[0], free_check=True)
    got[1] = (f1, rc1)
    assert free1 == free0, (free0, free1)
    after = context_snapshot(eng)
    for a, b in zip(before[0], after[0]):
        assert np.array_equal(a, b)
    for la, lb in zip(before[1], after[1]):
        for a, b in zip(la, lb):
            assert np.array_equal(a, b)
    assert before[2]["n_rebuild"] == after[2]["n_rebuild"]
    # the allocating path and the oracle on the same coordinates
    eng.set_state(np.concatenate(xs))
    eng.neighbor()
    for irep in (2, 1):
        ref, rc_ref = eng.force(irep)
        f, rc = got[irep]
        assert np.isfinite(f).all()
        assert rel_force_err(f, ref) < TOL[precision], irep
        assert rc == rc_ref
        s = eng.systems_of_lane[irep - 1]
        orc = Oracle(s, dict(par, precision=0), [temps[irep - 1]])
        orc.set_state(xs[irep - 1][None])
        orc.neighbor()
        fr, _ = orc.force()
        assert rel_force_err(f, fr) < TOL[precision], (irep, "oracle")
        orc.close()
    eng.close()


def test_static_ignores_context_flags(tis_lib):
    """An exhausted injected noise array leaves a sticky flag in the context;
    the static call does not inherit it."""
    s = synth.hairpin_coords(synth.set_friction(synth.dt15_chain(22, 1, stem=6), 0.5), 6, seed=1)
    par = synth.dt15_params(ionic_strength=0.15, precision=1)
    eng = Engine([s], par, [300.0])
    eng.set_state(s["xyz"])
    eng.set_noise(np.zeros((1, s["nmp"], 3)))
    eng.time_integral_pre()
    with pytest.raises(TisError) as e:
        eng.step(2)
    assert e.value.code == TIS_E_NOISE_EXHAUSTED
    f, rc = static_force(eng, 1, s["xyz"])
    assert rc >= 0 and np.isfinite(f).all()
    eng.close()


def test_static_rejects_oversize(tis_lib):
    s = synth.set_friction(synth.dt15_chain(12, 3, stem=3), 0.5)
    s = synth.add_ions(s, 200.0, {"K": 500, "Cl": 500}, 4, clash=4.0)
    par = synth.dt15_params(ionic_strength=0.15, precision=1, i_periodic=1, psize=(200.0, 200.0, 200.0))
    eng = Engine([s], par, [300.0])
    with pytest.raises(TisError) as e:
        static_force(eng, 1, s["xyz"])
    assert e.value.code == TIS_E_UNSUPPORTED
    assert "static area" in str(e.value)
    eng.close()


def test_static_rejects_brownian_hi(tis_lib):
    s = synth.bead_chain(24, 7)
    eng = Engine([s], synth.bdhi_params(), [300.0])
    with pytest.raises(TisError) as e:
        static_force(eng, 1, s["xyz"])
    assert e.value.code == TIS_E_UNSUPPORTED
    assert "Brownian-HI" in str(e.value)
    eng.close()

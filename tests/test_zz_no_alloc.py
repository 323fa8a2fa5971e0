"""tis_force_sumup_static: neighbour lists and forces for caller-owned device
arrays with all scratch in the library's fixed static device array.

Checked against the allocating path (tis_set_state + tis_neighbor +
tis_force_sumup) on the same coordinates, for two calls in a row on
different replicas of different sizes, so that a second call that saw the
first call's leftovers would differ.  Tolerances are the ones of the force
parity tests: FP64 relative 1e-9, mixed 1e-5 of max(|F_i|, median |F|).
"""
import ctypes as C

import numpy as np
import pytest

from tis_b200 import synth
from tis_b200.engine import Engine, TisError

pytestmark = pytest.mark.gpu

TOL = {0: 1e-9, 1: 1e-5}
TIS_E_UNSUPPORTED = -7


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


def static_force(eng, irep, xyz):
    import torch
    n = eng.lane_nmp[irep - 1]
    x = torch.tensor(np.ascontiguousarray(xyz, dtype=np.float64).reshape(n, 3), device="cuda:0")
    f = torch.full((n, 3), float("nan"), dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    rc = eng.L.tis_force_sumup_static(eng.h, irep, C.c_void_p(x.data_ptr()), C.c_void_p(f.data_ptr()))
    if rc < 0:
        raise TisError(rc, eng.L.tis_last_error(eng.h).decode())
    return f.cpu().numpy(), rc


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
    # two calls in a row, the larger replica first
    order = [2, 1]
    got = {irep: static_force(eng, irep, xs[irep - 1]) for irep in order}
    # the allocating path on the same coordinates
    eng.set_state(np.concatenate(xs))
    eng.neighbor()
    for irep in order:
        ref, rc_ref = eng.force(irep)
        f, rc = got[irep]
        assert np.isfinite(f).all()
        err = rel_force_err(f, ref)
        assert err < TOL[precision], (irep, err)
        assert rc == rc_ref
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

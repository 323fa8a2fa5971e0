"""The production noise path, checked statistically (every trajectory parity
test injects its noise, so these are the only tests of the generator the
timed runs use).

(a) The counter-based Gaussian stream (Philox4x32-10 + Box-Muller, read
    back with tis_get_random_number): per replica >= 10^6 draws; mean,
    variance, kurtosis, lag-1 correlation along the steps, correlation
    between the components of a bead, between neighbouring beads and
    between replicas, each within 5 standard errors of the Gaussian value,
    and a Kolmogorov-Smirnov test against the normal CDF.
(b) Long Langevin runs of the 22-nt C1 chain at 300 K, the GPU with its own
    noise against the oracle with numpy's: the mean kinetic temperature
    T_kin = sum(m v^2) / (3 N k_B) (write_T.F90:35-36) and radius of
    gyration over the same window of the same schedule, within 4.5 combined
    standard errors (from the spread of the per-replica means).  T_kin at
    dt = 0.05, 0.02 and 0.01 tau falls short of 300 K by a deficit that
    shrinks with dt, the behaviour the reference documents for its
    velocity Verlet Langevin integrator
    (integrator_test/Temperature_check/Temperature_check.ipynb).
"""
import json

import numpy as np
import pytest

from tis_b200 import synth
from tis_b200.engine import Engine
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

BOLTZ_KCAL_MOL = 1.38064852e-23 / 4184.0 * 6.022140857e23


@pytest.mark.parametrize("precision", [0, 1])
def test_counter_noise_moments(tis_lib, precision):
    systems, par, ladder = synth.workload_c3()
    s = systems[0]
    nrep = 8
    eng = Engine([s], dict(par, precision=precision), ladder[:nrep], nrep=[nrep])
    n = s["nmp"]
    nstep, chunk = 1500, 250
    acc = np.zeros((nrep, 4))            # sum z, z^2, z^3, z^4
    lag = np.zeros(nrep)                 # z(step) z(step + 1)
    comp = np.zeros(nrep)                # x y of one bead
    bead = np.zeros(nrep)                # bead i, bead i + 1
    cross = np.zeros(nrep)               # replica r, replica r + 1
    cnt = np.zeros(5)
    prev = None
    sample = []
    for c in range(nstep // chunk):
        z = eng.random_number(1 + c * chunk, chunk).reshape(chunk, nrep, n, 3)
        assert np.isfinite(z).all()
        for p in range(4):
            acc[:, p] += (z ** (p + 1)).sum(axis=(0, 2, 3))
        lag += (z[1:] * z[:-1]).sum(axis=(0, 2, 3))
        if prev is not None:
            lag += (z[0] * prev).sum(axis=(1, 2))
        prev = z[-1]
        comp += (z[..., 0] * z[..., 1]).sum(axis=(0, 2))
        bead += (z[:, :, 1:] * z[:, :, :-1]).sum(axis=(0, 2, 3))
        cross[:-1] += (z[:, 1:] * z[:, :-1]).sum(axis=(0, 2, 3))
        sample.append(z[:, 0, :, 0].ravel()[:20000])
    m = nstep * n * 3
    assert m >= 10 ** 6
    mean = acc[:, 0] / m
    var = acc[:, 1] / m - mean ** 2
    kurt = (acc[:, 3] / m) / var ** 2
    se = 1.0 / np.sqrt(m)
    assert np.abs(mean).max() < 5 * se
    assert np.abs(var - 1).max() < 5 * np.sqrt(2.0 / m)
    assert np.abs(kurt - 3).max() < 5 * np.sqrt(24.0 / m)
    assert np.abs(acc[:, 2] / m).max() < 5 * np.sqrt(15.0 / m)     # third moment
    assert np.abs(lag / ((nstep - 1) * n * 3)).max() < 5 * se
    assert np.abs(comp / (nstep * n)).max() < 5 * np.sqrt(3) * se
    assert np.abs(bead / (nstep * (n - 1) * 3)).max() < 5 * se
    assert np.abs(cross[:-1] / m).max() < 5 * se
    from scipy import stats
    ks = stats.kstest(np.concatenate(sample), "norm")
    assert ks.pvalue > 1e-3, ks
    # a different step or replica never repeats a triple
    z1 = eng.random_number(7, 2).reshape(2, nrep, n, 3)
    assert not np.any(np.all(z1[0] == z1[1], axis=-1))
    assert not np.any(np.all(z1[0, 0] == z1[0, 1], axis=-1))
    eng.close()


def observables(x, v, mass):
    """(T_kin, Rg) per replica: x, v of shape (nrep, N, 3)."""
    ekin2 = (mass[None, :, None] * v * v).sum(axis=(1, 2))
    T = ekin2 / (3 * x.shape[1] * BOLTZ_KCAL_MOL)
    com = x.mean(axis=1, keepdims=True)
    rg = np.sqrt(((x - com) ** 2).sum(axis=2).mean(axis=1))
    return T, rg


def gpu_run(s, par, nrep, nsteps, every):
    eng = Engine([s], par, [300.0] * nrep, nrep=[nrep])
    eng.set_state(np.tile(s["xyz"], (nrep, 1)))
    eng.time_integral_pre()
    mass = np.asarray(s["cmass"], dtype=np.float64)
    out = []
    for _ in range(nsteps // every):
        eng.step(every)
        x, v, _ = eng.get_state()
        out.append(observables(x.reshape(nrep, -1, 3), v.reshape(nrep, -1, 3), mass))
    eng.close()
    return np.array(out)            # (nsample, 2, nrep)


def oracle_run(s, par, nrep, nsteps, every, seed):
    orc = Oracle(s, dict(par, precision=0), [300.0] * nrep)
    orc.set_state(np.tile(s["xyz"], (nrep, 1, 1)))
    rng = np.random.default_rng(seed)
    n = s["nmp"]
    mass = np.asarray(s["cmass"], dtype=np.float64)
    out = []
    block = 25 * every
    orc.set_noise(rng.normal(size=(1, nrep, n, 3)))
    orc.time_integral_pre()
    for b in range(nsteps // block):
        orc.set_noise(rng.normal(size=(block, nrep, n, 3)))
        for _ in range(block // every):
            orc.step(every)
            x, v, _ = orc.get_state()
            out.append(observables(x, v, mass))
    orc.close()
    return np.array(out)


def window_mean(obs, k, first):
    """Mean of observable k over samples [first:] and its standard error from
    the spread of the per-replica means (replicas are independent)."""
    per_rep = obs[first:, k, :].mean(axis=0)
    return per_rep.mean(), per_rep.std(ddof=1) / np.sqrt(len(per_rep))


@pytest.mark.parametrize("precision", [0, 1])
def test_long_run_temperature_and_rg(tis_lib, precision):
    systems, par, _ = synth.workload_c1()
    s = systems[0]
    every = 100
    report = {}
    deficits = []
    for dt, nsteps, n_orc in ((0.05, 50000, 8), (0.02, 20000, 4), (0.01, 20000, 4)):
        p = dict(par, precision=precision, tstep=dt, seed=777 + int(1000 * dt))
        g = gpu_run(s, p, 32, nsteps, every)
        o = oracle_run(s, p, n_orc, nsteps, every, seed=int(1e4 * dt))
        first = 50                     # 5,000 steps of equilibration
        tg, tg_se = window_mean(g, 0, first)
        to, to_se = window_mean(o, 0, first)
        report[dt] = {"T_gpu": tg, "T_gpu_se": tg_se, "T_oracle": to, "T_oracle_se": to_se}
        assert abs(tg - to) < 4.5 * np.hypot(tg_se, to_se), report[dt]
        deficits.append((300.0 - tg, tg_se))
        if dt == 0.05:
            rg, rg_se = window_mean(g, 1, first)
            ro, ro_se = window_mean(o, 1, first)
            report[dt].update({"Rg_gpu": rg, "Rg_gpu_se": rg_se, "Rg_oracle": ro, "Rg_oracle_se": ro_se})
            assert abs(rg - ro) < 4.5 * np.hypot(rg_se, ro_se), report[dt]
    print(json.dumps({"precision": precision, "tkin_rg": report}))
    # the Verlet-Langevin deficit shrinks with the time step
    (d5, s5), (d2, s2), (d1, s1) = deficits
    assert d5 > d2 + 3 * np.hypot(s5, s2)
    assert d2 > d1 - 3 * np.hypot(s2, s1)
    assert d5 > 0

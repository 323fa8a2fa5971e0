"""Brownian dynamics with hydrodynamic interactions (Ermak-McCammon with the
Rotne-Prager tensor and its Cholesky factor, time_integral.F90:429-457,
simu_hydro_tensors.F90) on the GPU against the CPU restatement, through the
C-ABI.  Bead chains with FENE bonds and WCA records for every non-bonded
pair.  Everything is FP64: forces and energies relative 1e-9, trajectories
with injected noise 1e-9 A.
"""
import numpy as np
import pytest

from tis_b200 import synth
from tis_b200.engine import Engine, TisError
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu
TIS_E_NOT_SPD = -4


def rel_force_err(f, ref):
    mag = np.linalg.norm(ref, axis=1)
    den = np.maximum(mag, np.median(mag))
    return np.max(np.linalg.norm(f - ref, axis=1) / den)


def squeezed_chain(n, seed):
    """A chain pulled together so that some WCA pairs are inside sigma."""
    s = synth.bead_chain(n, seed)
    s = dict(s)
    s["xyz"] = s["xyz"] * 0.85
    return s


@pytest.mark.parametrize("n", [24, 90])
def test_bdhi_forces_and_energy(tis_lib, n):
    s = squeezed_chain(n, 7)
    par = synth.bdhi_params()
    eng = Engine([s], par, [300.0])
    orc = Oracle(s, par, [300.0])
    eng.set_state(s["xyz"])
    orc.set_state(s["xyz"][None])
    orc.neighbor()
    f, _ = eng.force()
    fr, _ = orc.force()
    assert np.abs(orc.force_term("wca")).max() > 0.1       # WCA pairs inside sigma
    assert rel_force_err(f, fr) < 1e-9
    e = eng.energy()
    er = orc.energy()
    for k in (3, 23, 24):   # BOND (FENE), WCA_REP, WCA_ATT
        assert abs(e[k - 1] - er[k - 1]) <= 1e-9 * max(1.0, abs(er[k - 1])), k
    eng.close()


def test_energy_of_a_batch_with_a_lane_too_large_to_stage(tis_lib):
    """The energy kernel stages pxyz in shared memory for lanes of up to
    1,472 beads and reads the larger ones from global memory; in a batch of
    both, each lane's energies equal the oracle's."""
    systems = [synth.bead_chain(1500, 31), squeezed_chain(60, 32)]
    par = synth.bdhi_params()
    eng = Engine(systems, par, [300.0, 300.0])
    eng.set_state(np.vstack([s["xyz"] for s in systems]))
    for k, s in enumerate(systems):
        orc = Oracle(s, par, [300.0])
        orc.set_state(s["xyz"][None])
        orc.neighbor()
        e = eng.energy(k + 1)
        er = orc.energy()
        for t in (3, 23, 24):   # BOND (FENE), WCA_REP, WCA_ATT
            assert abs(e[t - 1] - er[t - 1]) <= 1e-9 * max(1.0, abs(er[t - 1])), (k, t)
    eng.close()


@pytest.mark.parametrize("every", [1, 3])
def test_bdhi_trajectory_injected_noise(tis_lib, every):
    ns = [30, 47, 64]
    systems = [squeezed_chain(n, 11 + k) for k, n in enumerate(ns)]
    par = synth.bdhi_params(n_step_hydro=every)
    nsteps = 7
    eng = Engine(systems, par, [290.0, 300.0, 310.0], nrep=[1, 1, 1])
    eng.set_state(np.concatenate([s["xyz"] for s in systems]))
    rng = np.random.default_rng(5)
    noise = rng.normal(size=(nsteps + 1, sum(ns), 3))
    eng.set_noise(noise)
    assert eng.time_integral_pre() >= 0
    assert eng.step(nsteps) >= 0
    x, _, _ = eng.get_state()
    off = 0
    for k, (s, T) in enumerate(zip(systems, [290.0, 300.0, 310.0])):
        orc = Oracle(s, par, [T])
        orc.set_state(s["xyz"][None])
        orc.set_noise(noise[:, off:off + s["nmp"]].reshape(nsteps + 1, 1, s["nmp"], 3))
        assert orc.time_integral_pre() == 0
        assert orc.step(nsteps) == 0
        assert not orc.not_spd()
        xr = orc.get_state()[0].reshape(-1, 3)
        moved = np.abs(xr - s["xyz"]).max()
        assert moved > 1e-3
        assert np.abs(x[off:off + s["nmp"]] - xr).max() < 1e-9, k
        off += s["nmp"]
    eng.close()


def test_bdhi_reports_non_spd_tensor(tis_lib):
    s = synth.bead_chain(40, 3)
    s = dict(s)
    x = s["xyz"].copy()
    x[5] = x[20] + np.array([0.05, 0.0, 0.0])   # two beads almost on top of each other
    s["xyz"] = x
    par = synth.bdhi_params()
    orc = Oracle(s, par, [300.0])
    orc.set_state(x[None])
    _, _, rc = orc.hydro_tensors()
    assert rc == TIS_E_NOT_SPD
    eng = Engine([s], par, [300.0])
    eng.set_state(x)
    eng.time_integral_pre()
    with pytest.raises(TisError) as e:
        eng.step(1)
    assert e.value.code == TIS_E_NOT_SPD
    assert eng.status()["not_spd"] == 1
    eng.close()


@pytest.mark.parametrize("precision,tol", [(0, 1e-12), (1, 1e-5)])
def test_bdhi_cholesky_factor(tis_lib, precision, tol):
    """The refreshed diffusion tensor and its Cholesky factor against the
    restatement; precision 1 runs the trailing updates on the tensor cores
    (3xTF32 split, FP32 accumulation) and keeps D in FP32, precision 0 is
    FP64 throughout."""
    s = squeezed_chain(150, 9)           # 3N = 450: 8 tiles of 64, the last one partial
    par = synth.bdhi_params(precision=precision)
    eng = Engine([s], par, [300.0])
    eng.set_state(s["xyz"])
    eng.set_noise(np.zeros((2, s["nmp"], 3)))
    eng.time_integral_pre()
    x0 = s["xyz"].copy()
    assert eng.step(1) >= 0              # refreshes D and L at the initial coordinates
    D, L = eng.hydro_tensors()
    orc = Oracle(s, dict(par, precision=0), [300.0])
    orc.set_state(x0[None])
    Dr, Lr, rc = orc.hydro_tensors()
    assert rc == 0
    dtol = 1e-12 if precision == 0 else 1e-7   # precision 1 keeps D in FP32 for the step
    assert np.abs(D - Dr).max() <= dtol * np.abs(Dr).max()
    assert np.abs(np.triu(L, 1)).max() == 0.0
    assert np.abs(L - Lr).max() <= tol * np.abs(Lr).max()
    cov = np.linalg.norm(L @ L.T - Dr) / np.linalg.norm(Dr)
    assert cov <= tol
    eng.close()


@pytest.mark.parametrize("precision,tol", [(0, 1e-12), (1, 1e-5)])
def test_bdhi_cholesky_many_lanes(tis_lib, precision, tol):
    """A batch whose panel launches hold more CTAs than the GPU runs at once
    (24 lanes, 3N up to 1800), so CTAs of one launch run in several waves:
    every lane's factor against an FP64 factorisation of its own D."""
    rng = np.random.default_rng(17)
    ns = [int(v) for v in rng.integers(120, 601, size=24)]
    systems = [synth.bead_chain(n, 300 + k) for k, n in enumerate(ns)]
    par = synth.bdhi_params(precision=precision)
    eng = Engine(systems, par, [300.0] * len(ns), nrep=[1] * len(ns))
    eng.set_state(np.vstack([s["xyz"] for s in systems]))
    eng.time_integral_pre()
    assert eng.step(1) >= 0
    for irep in range(1, len(ns) + 1):
        D, L = eng.hydro_tensors(irep)
        Lr = np.linalg.cholesky(D)
        assert np.abs(np.triu(L, 1)).max() == 0.0
        err = np.abs(L - Lr).max() / np.abs(Lr).max()
        assert err <= tol, (irep, ns[irep - 1], err)
    eng.close()


def test_bdhi_tensor_core_trajectory(tis_lib):
    """Mixed precision (tensor-core factor) trajectory against the FP64
    restatement with the same injected noise."""
    s = squeezed_chain(70, 13)
    par = synth.bdhi_params(precision=1, n_step_hydro=2)
    nsteps = 6
    noise = np.random.default_rng(8).normal(size=(nsteps + 1, s["nmp"], 3))
    eng = Engine([s], par, [300.0])
    eng.set_state(s["xyz"])
    eng.set_noise(noise)
    eng.time_integral_pre()
    assert eng.step(nsteps) >= 0
    x = eng.get_state()[0]
    orc = Oracle(s, dict(par, precision=0), [300.0])
    orc.set_state(s["xyz"][None])
    orc.set_noise(noise.reshape(nsteps + 1, 1, s["nmp"], 3))
    orc.time_integral_pre()
    orc.step(nsteps)
    xr = orc.get_state()[0].reshape(-1, 3)
    assert np.abs(xr - s["xyz"]).max() > 1e-3
    assert np.abs(x - xr).max() < 1e-6
    eng.close()


def _variant_chain(kind, n, seed, nest):
    """Bead chain squeezed so that neighbours overlap; Zuk-RPY gets per-bead
    radii and, with nest, one small bead inside a large one (its WCA record
    with that bead removed, so forces stay finite)."""
    s = dict(synth.bead_chain(n, seed))
    x = s["xyz"] * 0.85
    if kind == 4:
        rng = np.random.default_rng(seed)
        r = rng.uniform(1.2, 2.8, n)
        if nest:
            i, j = n // 2 - 3, n // 2
            r[i], r[j] = 2.6, 1.0
            x = x.copy()
            x[j] = x[i] + np.array([0.3, 0.1, -0.2])
            keep = ~((s["iwca2mp"][:, 0] == i + 1) & (s["iwca2mp"][:, 1] == j + 1))
            s["iwca2mp"] = s["iwca2mp"][keep]
            s["wca_nat"] = s["wca_nat"][keep]
            s["coef_wca"] = s["coef_wca"][:, keep]
            s["nwca"] = int(keep.sum())
        s["radius"] = r
    s["xyz"] = x
    return s


@pytest.mark.parametrize("kind", [1, 2, 3, 4])
@pytest.mark.parametrize("precision", [0, 1])
def test_bdhi_tensor_variants(tis_lib, kind, precision):
    """HI_TENSOR RPY, RPY_OVER, ERMAK_OVER and Zuk-RPY with per-bead radii
    (simu_hydro_tensors.F90:50-300): D of the refresh against the oracle
    (FP64: the same rounded operations, relative 1e-15; mixed keeps D in
    FP32: 1e-7) and its factor (FP64 1e-12, mixed 1e-5)."""
    s = _variant_chain(kind, 90, 40 + kind, nest=True)
    par = synth.bdhi_params(precision=precision, i_hydro_tensor=kind)
    orc = Oracle(s, dict(par, precision=0), [300.0])
    orc.set_state(s["xyz"][None])
    Dr, Lr, rc = orc.hydro_tensors()
    eng = Engine([s], par, [300.0])
    eng.set_state(s["xyz"])
    eng.set_noise(np.zeros((2, s["nmp"], 3)))
    eng.time_integral_pre()
    if rc != 0:
        # the Ermak-McCammon overlap formula is not positive definite on
        # every squeezed chain: the GPU must then report the same failure
        assert kind == 3 and rc == TIS_E_NOT_SPD
        with pytest.raises(TisError) as e:
            eng.step(1)
        assert e.value.code == TIS_E_NOT_SPD
        eng.close()
        return
    assert eng.step(1) >= 0
    D, L = eng.hydro_tensors()
    dtol = 1e-15 if precision == 0 else 1e-7
    assert np.abs(D - Dr).max() <= dtol * np.abs(Dr).max()
    ltol = 1e-12 if precision == 0 else 1e-5
    assert np.abs(L - Lr).max() <= ltol * np.abs(Lr).max()
    eng.close()


@pytest.mark.parametrize("kind", [2, 4])
def test_bdhi_tensor_variant_trajectory(tis_lib, kind):
    s = _variant_chain(kind, 50, 60 + kind, nest=False)
    par = synth.bdhi_params(i_hydro_tensor=kind, n_step_hydro=2)
    nsteps = 6
    noise = np.random.default_rng(kind).normal(size=(nsteps + 1, s["nmp"], 3))
    eng = Engine([s], par, [300.0])
    eng.set_state(s["xyz"])
    eng.set_noise(noise)
    eng.time_integral_pre()
    assert eng.step(nsteps) >= 0
    x = eng.get_state()[0]
    orc = Oracle(s, par, [300.0])
    orc.set_state(s["xyz"][None])
    orc.set_noise(noise.reshape(nsteps + 1, 1, s["nmp"], 3))
    orc.time_integral_pre()
    orc.step(nsteps)
    xr = orc.get_state()[0].reshape(-1, 3)
    assert np.abs(xr - s["xyz"]).max() > 1e-3
    assert np.abs(x - xr).max() < 1e-9
    eng.close()


@pytest.mark.parametrize("refine", [0, 1])
def test_bdhi_refined_noise_covariance(tis_lib, refine):
    """hi_refine (mixed precision): the matrix M the step applies to the
    noise, read column by column (unit noise vectors, no forces, one
    refresh at x0), has ||M M^T - D|| / ||D|| ~ 1e-7 with the FP32 factor
    alone and below 1e-10 with the refinement (D: the oracle's FP64 tensor
    at x0)."""
    s = dict(synth.bead_chain(100, 77))
    s.update(nfene=0, nwca=0)                         # no forces: dx = sqrt(2 dt) M xi
    par = synth.bdhi_params(precision=1, n_step_hydro=1 << 30, hi_refine=refine)
    n = 3 * s["nmp"]
    noise = np.zeros((n + 1, s["nmp"], 3))
    for i in range(n):
        noise[1 + i].reshape(-1)[i] = 1.0
    eng = Engine([s], par, [300.0])
    eng.set_state(s["xyz"])
    eng.set_noise(noise)
    eng.time_integral_pre()
    rl2 = np.sqrt(2.0 * par["tstep"])
    M = np.zeros((n, n))
    x_prev = eng.get_state()[0].reshape(-1)
    for i in range(n):
        assert eng.step(1) >= 0
        x = eng.get_state()[0].reshape(-1)
        M[:, i] = (x - x_prev) / rl2
        x_prev = x
    eng.close()
    orc = Oracle(s, dict(par, precision=0), [300.0])
    orc.set_state(s["xyz"][None])
    D, _, rc = orc.hydro_tensors(cholesky=False)
    cov = np.linalg.norm(M @ M.T - D) / np.linalg.norm(D)
    if refine:
        assert cov < 1e-10, cov
    else:
        assert 1e-9 < cov < 1e-5, cov
    print({"refine": refine, "covariance_error": cov})


def test_bdhi_refined_trajectory(tis_lib):
    """The refined mixed-precision step against the FP64 restatement with
    the same injected noise (the correction is of order 1e-7)."""
    s = _variant_chain(1, 70, 19, nest=False)
    par = synth.bdhi_params(precision=1, n_step_hydro=2, hi_refine=1)
    nsteps = 6
    noise = np.random.default_rng(12).normal(size=(nsteps + 1, s["nmp"], 3))
    eng = Engine([s], par, [300.0])
    eng.set_state(s["xyz"])
    eng.set_noise(noise)
    eng.time_integral_pre()
    assert eng.step(nsteps) >= 0
    x = eng.get_state()[0]
    orc = Oracle(s, dict(par, precision=0), [300.0])
    orc.set_state(s["xyz"][None])
    orc.set_noise(noise.reshape(nsteps + 1, 1, s["nmp"], 3))
    orc.time_integral_pre()
    orc.step(nsteps)
    xr = orc.get_state()[0].reshape(-1, 3)
    assert np.abs(xr - s["xyz"]).max() > 1e-3
    assert np.abs(x - xr).max() < 1e-6
    eng.close()

"""Two CTAs per replica (a thread-block cluster that splits the beads and the
bonded items) against one CTA per replica and against the CPU restatement,
through the C-ABI.  The split is used by tis_step for mixed precision,
non-periodic systems of >= 64 beads with a fixed rebuild cadence when the
replicas fill at most half of the SMs; tis_params.launch_ctas chooses it.

Tolerances: two-CTA vs one-CTA positions 1e-9 A after 25 steps (the same
FP32 pair forces, FP64 sums grouped differently); against the oracle the
mixed-precision trajectory tolerance 1e-4 A.
"""
import numpy as np
import pytest

from tis_b200 import synth
from tis_b200.engine import Engine
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def run(system, par, temps, noise, nsteps, pair, uniforms=None):
    eng = Engine([system], dict(par, launch_ctas=2 if pair else 1), temps, nrep=[len(temps)])
    assert eng.status()["ctas_per_lane"] == (2 if pair else 1)
    eng.set_state(np.tile(system["xyz"], (len(temps), 1)))
    eng.set_noise(noise, uniforms)
    assert eng.time_integral_pre() >= 0
    assert eng.step(nsteps) >= 0
    x, v, a = eng.get_state()
    st = eng.status()
    eng.close()
    return x, v, st


def oracle_run(system, par, temps, noise, nsteps, uniforms=None):
    n = system["nmp"]
    orc = Oracle(system, dict(par, precision=0), temps)
    orc.set_state(np.tile(system["xyz"], (len(temps), 1, 1)))
    orc.set_noise(noise.reshape(nsteps + 1, len(temps), n, 3), uniforms)
    assert orc.time_integral_pre() == 0
    orc.step(nsteps)
    return orc.get_state()[0].reshape(-1, 3)


def test_pair_matches_single_cta_and_oracle(tis_lib):
    systems, par, temps = synth.workload_c3()
    s = systems[0]
    temps = list(temps[::16])          # 4 replicas of the 227-bead chain
    nsteps = 25                        # rebuilds at steps 1, 11, 21
    noise = np.random.default_rng(4).normal(size=(nsteps + 1, len(temps) * s["nmp"], 3))
    x2, v2, st2 = run(s, par, temps, noise, nsteps, pair=True)
    x1, v1, st1 = run(s, par, temps, noise, nsteps, pair=False)
    assert np.abs(x2 - x1).max() < 1e-9
    assert np.abs(v2 - v1).max() < 1e-8
    assert st2["n_rebuild"] == st1["n_rebuild"]
    xr = oracle_run(s, par, temps, noise, nsteps)
    assert np.abs(x2 - xr).max() < 1e-4


def test_pair_with_valence_pruning(tis_lib):
    base = synth.set_friction(synth.dt15_chain(22, 3, stem=6), 0.5)
    s = synth.duplicate_hbonds(synth.hairpin_coords(base, 6, seed=3), seed=4)
    par = synth.dt15_params(ionic_strength=0.15, precision=1)
    temps = [300.0, 310.0]
    nsteps = 12
    noise = np.random.default_rng(6).normal(size=(nsteps + 1, len(temps) * s["nmp"], 3))
    u = np.random.default_rng(7).uniform(1e-6, 1.0, size=(len(temps), 8192))
    x2, _, _ = run(s, par, temps, noise, nsteps, pair=True, uniforms=u)
    x1, _, _ = run(s, par, temps, noise, nsteps, pair=False, uniforms=u)
    assert np.abs(x2 - x1).max() < 1e-9
    xr = oracle_run(s, par, temps, noise, nsteps, uniforms=u)
    assert np.abs(x2 - xr).max() < 1e-4

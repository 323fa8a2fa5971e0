"""A 16-replica ladder held by two ladder contexts of 8 replicas each (two
ranks' shares, here in one process on one GPU: their kernels never wait on
each other) against one context holding all 16, through the C-ABI.

Counter-based noise is keyed by the global replica, so every replica moves
bit-identically in either layout; an exchange from the gathered
replica_energy(2, 16) (tis_rex_energies + tis_rex_exchange_all) gives the
labels, accept counts and rescaled velocities of the one-context device
exchange (tis_replica_exchange), with injected and with counter-based
uniforms.  Bit-exact throughout.
"""
import numpy as np
import pytest

from tis_b200 import remd, synth
from tis_b200.engine import Engine

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [0, 1])
def test_ladder_contexts_match_one_context(tis_lib, precision):
    systems, par, _ = synth.workload_c3()
    s = systems[0]
    par = dict(par, precision=precision)
    nall = 16
    ladder = synth.temperature_ladder(nall, 280.0, 400.0)
    n = s["nmp"]
    one = Engine([s], par, ladder, nrep=[nall])
    parts = []
    for rank in range(2):
        first, count = remd.ladder_share(nall, 2, rank)
        parts.append((first, Engine([s], par, ladder[first - 1:first - 1 + count], nrep=[count],
                                    ladder=(ladder, first))))
    for e in [one] + [p for _, p in parts]:
        e.set_state(np.tile(s["xyz"], (e.nlane, 1)))
        e.time_integral_pre()
    rng = np.random.default_rng(9)

    def compare():
        x1, v1, _ = one.get_state()
        lab1 = one.labels()
        for first, e in parts:
            x, v, _ = e.get_state()
            sl = slice((first - 1) * n, (first - 1 + e.nlane) * n)
            assert np.array_equal(x, x1[sl]) and np.array_equal(v, v1[sl])
            assert np.array_equal(e.labels(), lab1[first - 1:first - 1 + e.nlane])

    total = 0
    for k in range(4):
        for e in [one] + [p for _, p in parts]:
            e.step(40)
        compare()
        u = rng.uniform(size=nall) if k % 2 == 0 else None
        na = one.replica_exchange(u)
        e_all = np.concatenate([e.rex_energies() for _, e in parts])
        nb = [e.rex_exchange_all(e_all, u) for _, e in parts]
        assert nb == [na, na]
        total += na
        compare()
    assert total > 0
    for e in [one] + [p for _, p in parts]:
        e.close()

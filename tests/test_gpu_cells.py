"""The binned (cell-list) neighbour build of large one-CTA lanes: bins at
least as wide as the largest list cutoff, each row testing the beads of the
27 bins around its own (across the box when periodic).  The pair test is
the all-pairs one (neighbor_list.F90:49-90, neighbor_assign.F90:481-557,
neighbor_list_ele.F90:123-210), so the exv and ele lists, the mirror
images and coef_ele must stay bit-exact with the oracle.

Systems where the binned build is taken (>= 384 beads, more than 27 bins):
a 200-nt chain without electrostatics (exv cutoff 11.2 A, open boundaries),
and the explicit-ion Ewald box (28 A bins in the 150 A box, periodic),
also after a run in which the skin rule rebuilt the lists with beads moved
across the box faces.
"""
import numpy as np
import pytest

from tis_b200 import synth
from tis_b200.engine import Engine
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

CELL_MIN = 384


def binned(s, par, warps=16):
    """Whether the lane kernel bins this system (the conditions of
    build_lists): enough beads, and bins of at least the largest cutoff,
    widened by 1.25 until their tables fit 6144 ints of scratch, that
    number more than 27 (at least 3 per side when periodic)."""
    n = s["nmp"]
    if n < CELL_MIN:
        return False
    margin = par.get("neigh_margin", 8.0)
    rc = 3.2 + margin   # RNA-RNA exv cutoff plus margin; ion radius sums are smaller
    if par.get("i_ele", 0) == 2:
        rc = max(rc, par["cutoff_ele"] + margin)
    elif par.get("i_ele", 0) != 0:
        return False   # Debye-Hueckel cutoffs span the whole chain
    per = par.get("i_periodic", 0)
    ext = np.array(par["psize"]) if per else s["xyz"].max(axis=0) - s["xyz"].min(axis=0)
    room = 6144 - 1 - n - 56 * warps
    w = rc
    for _ in range(40):
        nb = np.floor(ext / w) + (0 if per else 1)
        if (per and nb.min() < 3) or np.prod(nb) <= 27:
            return False
        if 2 * np.prod(nb) <= room:
            return True
        w *= 1.25
    return False


def long_chain():
    s = synth.set_friction(synth.dt15_chain(200, 17, hb_fraction=0.3), 0.5)
    # one CTA per replica: the binned build is that kernel's
    return s, synth.dt15_params(i_ele=0, precision=1, launch_ctas=1)


def c2():
    systems, par, _ = synth.workload_c2()
    return systems[0], par


def compare_lists(eng, orc):
    assert np.array_equal(eng.exv_list(), orc.exv_list())
    ge, gc = eng.ele_list()
    oe, oc = orc.ele_list()
    assert np.array_equal(ge, oe)
    assert np.array_equal(gc, oc)


@pytest.mark.parametrize("make", [long_chain, c2])
def test_binned_lists_bit_exact(tis_lib, make):
    s, par = make()
    eng = Engine([s], par, [300.0])
    st = eng.status()
    assert st["ctas_per_lane"] == 1
    assert binned(s, par, st["threads_per_cta"] // 32)
    orc = Oracle(s, dict(par, precision=0), [300.0])
    eng.set_state(s["xyz"])
    orc.set_state(s["xyz"][None])
    eng.neighbor()
    orc.neighbor()
    compare_lists(eng, orc)
    assert len(eng.exv_list()) > 0
    eng.close()


@pytest.mark.parametrize("make", [long_chain, c2])
def test_binned_lists_of_skin_rebuilds(tis_lib, make):
    """Lists rebuilt inside the step kernel by the skin rule (a 2 A margin:
    frequent rebuilds), one step per call: whenever a step rebuilt them, they
    equal the oracle's lists from the positions that step started from (the
    GPU's pxyz, so both wrap the periodic box alike)."""
    s, par = make()
    par = dict(par, n_step_neighbor=0, neigh_margin=2.0)
    eng = Engine([s], par, [300.0])
    assert binned(s, par, eng.status()["threads_per_cta"] // 32)
    eng.set_state(s["xyz"])
    eng.time_integral_pre()
    orc = Oracle(s, dict(par, precision=0), [300.0])
    checked = 0
    n_prev, _ = eng.rebuild_info(1)
    for _ in range(600):
        p0 = eng.get_pxyz()
        assert eng.step(1) >= 0
        n, _ = eng.rebuild_info(1)
        if n > n_prev:
            orc.set_state(p0[None])
            orc.neighbor()
            compare_lists(eng, orc)
            checked += 1
            if checked == 3:
                break
        n_prev = n
    assert checked == 3
    eng.close()

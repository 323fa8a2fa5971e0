"""The committed fixtures of tests/golden (see make_golden.py there): the CPU
restatement must reproduce them (CPU), and the CUDA path must match them
through the C-ABI (GPU): lists bit-exact; forces FP64 relative 1e-9, mixed
1e-5 of max(|F_i|, median |F|); energies FP64 relative 1e-9."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402

CASES = {name: (s, par, T) for name, s, par, T in make_golden.cases()}


def fixture(name):
    return np.load(os.path.join(HERE, "golden", name + ".npz"))


def rel_force_err(f, ref):
    mag = np.linalg.norm(ref, axis=1)
    den = np.maximum(mag, np.median(mag))
    return np.max(np.linalg.norm(f - ref, axis=1) / den)


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_reproduces_fixture(name):
    from oracle.oracle import Oracle
    s, par, T = CASES[name]
    g = fixture(name)
    assert np.array_equal(s["xyz"], g["xyz"])
    o = Oracle(s, par, [T])
    o.set_state(s["xyz"][None])
    o.neighbor()
    assert np.array_equal(o.exv_list(), g["exv"])
    ele, coef = o.ele_list()
    assert np.array_equal(ele, g["ele"])
    assert np.allclose(coef, g["coef_ele"], rtol=1e-14, atol=0)
    assert np.array_equal(o.hb_list(), g["hb"])
    f, rc = o.force()
    assert rel_force_err(f, g["force"]) < 1e-12
    assert np.allclose(o.energy(reuse_hb=True), g["energy"], rtol=1e-12, atol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", list(CASES))
def test_cuda_matches_fixture(tis_lib, name, precision):
    from tis_b200.engine import Engine
    s, par, T = CASES[name]
    g = fixture(name)
    eng = Engine([s], dict(par, precision=precision), [T])
    eng.set_state(g["xyz"])
    eng.neighbor()
    assert np.array_equal(eng.exv_list(), g["exv"])
    ele, coef = eng.ele_list()
    assert np.array_equal(ele, g["ele"])
    assert np.allclose(coef, g["coef_ele"], rtol=1e-14, atol=0)
    assert np.array_equal(eng.hb_list(), g["hb"])
    f, rc = eng.force()
    assert rel_force_err(f, g["force"]) < (1e-9 if precision == 0 else 1e-5)
    if precision == 0:
        e = eng.energy()
        assert np.allclose(e, g["energy"], rtol=1e-9, atol=1e-9)
    eng.close()

"""Restart through the reference's restart blocks: a run stopped at a
rebuild boundary, written with write_rst's layout, read back into a fresh
context (state, step counter) continues exactly like the uninterrupted run
(counter-based noise and pruning uniforms follow the step counter).  The
DCD frames hold the positions in real(4)."""
import numpy as np
import pytest

from tis_b200 import synth, trajio
from tis_b200.engine import Engine

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [0, 1])
def test_restart_continues_the_run(tis_lib, tmp_path, precision):
    s = synth.hairpin_tertiary(1)
    par = synth.dt15_params(ionic_strength=0.15, precision=precision)
    eng = Engine([s], par, [300.0])
    eng.set_state(s["xyz"])
    eng.time_integral_pre()
    dcd = trajio.DCDWriter(tmp_path / "t.dcd", nmp=s["nmp"], lunit_end=[s["nmp"]], tempk=300.0,
                           istrt=0, nstep=50, nsavc=10, tstep=par["tstep"])
    saved = []
    for k in range(3):
        eng.step(10)
        x, v, a = eng.get_state()
        dcd.write(x)
        saved.append(x.copy())
    hb, st = eng.dtrna_status()
    assert (st == 0).any() and (st == 1).any()
    istep = eng.status()["step"]
    trajio.write_rst(tmp_path / "t.rst", 1, 0, istep, x, v, a, hb, st)
    eng.step(20)
    xa, va, _ = eng.get_state()
    eng.close()
    dcd.close()
    _, frames = trajio.read_dcd(tmp_path / "t.dcd")
    for k in range(3):
        assert np.array_equal(frames[k], saved[k].astype(np.float32))
    r = trajio.read_rst(tmp_path / "t.rst")
    eng2 = Engine([s], par, [300.0])
    eng2.set_state(r["xyz"], r["velo"], r["accel"])
    eng2.set_step(r["istep"])
    eng2.neighbor()
    eng2.step(20)
    xb, vb, _ = eng2.get_state()
    assert np.array_equal(xa, xb)
    assert np.array_equal(va, vb)
    eng2.close()

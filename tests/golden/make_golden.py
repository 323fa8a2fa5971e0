"""Writes the golden fixtures of this directory from the CPU restatement
(oracle/).  The reference (Fortran) cannot be built or run here and ships no
vectors for this path, so these fixtures are outputs of the restatement,
whose own pins (F = -grad E, Ewald vs lattice sum, analytic cases) are in
tests/test_oracle_pins.py.  They freeze those outputs so that the CUDA path
and later changes of the restatement are both checked against the same
committed numbers.

  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tis_b200 import synth  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402


def cases():
    s = synth.hairpin_coords(synth.set_friction(synth.dt15_chain(22, 1, stem=6), 0.5), 6, seed=1)
    yield "hairpin_dh150", s, synth.dt15_params(ionic_strength=0.15), 300.0
    s = synth.set_friction(synth.dt15_chain(30, 5, min_dist=3.0, confine=10.0), 0.5)
    yield "dense_dh100_280K", s, synth.dt15_params(ionic_strength=0.10), 280.0
    s = synth.set_friction(synth.dt15_chain(12, 7, stem=3), 0.5)
    s = synth.add_ions(s, 40.0, {"Mg": 2, "K": 12, "Cl": 5}, 8, clash=4.0)
    yield "periodic_ions_dh150", s, synth.dt15_params(ionic_strength=0.15, i_periodic=1,
                                                       psize=(40.0, 40.0, 40.0)), 300.0
    s, par, _ = synth.workload_c3()
    s = s[0]
    yield "c3_chain_dh100_400K", s, dict(par, precision=0), 400.0


def main():
    for name, s, par, T in cases():
        o = Oracle(s, par, [T])
        o.set_state(s["xyz"][None])
        o.neighbor()
        exv = o.exv_list()
        ele, coef = o.ele_list()
        hb = o.hb_list()
        f, rc = o.force()
        e = o.energy(reuse_hb=True)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), xyz=s["xyz"], exv=exv, ele=ele, coef_ele=coef,
                            hb=hb, force=f, energy=e, rc=rc, tempk=T)
        print(name, s["nmp"], len(exv), len(ele), len(hb), rc)


if __name__ == "__main__":
    main()

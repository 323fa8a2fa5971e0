"""Writes hairpin_tertiary.cg.pdb and hairpin_tertiary.ninfo: the seeded
22-nt hairpin with tertiary stacks of tis_b200.synth, every second hydrogen
bond typed tertiary ('T'), plus an ion unit, in the reference's CG PDB and
.ninfo layouts (tis_b200.ninfo writers).  The GPU parity tests read them
back through tis_b200.ninfo, so the input path from files to the device is
covered end to end.

  python tests/golden/make_ninfo_fixture.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from tis_b200 import ninfo, synth  # noqa: E402

NAME = "hairpin_tertiary"


def system():
    s = synth.hairpin_tertiary()
    s["flg_hb_tertiary"] = (np.arange(s["nhb"]) % 2).astype(np.int32)
    return synth.add_ions(s, 60.0, {"Mg": 2, "K": 4, "Cl": 3}, 9, clash=4.0)


def texts():
    s = system()
    return ninfo.write_pdb_cg(s), ninfo.write_ninfo(s)


def main():
    pdb, nin = texts()
    with open(os.path.join(HERE, NAME + ".cg.pdb"), "w") as f:
        f.write(pdb)
    with open(os.path.join(HERE, NAME + ".ninfo"), "w") as f:
        f.write(nin)


if __name__ == "__main__":
    main()

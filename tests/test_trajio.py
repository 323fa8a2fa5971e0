"""DCD and restart files (write_xyz_dcd.F90 with doc/file_format_DCD.md,
write_rst.F90 / read_rst.F90): byte layout and round trips, no GPU."""
import struct

import numpy as np

from tis_b200 import trajio


def test_dcd_header_layout(tmp_path):
    p = tmp_path / "a.dcd"
    w = trajio.DCDWriter(p, nmp=5, lunit_end=[3, 5], tempk=300.0, istrt=0, nstep=100, nsavc=10, tstep=0.05)
    rng = np.random.default_rng(1)
    frames = [rng.normal(size=(5, 3)) * 10 for _ in range(3)]
    for f in frames:
        w.write(f)
    w.close()
    b = p.read_bytes()
    i = lambda off: struct.unpack_from("<i", b, off)[0]
    assert i(0) == 84 and b[4:8] == b"CORD"
    assert i(8) == 11                      # nset = (nstep - istrt) / nsavc + 1
    assert i(20) == 100 and i(24) == 2     # nstep, nunit_real
    assert abs(struct.unpack_from("<f", b, 44)[0] - 0.05) < 1e-7
    assert i(84) == 24 and i(88) == 84     # nver, closing marker of the first block
    ntitle = 3 + 2
    assert i(92) == 4 + 80 * ntitle and i(96) == ntitle
    off = 100 + 80 * ntitle
    assert i(off) == 4 + 80 * ntitle and i(off + 4) == 4 and i(off + 8) == 5 and i(off + 12) == 4
    hdr, fr = trajio.read_dcd(p)
    assert hdr["nmp"] == 5 and hdr["nunit"] == 2 and hdr["kind"] == "CORD" and fr.shape == (3, 5, 3)
    assert hdr["titles"][3].strip() == "3" and hdr["titles"][4].strip() == "5"
    for k in range(3):
        assert np.array_equal(fr[k], frames[k].astype(np.float32))
    # one frame: 3 blocks of (4 + 4 nmp + 4) bytes
    assert len(b) == off + 16 + 3 * 3 * (8 + 4 * 5)


def test_restart_blocks(tmp_path):
    p = tmp_path / "a.rst"
    rng = np.random.default_rng(2)
    n = 7
    x, v, a = (rng.normal(size=(n, 3)) for _ in range(3))
    hb = np.array([1, 0, 1], dtype=np.int32)
    st = np.array([1, 1, 0, 1], dtype=np.int32)
    trajio.write_rst(p, 2, 0, 123456789012, x, v, a, hb, st, rep2lab=[2, 1, 3])
    b = p.read_bytes()
    i = lambda off: struct.unpack_from("<i", b, off)[0]
    # REPLICA block: id 5, size 4 (1 + 2 n), n, (i, rep2lab(i)) pairs
    assert (i(0), i(4), i(8)) == (5, 4 * 7, 3)
    off = 8 + 4 * 7
    # STEP block: id 1, size 4 + 8 (calc_size(1, 1, 0, 0, 0)), istep_sim, istep
    assert (i(off), i(off + 4), i(off + 8)) == (1, 12, 0)
    assert struct.unpack_from("<q", b, off + 12)[0] == 123456789012
    off += 20
    # XYZ / VELO / ACCEL: id, size 8 + 24 n, grep, nmp, doubles
    for bid in (2, 3, 4):
        assert (i(off), i(off + 4), i(off + 8), i(off + 12)) == (bid, 8 + 24 * n, 2, n)
        off += 16 + 24 * n
    # DTRNA15: id 6, size 12 + 4 (nhb + nst)
    assert (i(off), i(off + 4), i(off + 12), i(off + 16)) == (6, 12 + 4 * 7, 3, 4)
    assert len(b) == off + 20 + 4 * 7
    r = trajio.read_rst(p)
    assert r["istep"] == 123456789012 and r["grep"] == 2
    assert np.array_equal(r["xyz"], x) and np.array_equal(r["velo"], v) and np.array_equal(r["accel"], a)
    assert np.array_equal(r["hb_status"], hb) and np.array_equal(r["st_status"], st)
    assert np.array_equal(r["rep2lab"], [2, 1, 3])

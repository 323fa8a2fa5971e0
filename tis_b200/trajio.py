"""Trajectory and restart files of the reference, written from (and read
into) the device state: the DCD of write_xyz_dcd.F90 (layout in the
reference's doc/file_format_DCD.md) and the restart blocks of write_rst.F90
(read back by read_rst.F90).

Both files are Fortran stream-unformatted: every record is written with its
own byte-count markers by the program, so they are plain little-endian
bytes here.  Default integers are 4 bytes, the step counter 8, reals of the
coordinates 8 (restart) or 4 (DCD), logicals 4."""
import struct

import numpy as np

# block ids of write_rst.F90 (const_index.F90 RSTBLK)
RST_STEP, RST_XYZ, RST_VELO, RST_ACCEL, RST_REPLICA, RST_DTRNA15 = 1, 2, 3, 4, 5, 6


def _i4(v):
    return struct.pack("<i", int(v))


def _title(text: str) -> bytes:
    return text.encode("ascii", "replace")[:80].ljust(80, b" ")


def dcd_header(nmp: int, lunit_end, tempk: float, istrt: int, nset: int, nsavc: int, nstep: int,
               tstep: float, velocity: bool = False) -> bytes:
    """write_xyz_dcd.F90 header block (ihead == 1).  lunit_end: the last bead
    (1-based) of every unit, lunit2mp(2, :).  The two banner lines are this
    library's; the temperature line is list-directed like the reference's."""
    out = [_i4(84), b"VELD" if velocity else b"CORD", _i4(nset), _i4(istrt), _i4(nsavc), _i4(nstep),
           _i4(len(lunit_end)), _i4(0), _i4(0), _i4(0), _i4(0), struct.pack("<f", float(tstep))]
    out += [_i4(0)] * 9
    out += [_i4(24), _i4(84)]
    ntitle = 3 + len(lunit_end)
    out += [_i4(4 + 80 * ntitle), _i4(ntitle)]
    out.append(_title("========================= Molecular Dynamics tis_b200 (B200 path) ================"))
    out.append(_title("==== trajectory of the DT15 force-and-integrate path, reference DCD layout ====="))
    out.append(_title(f"   {float(tempk):.15g}"))
    for e in lunit_end:
        out.append(_title(f"{int(e):6d}"))
    out += [_i4(4 + 80 * ntitle), _i4(4), _i4(nmp), _i4(4)]
    return b"".join(out)


def dcd_frame(xyz) -> bytes:
    """One frame: X, Y and Z blocks of real(4) with their byte-count markers."""
    x = np.asarray(xyz, dtype=np.float64).reshape(-1, 3)
    n = 4 * x.shape[0]
    out = []
    for d in range(3):
        out += [_i4(n), x[:, d].astype("<f4").tobytes(), _i4(n)]
    return b"".join(out)


class DCDWriter:
    """Writes the coordinate (or velocity) DCD of one replica."""

    def __init__(self, path, nmp, lunit_end, tempk, istrt, nstep, nsavc, tstep, velocity=False):
        self.f = open(path, "wb")
        nset = (int(nstep) - int(istrt)) // int(nsavc) + 1
        self.f.write(dcd_header(nmp, lunit_end, tempk, istrt, nset, nsavc, nstep, tstep, velocity))
        self.nmp = int(nmp)

    def write(self, xyz):
        x = np.asarray(xyz).reshape(-1, 3)
        assert x.shape[0] == self.nmp
        self.f.write(dcd_frame(x))

    def close(self):
        self.f.close()


def read_dcd(path):
    """(header dict, frames (nframe, nmp, 3) float32) of a DCD written as
    above (or by the reference)."""
    b = open(path, "rb").read()
    p = 0

    def i4():
        nonlocal p
        v = struct.unpack_from("<i", b, p)[0]
        p += 4
        return v
    assert i4() == 84
    kind = b[p:p + 4].decode()
    p += 4
    nset, istrt, nsavc, nstep, nunit = i4(), i4(), i4(), i4(), i4()
    p += 16
    tstep = struct.unpack_from("<f", b, p)[0]
    p += 4 + 36
    assert i4() == 24 and i4() == 84
    size = i4()
    ntitle = i4()
    titles = [b[p + 80 * k:p + 80 * (k + 1)].decode("ascii", "replace") for k in range(ntitle)]
    p += 80 * ntitle
    assert i4() == size and i4() == 4
    nmp = i4()
    assert i4() == 4
    frames = []
    while p < len(b):
        fr = np.zeros((nmp, 3), dtype=np.float32)
        for d in range(3):
            assert i4() == 4 * nmp
            fr[:, d] = np.frombuffer(b, dtype="<f4", count=nmp, offset=p)
            p += 4 * nmp
            assert i4() == 4 * nmp
        frames.append(fr)
    hdr = dict(kind=kind, nset=nset, istrt=istrt, nsavc=nsavc, nstep=nstep, nunit=nunit, tstep=tstep,
               titles=titles, nmp=nmp)
    return hdr, np.array(frames)


def write_rst(path, grep, istep_sim, istep, xyz, velo, accel, hb_status=None, st_status=None, rep2lab=None):
    """write_rst.F90:53-113 for replica grep (1-based): REPLICA (when
    rep2lab is given: the first replica's file of a multi-replica run), STEP,
    XYZ, VELO, ACCEL and, for DT15 runs, DTRNA15 blocks."""
    x = np.asarray(xyz, dtype="<f8").reshape(-1, 3)
    v = np.asarray(velo, dtype="<f8").reshape(-1, 3)
    a = np.asarray(accel, dtype="<f8").reshape(-1, 3)
    out = []
    if rep2lab is not None and len(rep2lab) > 1:
        n = len(rep2lab)
        out += [_i4(RST_REPLICA), _i4(4 * (1 + 2 * n)), _i4(n)]
        for i, lab in enumerate(rep2lab):
            out += [_i4(i + 1), _i4(lab)]
    out += [_i4(RST_STEP), _i4(4 + 8), _i4(istep_sim), struct.pack("<q", int(istep))]
    for bid, arr in ((RST_XYZ, x), (RST_VELO, v), (RST_ACCEL, a)):
        out += [_i4(bid), _i4(8 + 8 * arr.size), _i4(grep), _i4(arr.shape[0]), arr.tobytes()]
    if hb_status is not None and st_status is not None:
        hb = np.asarray(hb_status, dtype="<i4")
        st = np.asarray(st_status, dtype="<i4")
        out += [_i4(RST_DTRNA15), _i4(12 + 4 * (hb.size + st.size)), _i4(grep), _i4(hb.size), _i4(st.size),
                hb.tobytes(), st.tobytes()]
    with open(path, "wb") as f:
        f.write(b"".join(out))


def read_rst(path):
    """The blocks of a restart file as a dict (read_rst.F90)."""
    b = open(path, "rb").read()
    p = 0
    out = {}

    def i4():
        nonlocal p
        v = struct.unpack_from("<i", b, p)[0]
        p += 4
        return v
    while p < len(b):
        bid, size = i4(), i4()
        start = p
        if bid == RST_REPLICA:
            n = i4()
            out["rep2lab"] = np.array([struct.unpack_from("<ii", b, p + 8 * k)[1] for k in range(n)], dtype=np.int32)
        elif bid == RST_STEP:
            out["istep_sim"] = i4()
            out["istep"] = struct.unpack_from("<q", b, p)[0]
        elif bid in (RST_XYZ, RST_VELO, RST_ACCEL):
            out["grep"] = i4()
            n = i4()
            arr = np.frombuffer(b, dtype="<f8", count=3 * n, offset=p).reshape(n, 3).copy()
            out[{RST_XYZ: "xyz", RST_VELO: "velo", RST_ACCEL: "accel"}[bid]] = arr
        elif bid == RST_DTRNA15:
            i4()
            nhb, nst = i4(), i4()
            out["hb_status"] = np.frombuffer(b, dtype="<i4", count=nhb, offset=p).copy()
            out["st_status"] = np.frombuffer(b, dtype="<i4", count=nst, offset=p + 4 * nhb).copy()
        p = start + size
    return out

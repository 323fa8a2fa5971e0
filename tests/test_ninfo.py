"""CG PDB and .ninfo input (read_pdb_cg.F90, read_nativeinfo.F90,
setp_dtrna15.F90, setp_mass_fric.F90, setp_native_charge.F90): columns,
record rules, error cases, the writers' round trip and the oracle on a
system read from files.  No GPU."""
import math
import os

import numpy as np
import pytest

from tis_b200 import ninfo as N
from tis_b200 import synth
from tis_b200.abi import CLASS_ION, CLASS_RNA, MP_ION_CL, MP_ION_MG, MP_RNA_BASE, MP_RNA_PHOS, MP_RNA_SUGAR

# the reference source tree (Hori-Lab/TIS), when present: its input files
# are read as test data; the tests that need it skip otherwise
REF = os.environ.get("TIS_REFERENCE_DIR", "")

# A 4-nucleotide chain with a 5' phosphate (P S B per nucleotide, beads 1-12)
# and an ion unit, in the fixed columns of read_pdb_cg.F90 (coordinates
# glued together as the reference's ion files have them, one field without
# a decimal point, which f8.3 reads with 3 implied decimals).
PDB = """\
ATOM      1  P   RG  A   1       0.000   0.000   0.000
ATOM      2  S   RG  A   1       3.000   1.000   0.000
ATOM      3  Gb  RG  A   1       6.000   1.500   0.500
ATOM      4  P   RC  A   2       2.000   4.000   0.000
ATOM      5  S   RC  A   2       5.000   5.000   0.000
ATOM      6  Cb  RC  A   2       8.000   5.500   0.500
ATOM      7  P   RA  A   3       4.000   8.000   0.000
ATOM      8  S   RA  A   3       7.000   9.000   0.000
ATOM      9  Ab  RA  A   3      10.000   9.500   0.500
ATOM     10  P   RU  A   4       6.000  12.000   0.000
ATOM     11  S   RU  A   4       9.000  13.000   0.000
ATOM     12  Ub  RU  A   4      12.000  13.500   0.500
TER
ATOM     13 MG   Mg  B   1    -205.195-149.235 130.726
ATOM     14 CL   Cl  B   2       12345   1.000   2.000
TER
"""

# One record of each DT15 kind.  hb-dist lists the higher bead first (the
# reference stores the pair sorted; its atom columns name the lower bead's
# atom first), tbs-dist likewise (its side types swap with the beads).
NINFO = """\
<<<< native bond length
** comment lines and blocks are ignored
bond      1  1  1   2   3   2   3   4.9659 1.0 1.0  10.0000 SG
bond      2  1  1   2   4   2   4   3.8157 1.0 1.0  64.0000 SP
angl      1  1  1   3   2   4   3   2   4  109.7214 1.0 1.0  5.0000 GSP
>>>>
bs-dist   1  1  1   3   6   3   6   4.7199  4.370  343.363  4.25  1.4  G-C
bs-dihd   1  1  1  1   1   2   4   5   1   2   4   5 -148.22 4.0 PSPS
bs-dihd   1  2  1  1   2   4   5   7   2   4   5   7  175.98 4.0 SPSP
hb-dist   1  1  1  12   3  12   3  -5.86 5.80 5.0 T 2 N1 N3 O6 O4
hb-angl   1  1  1  1   2   3  12   2   3  12  142.31 1.5
hb-angl   1  2  1  1  11  12   3  11  12   3  161.75 1.5
hb-dihd   1  1  1  1   2   3  12  11   2   3  12  11   79.65 0.15
hb-dihd   1  2  1  1  12   3   2   4  12   3   2   4   69.75 0.15
hb-dihd   1  3  1  1   3  12  11  10   3  12  11  10   43.65 0.15
tbs-dist  1  1  1   9   3   9   3  -5.0 5.07 5.0 -1 +2
tbs-angl  1  1  1  1   2   3   9   2   3   9   81.57 1.5
tbs-angl  1  2  1  1   3   9   8   3   9   8   99.12 1.5
tbs-dihd  1  1  1  1   2   3   9   8   2   3   9   8  -13.33 0.15
tbs-dihd  1  2  1  1   4   2   3   9   4   2   3   9  165.45 0.15
tbs-dihd  1  3  1  1   3   9   8  10   3   9   8  10   42.00 0.15
"""


def dih(v):
    return v * math.pi / 180.0


def test_pdb_columns():
    st = N.read_pdb_cg(PDB)
    assert st.nmp == 14 and st.nunit == 2
    assert st.lunit2mp.tolist() == [[1, 12], [13, 14]]
    assert st.iclass_unit == [CLASS_RNA, CLASS_ION]
    assert st.imp2type[:3].tolist() == [MP_RNA_PHOS, MP_RNA_SUGAR, MP_RNA_BASE]
    assert st.imp2type[12] == MP_ION_MG and st.imp2type[13] == MP_ION_CL
    assert st.cmp2seq[12] == "Mg " and st.cmp2seq[13] == "Cl "
    assert st.cmp2atom[2] == " Gb "
    assert st.xyz[12].tolist() == [-205.195, -149.235, 130.726]
    assert st.xyz[13].tolist() == [12.345, 1.0, 2.0]
    assert st.ires_mp.tolist() == [1, 1, 1, 2, 2, 2, 3, 3, 3, 4, 4, 4, 5, 6]


@pytest.mark.parametrize("text,msg", [
    ("ATOM      1  S   RG  A   1       0.000   0.000   0.000\n"
     "ATOM      2  Gb  RG  B   1       0.000   0.000   0.000\n", "chainid"),
    ("ATOM      1  S   RG  A   1       0.000   0.000   0.000\n"
     "ATOM      2 MG   Mg  A   1       0.000   0.000   0.000\n", "iclass"),
    ("ATOM      1  Q   RG  A   1       0.000   0.000   0.000\n", "mp-type"),
    ("ATOM      1  X   ZZZ A   1       0.000   0.000   0.000\n", "unknown class"),
    ("ATOM      1  CA  ALA A   1       0.000   0.000   0.000\n", "outside the DT15 path"),
])
def test_pdb_errors(text, msg):
    with pytest.raises(N.NinfoError, match=msg):
        N.read_pdb_cg(text)


def test_hbsite_numbering():
    st = N.read_pdb_cg(PDB)
    tab, n, val = N.hbsite_table(st)
    # P 2 sites, S 4, G 5, C 3, A 4, U 3; ions none (setp_dtrna15.F90:36-66)
    assert tab[:12].tolist() == [[1, 2], [3, 6], [7, 11], [12, 13], [14, 17], [18, 20],
                                 [21, 22], [23, 26], [27, 30], [31, 32], [33, 36], [37, 39]]
    assert tab[12:].tolist() == [[0, 0], [0, 0]] and n == 39
    assert val[6:11].tolist() == [1, 2, 1, 2, 1] and val[2:6].tolist() == [2, 1, 1, 1]
    assert N.site_local("RG ", "N3") == 3 and N.site_local("RA ", "N3") == 2
    assert N.site_local("RA ", "N7") == 4 and N.site_local("RG ", "N7") == 5
    assert N.site_local("RU ", "O2'") == 1 and N.site_local("RU ", "OP2") == 2
    with pytest.raises(N.NinfoError, match="hbsite_local"):
        N.site_local("RC ", "N7")


def test_records():
    st = N.read_pdb_cg(PDB)
    s = N.build_system(st, N.read_ninfo(NINFO, st))
    assert s["nbd"] == 2 and s["ibd2mp"].tolist() == [[2, 3], [2, 4]]
    assert s["bd_nat"].tolist() == [4.9659, 3.8157] and s["coef_bd"].tolist() == [10.0, 64.0]
    assert s["ba_nat"][0] == (109.7214 / 180.0) * N.F_PI and s["iba2mp"].tolist() == [[3, 2, 4]]
    # bs-dist: B1 B2 P1 S1 P2 S2 P3 = imp1, imp2, imp1-2, imp1-1, imp1+1, imp1+2, imp1+4
    assert s["idtrna_st2mp"].tolist() == [[3, 6, 1, 2, 4, 5, 7]]
    assert s["dtrna_st_hsTm"].tolist() == [[4.7199, 4.370, 343.363]]
    assert s["dtrna_st_nat"][0].tolist() == [4.25, -148.22 * N.F_PI / 180.0, 175.98 * N.F_PI / 180.0]
    assert s["coef_dtrna_st"].tolist() == [[1.4, 4.0, 4.0]]
    # hb-dist 12-3 is stored as (3, 12); angles fill slots 3 and 4, the
    # dihedrals slots 5 and 6
    assert s["idtrna_hb2mp"].tolist() == [[3, 12, 2, 11, 4, 10]]
    assert np.allclose(s["dtrna_hb_nat"][0], [5.80] + [dih(v) for v in (142.31, 161.75, 79.65, 69.75, 43.65)],
                       rtol=1e-15, atol=0)
    assert s["coef_dtrna_hb"].tolist() == [[-5.86, 5.0, 1.5, 1.5, 0.15, 0.15, 0.15]]
    # atoms (N1 of G3, N3 of U12), (O6 of G3, O4 of U12); side 1 is imp1 =
    # bead 12 as read (read_nativeinfo.F90:582-603)
    u_off, g_off = 37 - 1, 7 - 1
    assert s["idtrna_hb2hbsite"].tolist() == [[u_off + N.site_local("RU ", "N3"), u_off + N.site_local("RU ", "O4"), 0,
                                              g_off + N.site_local("RG ", "N1"), g_off + N.site_local("RG ", "O6"), 0]]
    assert s["idtrna_hb2hbsite"].tolist() == [[38, 39, 0, 7, 10, 0]]
    assert s["flg_hb_tertiary"].tolist() == [1] and s["nhbsite"] == 39
    # tbs-dist 9-3 -> (3, 9) with the side types swapped: (+2, -1)
    assert s["idtrna_tst2mp"].tolist() == [[3, 9, 2, 8, 4, 10]]
    assert s["idtrna_tst2side"].tolist() == [[2, 1]] and s["flg_tst_exclusive"].tolist() == [[1, 0]]
    assert np.allclose(s["dtrna_tst_nat"][0], [5.07] + [dih(v) for v in (81.57, 99.12, -13.33, 165.45, 42.0)],
                       rtol=1e-15, atol=0)
    assert s["coef_dtrna_tst"].tolist() == [[-5.0, 5.0, 1.5, 1.5, 0.15, 0.15, 0.15]]
    # set-up: masses, DT15 exv, charges (P -1, Mg +2, Cl -1)
    assert s["cmass"][2] == N.MASS["G"] and s["cmass"][12] == N.MASS["MG"]
    assert s["exv_radius"][12] == 0.7926 and s["exv_epsilon"][12] == math.sqrt(0.894700)
    assert s["icharge2mp"].tolist() == [1, 4, 7, 10, 13, 14]
    assert s["coef_charge"].tolist() == [-1.0, -1.0, -1.0, -1.0, 2.0, -1.0]
    assert np.all(s["fric"] == N.FRIC_CONST_DEFAULT)


def test_stokes_friction_and_charge_change():
    st = N.read_pdb_cg(PDB)
    s = N.build_system(st, N.read_ninfo(NINFO, st), i_fric=1, viscosity=0.001, charge_change={10: 0.0})
    visc = 0.001 * math.sqrt(1.0e3 / 4184.0) * 6.022140857e23 * 1.0e-20
    assert s["fric"][1] == pytest.approx(6.0 * math.pi * visc * 4.0 / N.MASS["S"], rel=1e-15)
    assert s["fric"][12] == pytest.approx(6.0 * math.pi * visc * 4.28 / N.MASS["MG"], rel=1e-15)
    assert s["coef_charge"][s["icharge2mp"].tolist().index(10)] == 0.0


def _without(text, prefix):
    return "\n".join(l for l in text.splitlines() if not l.startswith(prefix)) + "\n"


@pytest.mark.parametrize("edit,msg", [
    (lambda t: _without(t, "hb-dihd   1  3"), "ihb does not have dihedral"),
    (lambda t: _without(t, "hb-angl   1  2"), "ihb does not have angle"),
    (lambda t: _without(t, "bs-dihd   1  2"), "ist does not have dihedral"),
    (lambda t: _without(t, "tbs-angl  1  1"), "itst does not have angle"),
    (lambda t: _without(t, "tbs-dihd  1  2"), "itst does not have dihedral"),
    (lambda t: t.replace("4.0 PSPS", "4.0 PSXX"), "read error"),
    (lambda t: t.replace("5.0 T 2", "5.0 Q 2"), "read error"),
    (lambda t: t.replace("5.0 T 2", "5.0 T 4"), "invalid nHB"),
    # atom columns not in lower-bead-first order: O6 is not a site of U12
    (lambda t: t.replace("N1 N3 O6 O4", "N3 N1 O4 O6"), "is not a site of bead 12"),
    (lambda t: t.replace("5.0 -1 +2", "5.0 -3 +2"), "read error"),
    # the DT15 bs-dist columns before h, s, Tm were added (energy0 dist coef type)
    (lambda t: t.replace("4.7199  4.370  343.363  4.25  1.4  G-C", "-3.731 4.25 1.40 C-C"), "read error"),
    (lambda t: t.replace("hb-angl   1  2  1  1  11  12   3", "hb-angl   1  2  1  1   9  12   3"), "read error"),
    (lambda t: t.replace("bond      2  1  1   2   4", "bond      2  1  1   2  40"), "out of range"),
    (lambda t: t.replace("hb-angl   1  1  1  1   2   3  12", "hb-angl   2  1  1  1   2   3  12"), "no distance record"),
    (lambda t: t.replace("bs-dist   1", "bs-dist   2").replace("bs-dihd   1", "bs-dihd   2"), "must run"),
    (lambda t: t + "contact 1 1 1 1 5 1 5 6.0 1.0 1 1.0 p-p\n", "outside the DT15 path"),
    (lambda t: t.replace("64.0000 SP", ""), "read error"),
])
def test_ninfo_errors(edit, msg):
    st = N.read_pdb_cg(PDB)
    with pytest.raises(N.NinfoError, match=msg):
        N.read_ninfo(edit(NINFO), st)


def test_one_by_one_offsets():
    """NINFO(2/2): the unit-local columns plus the offset of unit 2
    (read_nativeinfo.F90:101-102, 134-141)."""
    two = PDB.replace("TER\nATOM     13", "TER\nATOM     13").split("TER\n")[0] + "TER\n"
    text = two + two.replace(" A ", " B ")
    st = N.read_pdb_cg(text)
    assert st.lunit2mp.tolist() == [[1, 12], [13, 24]]
    local = "bond 1 2 2 99 99 2 3 4.9659 1.0 1.0 10.0 SG\n"
    ni = N.read_ninfo(local, st, all_in_one=False, units=(2, 2))
    assert ni.ibd2mp == [[14, 15]]


def test_writer_round_trip():
    s = synth.hairpin_tertiary()
    s["flg_hb_tertiary"] = (np.arange(s["nhb"]) % 2).astype(np.int32)
    s = synth.add_ions(s, 60.0, {"Mg": 2, "K": 4, "Cl": 3}, 9, clash=4.0)
    st = N.read_pdb_cg(N.write_pdb_cg(s))
    r = N.build_system(st, N.read_ninfo(N.write_ninfo(s), st), i_fric=0, fric_const=0.5)
    for k, v in s.items():
        if k in ("seq", "pairs", "ion_names"):
            continue
        a, b = np.asarray(v), np.asarray(r[k])
        if a.dtype.kind in "iu":
            assert np.array_equal(a, b), k
        elif k == "xyz":
            assert np.abs(a - b).max() <= 5.0001e-4
        else:
            # distances and coefficients exactly; angles through degrees within 1e-15
            assert a.shape == b.shape and np.allclose(a, b, rtol=1e-15, atol=0), k


needs_ref = pytest.mark.skipif(not REF or not os.path.isdir(REF), reason="TIS_REFERENCE_DIR not set")


@needs_ref
def test_reference_inputs_bwyv19(oracle_lib):
    """The reference's DT input in the current record layout (bwyv19.ninfo on
    bwyv19_force_check.*.pdb): counts match the file, every record's beads
    have the types its term expects, and the oracle evaluates the system."""
    from oracle.oracle import Oracle
    pdb = [f"{REF}/pdb/bwyv19_force_check.rna.pdb", f"{REF}/pdb/bwyv19_force_check.ion.pdb"]
    path = f"{REF}/ninfo/bwyv19.ninfo"
    st = N.read_pdb_cg(pdb)
    s = N.build_system(st, N.read_ninfo(path, st), i_fric=1, viscosity=0.000015, charge_change={85: 0.0})
    with open(path) as f:
        heads = [l.split()[0] for l in f if l.strip()]
    for rec, key in (("bond", "nbd"), ("angl", "nba"), ("bs-dist", "nst"), ("hb-dist", "nhb"), ("tbs-dist", "ntst")):
        assert s[key] == heads.count(rec), rec
    assert st.nmp == 291 and st.lunit2mp.tolist() == [[1, 85], [86, 291]]
    t = st.imp2type
    B, P, S = MP_RNA_BASE, MP_RNA_PHOS, MP_RNA_SUGAR
    for m in s["idtrna_st2mp"]:
        assert [t[i - 1] for i in m] == [B, B, P, S, P, S, P]
    for m in s["idtrna_tst2mp"]:
        assert [t[i - 1] for i in m] == [B, B, S, S, P, P]
    tab, _, _ = N.hbsite_table(st)
    for m, sites in zip(s["idtrna_hb2mp"], s["idtrna_hb2hbsite"]):
        assert t[m[0] - 1] in (B, S, P) and t[m[1] - 1] in (B, S, P)
        for side, bead in ((sites[:3], m[0]), (sites[3:], m[1])):
            used = side[side > 0]
            assert len(used) > 0
            assert np.all((used >= tab[bead - 1, 0]) & (used <= tab[bead - 1, 1]))
    # every phosphate (bead 85 with the CHARGE_CHANGE value 0) and every Mg
    assert s["ncharge"] == int(np.sum(t == P)) + 206 and s["coef_charge"][28] == 0.0
    par = synth.dt15_params(i_periodic=1, psize=(700.0, 700.0, 700.0), ionic_strength=0.057,
                            i_DH_cutoff_type=1, cutoff_ele=50.0)
    o = Oracle(s, par, [310.15])
    o.set_state(s["xyz"][None])
    o.neighbor()
    f, _ = o.force()
    e = o.energy()
    assert np.all(np.isfinite(f)) and np.all(np.isfinite(e))
    assert e[16 - 1] < 0 and e[17 - 1] + e[20 - 1] <= 0


@needs_ref
@pytest.mark.parametrize("name", ["dtrna15", "L10", "uuuu", "bwyv"])
def test_reference_inputs_old_bs_dist_layout(name):
    """These files carry bs-dist records without h, s and Tm; the current
    read_nativeinfo.F90:441-449 stops on them with a read error, and so
    does this reader."""
    pdb = {"dtrna15": "azo.rna.pdb", "L10": "L10.cg.pdb", "uuuu": "uuuu.pdb", "bwyv": "bwyv_cg.pdb"}[name]
    st = N.read_pdb_cg(f"{REF}/pdb/{pdb}")
    with pytest.raises(N.NinfoError, match="read error =>bs-dist"):
        N.read_ninfo(f"{REF}/ninfo/{name}.ninfo", st)


def test_oracle_tertiary_hbond_energy_split(oracle_lib):
    """energy_dtrna_hbond15.F90:135-143: 'T' bonds count in THBOND_DTRNA,
    the rest in HBOND_DTRNA; forces do not change."""
    from oracle.oracle import Oracle
    s = synth.hairpin_coords(synth.set_friction(synth.dt15_chain(22, 1, stem=6), 0.5), 6, seed=1)
    par = synth.dt15_params()
    out = []
    for flags in (None, (np.arange(s["nhb"]) % 2).astype(np.int32)):
        s2 = dict(s)
        if flags is not None:
            s2["flg_hb_tertiary"] = flags
        o = Oracle(s2, par, [300.0])
        o.set_state(s["xyz"][None])
        o.neighbor()
        f, _ = o.force()
        out.append((f, o.energy(reuse_hb=True)))
    (f0, e0), (f1, e1) = out
    assert np.array_equal(f0, f1)
    assert e0[20 - 1] == 0.0 and e1[20 - 1] < 0.0 and e1[17 - 1] < 0.0
    assert e1[17 - 1] + e1[20 - 1] == pytest.approx(e0[17 - 1], rel=1e-12)
    assert e1[0] == pytest.approx(e0[0], rel=1e-12)


def test_fixture_files_current():
    """The committed tests/golden/hairpin_tertiary.* files are what their
    generator writes now."""
    import importlib.util
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    spec = importlib.util.spec_from_file_location("make_ninfo_fixture", os.path.join(here, "make_ninfo_fixture.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    pdb, nin = mod.texts()
    with open(os.path.join(here, "hairpin_tertiary.cg.pdb")) as f:
        assert f.read() == pdb
    with open(os.path.join(here, "hairpin_tertiary.ninfo")) as f:
        assert f.read() == nin
    s = N.load(os.path.join(here, "hairpin_tertiary.cg.pdb"), os.path.join(here, "hairpin_tertiary.ninfo"))
    assert s["ntst"] == 3 and s["flg_hb_tertiary"].sum() > 0 and s["nunit"] == 2

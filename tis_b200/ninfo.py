"""Input formats of the DT15 path: the coarse-grained PDB of RNA chains and
ions, the native-info (.ninfo) records of the DT15 model, and the set-up
that turns them into the topology the library takes.

* ``read_pdb_cg`` follows src/read_pdb_cg.F90:76-170 (fixed columns
  ``(a6, i5, 1x, a4, a1, a3, a2, i4, 4x, 3f8.3)``, a unit ends at ``TER``
  or ``>>``, class and bead type from the residue and atom names).
* ``read_ninfo`` follows src/read_nativeinfo.F90: a first pass over
  bond/fene/angl/wca/bs-dist/hb-dist/tbs-dist records, a second over
  bs-dihd/hb-angl/hb-dihd/tbs-angl/tbs-dihd, then the completeness checks
  of :1107-1150.  The hydrogen-bond sites of hb-dist records need the
  structure (site numbering of setp_dtrna15.F90:36-66, atom names through
  ``site_local`` of read_nativeinfo.F90:1286-1336).
* ``build_system`` adds what setp_mass_fric.F90 (masses, friction),
  setp_dtrna15.F90:84-161 (excluded-volume radius and epsilon, site
  valences) and setp_native_charge.F90:82-112 (charges) derive from the
  structure, and returns the dict ``tis_b200.abi.make_topology`` takes.
* ``write_pdb_cg`` / ``write_ninfo`` write the same formats from such a
  dict, so synthetic systems can be exported and read back.

Every error the reference stops on (``util_error(ERROR%STOP_ALL, ...)``)
raises ``NinfoError`` with the offending line.  Four rules are stricter
than the reference: record numbers of each kind must run 1..n without
gaps (the reference indexes its arrays by the record number but counts
records), angle/dihedral records must refer to a distance record that
exists, every hb-dist atom must name a site of its own bead (the
reference adds the atom's local index to the bead's first site without
checking it), and a record must carry all its numeric columns (a short
line ends the reference's list-directed read without an error status and
leaves the previous record's values in the missing items).  Records of
models outside this path (contact, LJ, rouse, con_gauss,
basepair/basestack, dihd) raise as well.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

from .abi import (CLASS_ION, CLASS_RNA, MP_ION_CA2, MP_ION_CL, MP_ION_K, MP_ION_MG, MP_ION_NA,
                  MP_RNA_BASE, MP_RNA_PHOS, MP_RNA_SUGAR)

F_PI = 3.14159265358979323846264338327950288419716939937510  # const_physical.F90
N_AVO = 6.022140857e23
KCAL2JOUL = 4184.0
JOUL2KCAL = 1.0 / KCAL2JOUL

# chemical types (setp_mass_fric.F90:283-330): bead atom name -> type for
# RNA, residue name (after normalisation) -> type for ions
_ATOM_CHEM = {" P  ": "P", " S  ": "S", " Ab ": "A", " Gb ": "G", " Ub ": "U", " Cb ": "C"}
_ION_CHEM = {"Mg ": "MG", "Ca2": "CA2", "K  ": "K", "Na ": "NA", "Cl ": "CL"}
# para/general.para:76-87 (MASS) and :153-166 (RADIUS, the Stokes radii)
MASS = {"P": 62.972561, "S": 131.10668, "A": 134.11876, "G": 150.11816, "C": 110.09406,
        "U": 111.07882, "MG": 24.3050, "CL": 35.4500, "K": 39.1000, "NA": 22.9900, "CA2": 40.078}
STOKES_RADIUS = {"P": 3.1, "S": 4.0, "A": 3.9, "G": 4.1, "C": 3.8, "U": 3.8,
                 "MG": 4.28, "CL": 3.32, "K": 3.31, "NA": 3.58, "CA2": 4.12}
RMASS_DEFAULT = 10.0      # general.para rmass (i_mass = 0)
FRIC_CONST_DEFAULT = 0.25  # general.para fric_const (i_fric = 0)
VISCOSITY_DEFAULT = 0.001  # general.para viscosity [Pa s]
# para/rna.para:402-416 (DT15_exv_param): radius, epsilon
DT15_EXV = {"P": (2.1, 0.2), "S": (2.9, 0.2), "A": (2.8, 0.2), "G": (3.0, 0.2), "C": (2.7, 0.2),
            "U": (2.7, 0.2), "MG": (0.7926, 0.894700), "CA2": (1.7131, 0.459789),
            "CL": (1.9480, 0.265000), "K": (2.6580, 0.000328), "NA": (1.8680, 0.002770)}
# para/rna.para:495-507 (NHT19_exv_param, the DT19 model): radius, epsilon.
# It has no entries for the monovalent ions (the model keeps them implicit).
NHT19_EXV = {"P": (1.8900, 0.2), "S": (2.6100, 0.2), "A": (2.5200, 0.2), "G": (2.7000, 0.2),
             "C": (2.4300, 0.2), "U": (2.4300, 0.2), "MG": (2.0000, 0.894700), "CA2": (2.8000, 1.0)}
# para/electrostatic.para:42 (LENGTH_PER_UNIT of P, the Manning length b)
LENGTH_PER_UNIT_P = 4.38178046
# para/electrostatic.para:33-40 (CHARGE_TYPE)
CHARGE_TYPE = {"P": -1.0, "MG": 2.0, "CA2": 2.0, "K": 1.0, "NA": 1.0, "CL": -1.0}
# hydrogen-bond sites per bead (setp_dtrna15.F90:40-66) and their valences (:114-161)
_SITE_VALENCE = {" S  ": (2, 1, 1, 1), " P  ": (1, 1), " Ab ": (1, 1, 2, 1), " Cb ": (2, 1, 2),
                 " Gb ": (1, 2, 1, 2, 1), " Ub ": (2, 1, 1)}
_ION_TYPE = {"MG": MP_ION_MG, "CA2": MP_ION_CA2, "NA": MP_ION_NA, "K": MP_ION_K, "CL": MP_ION_CL}
# read_pdb_cg.F90:183-197: residue names of RNA units
_RNA_RES = {"RA ", "RU ", "RG ", "RC ", "OMG", "2MG", "M2G", "YYG", "1MG", "7MG", "OMU", "PSU",
            "H2U", "OMC", "5MC", "5MU", "1MA", "UR3", "MA6", "4OC", "  I", "PYY", "CB2", "AET",
            "QUO", "FHU", "T6A", "RIA", "MIA", "PRF"}
_PROTEIN_RES = {"ALA", "ARG", "ASN", "ASP", "CYS", "GLN", "GLU", "GLY", "HIS", "ILE", "LEU", "LYS",
                "MET", "PHE", "PRO", "SER", "THR", "TRP", "TYR", "VAL"}
# read_pdb_cg.F90:207-232: ion residue names -> normalised name
_ION_RES = {"MG ": "Mg ", " MG": "Mg ", "Mg ": "Mg ", " Mg": "Mg ", "Na ": "Na ", " Na": "Na ",
            "K  ": "K  ", " K ": "K  ", "  K": "K  ", "Cl ": "Cl ", " Cl": "Cl ",
            "CA2": "Ca2", "Ca2": "Ca2"}
_OTHER_MODELS = ("contact", "LJ", "rouse", "con_gauss", "basepair", "basestack", "dihd")


class NinfoError(ValueError):
    """An input the reference stops on (util_error ERROR%STOP_ALL)."""


# ----------------------------------------------------------------- CG PDB
@dataclass
class Structure:
    """Beads of one or more CG PDB files (read_pdb_cg.F90 outputs).
    ``lunit2mp`` is (nunit, 2) 1-based; the per-bead lists are 0-based by
    bead.  ``cmp2atom`` keeps the 4-character atom field, ``cmp2seq`` the
    3-character residue field (ion names normalised)."""
    xyz: np.ndarray
    cmp2atom: list
    cmp2seq: list
    imp2type: np.ndarray
    iclass_unit: list
    lunit2mp: np.ndarray
    ires_mp: np.ndarray

    @property
    def nmp(self) -> int:
        return len(self.cmp2atom)

    @property
    def nunit(self) -> int:
        return len(self.iclass_unit)

    def iclass_mp(self) -> np.ndarray:
        c = np.zeros(self.nmp, dtype=np.int32)
        for u, (a, b) in enumerate(self.lunit2mp):
            c[a - 1:b] = self.iclass_unit[u]
        return c


def _fread(field_text: str, decimals: int) -> float:
    """Fortran fw.d input: blanks read as zero, a field without a decimal
    point carries d implied decimals."""
    t = field_text.strip()
    if not t:
        return 0.0
    if "." in t or "e" in t.lower():
        return float(t)
    return int(t) / 10.0 ** decimals


def _iread(field_text: str) -> int:
    t = field_text.strip()
    return int(t) if t else 0


def _classify(atom: str, res: str):
    """read_pdb_cg.F90:172-240 (the classes of this path): returns
    (class, type, normalised residue name)."""
    if res in _RNA_RES:
        if atom == " S  ":
            return CLASS_RNA, MP_RNA_SUGAR, res
        if atom == " P  ":
            return CLASS_RNA, MP_RNA_PHOS, res
        if atom in (" Ab ", " Ub ", " Rb ", " Gb ", " Cb ", " Yb "):
            return CLASS_RNA, MP_RNA_BASE, res
        raise NinfoError(f"Error: unknown mp-type in read_pdb_cg; {res},{atom}")
    if res in _ION_RES:
        r = _ION_RES[res]
        return CLASS_ION, _ION_TYPE[_ION_CHEM[r]], r
    if res in _PROTEIN_RES or atom == " X1 ":
        raise NinfoError(f"residue {res!r} atom {atom!r}: protein and ligand units are outside the DT15 path")
    raise NinfoError(f"Error: unknown class in read_pdb_cg; {res},{atom}")


def read_pdb_cg(sources) -> Structure:
    """Reads CG PDB files (paths or text), appending their units in order
    like successive read_pdb_cg calls (read_pdb_cg.F90:76-170)."""
    if isinstance(sources, (str, os.PathLike)):
        sources = [sources]
    xyz, atoms, seqs, types, ires = [], [], [], [], []
    classes, lunit = [], []
    nres = 0
    for src in sources:
        text = src
        if isinstance(src, os.PathLike) or (isinstance(src, str) and "\n" not in src and os.path.exists(src)):
            with open(src) as f:
                text = f.read()
        reading = False
        chain_save = cls_save = resnum_save = None
        for raw in text.splitlines():
            line = raw[:72].ljust(72)
            if reading and (line[:3] == "TER" or line[:2] == ">>"):
                lunit[-1][1] = len(atoms)
                reading = False
            if line[:4] != "ATOM":
                continue
            atom, res, chain = line[12:16], line[17:20], line[20:22]
            try:
                resnum = _iread(line[22:26])
                x, y, z = (_fread(line[30 + 8 * k:38 + 8 * k], 3) for k in range(3))
            except ValueError as e:
                raise NinfoError(f"Error: cannot read pdb file in read_pdb_cg => {raw}") from e
            cls, typ, res = _classify(atom, res)
            if not reading:
                lunit.append([len(atoms) + 1, 0])
                classes.append(cls)
                nres += 1
                chain_save, cls_save, resnum_save = chain, cls, resnum
                reading = True
            else:
                if chain != chain_save:
                    raise NinfoError("Error: chainid /= chainid_save in read_pdb_cg")
                if cls != cls_save:
                    raise NinfoError("Error: iclass /= iclass_save in read_pdb_cg")
                if resnum != resnum_save:
                    nres += 1
                    resnum_save = resnum
            xyz.append((x, y, z))
            atoms.append(atom)
            seqs.append(res)
            types.append(typ)
            ires.append(nres)
        if reading:
            lunit[-1][1] = len(atoms)
    return Structure(xyz=np.array(xyz, dtype=np.float64).reshape(-1, 3), cmp2atom=atoms, cmp2seq=seqs,
                     imp2type=np.array(types, dtype=np.int32), iclass_unit=classes,
                     lunit2mp=np.array(lunit, dtype=np.int32).reshape(-1, 2),
                     ires_mp=np.array(ires, dtype=np.int32))


# -------------------------------------------------------------- hb sites
def hbsite_table(st: Structure):
    """imp2hbsite (setp_dtrna15.F90:36-66): (nmp, 2) first/last 1-based
    site of each RNA bead (0 for beads without sites), the site count and
    nvalence_hbsite (:114-161)."""
    cls = st.iclass_mp()
    tab = np.zeros((st.nmp, 2), dtype=np.int32)
    val = []
    n = 0
    for b in range(st.nmp):
        if cls[b] != CLASS_RNA:
            continue
        v = _SITE_VALENCE.get(st.cmp2atom[b])
        if v is None:
            continue
        tab[b] = (n + 1, n + len(v))
        n += len(v)
        val += v
    return tab, n, np.array(val, dtype=np.int32)


def site_local(res: str, atom: str) -> int:
    """Local index of an atom's hydrogen-bond site within its bead
    (read_nativeinfo.F90:1286-1336); ``res`` is the 3-character residue
    field, ``atom`` the atom name of the hb-dist record."""
    a = (atom + "    ")[:4]
    r2 = res[:2]
    s = 0
    if a[:3] == "O2'":
        s = 1
    elif a[:3] == "O4'":
        s = 2
    elif a[:3] == "O3'":
        s = 3
    elif a[:3] == "O5'":
        s = 4
    elif a[:3] == "OP1":
        s = 1
    elif a[:3] == "OP2":
        s = 2
    elif a[:2] == "N1":
        s = 1
    elif a[:2] == "O2":
        s = 1
    elif a[:2] == "N2":
        s = 2
    elif a[:2] == "N3":
        if r2 == "RG":
            s = 3
        elif r2 in ("RA", "RC", "RU"):
            s = 2
    elif a[:2] in ("O4", "N4", "N6"):
        s = 3
    elif a[:2] == "O6":
        s = 4
    elif a[:2] == "N7":
        if r2 == "RA":
            s = 4
        elif r2 == "RG":
            s = 5
    if s == 0:
        raise NinfoError(f"Error: in hbsite_local (read_nativeinfo): {res},{atom}")
    return s


# ------------------------------------------------------------------ ninfo
@dataclass
class NativeInfo:
    """Records of one or more .ninfo files in the reference's arrays
    (record-major, 1-based bead numbers, radians)."""
    ibd2mp: list = field(default_factory=list)
    bd_nat: list = field(default_factory=list)
    factor_bd: list = field(default_factory=list)
    coef_bd: list = field(default_factory=list)
    bd_type: list = field(default_factory=list)
    iba2mp: list = field(default_factory=list)
    ba_nat: list = field(default_factory=list)
    factor_ba: list = field(default_factory=list)
    coef_ba: list = field(default_factory=list)
    ba_type: list = field(default_factory=list)
    ifene2mp: list = field(default_factory=list)
    fene_nat: list = field(default_factory=list)
    coef_fene: list = field(default_factory=list)
    dist2_fene: list = field(default_factory=list)
    iwca2mp: list = field(default_factory=list)
    wca_nat: list = field(default_factory=list)
    coef_wca: list = field(default_factory=list)      # (rep, att) per record
    st: dict = field(default_factory=dict)             # ist -> record
    hb: dict = field(default_factory=dict)             # ihb -> record
    tst: dict = field(default_factory=dict)            # itst -> record


def _tokens(line: str):
    """Fortran list-directed input items (blank or comma separated)."""
    return line.replace(",", " ").split()


def _to_int(t: str, line: str) -> int:
    try:
        return int(t)
    except ValueError as e:
        raise NinfoError(f"read error =>{line}") from e


def _to_real(t: str, line: str) -> float:
    try:
        return float(t.replace("d", "e").replace("D", "e"))
    except ValueError as e:
        raise NinfoError(f"read error =>{line}") from e


def _items(line: str, kinds: str, n_required: int | None = None):
    """Reads list-directed items of kinds 'i' (integer), 'r' (real), 'c'
    (character); items past the end of the line stay None (an end-of-record
    status the reference accepts), a malformed item raises."""
    tok = _tokens(line)[1:]
    if n_required is not None and len(tok) < n_required:
        raise NinfoError(f"read error =>{line}")
    out = []
    for k, kind in enumerate(kinds):
        if k >= len(tok):
            out.append(None)
            continue
        t = tok[k]
        out.append(_to_int(t, line) if kind == "i" else _to_real(t, line) if kind == "r" else t)
    return out


def _deg_dih(v: float) -> float:
    """dih * F_PI / 180.0 (read_nativeinfo.F90:767 and the hb/tbs records)."""
    return v * F_PI / 180.0


def _deg_angl(v: float) -> float:
    """(ba / 180.0) * F_PI (read_nativeinfo.F90:231, angl records)."""
    return (v / 180.0) * F_PI


def read_ninfo(sources, st: Structure, all_in_one: bool = True, units=(1, 1), ninfo: NativeInfo | None = None):
    """Parses .ninfo files (paths or text) of the DT15 model against the
    structure ``st`` and returns a ``NativeInfo``.

    all_in_one=True is NINFO(all/all): bead numbers imp1.. are global.
    all_in_one=False is NINFO(i/j) for the unit pair ``units``: bead numbers
    are the unit-local imp*un columns plus the units' offsets
    (read_nativeinfo.F90:101-102).  Pass ``ninfo`` to append to records
    read before, like successive read_nativeinfo calls."""
    if isinstance(sources, (str, os.PathLike)):
        sources = [sources]
    ni = ninfo if ninfo is not None else NativeInfo()
    iu, ju = units
    ii = int(st.lunit2mp[iu - 1, 0]) - 1
    jj = int(st.lunit2mp[ju - 1, 0]) - 1
    site_tab, _, _ = hbsite_table(st)
    texts = []
    for src in sources:
        if isinstance(src, os.PathLike) or (isinstance(src, str) and "\n" not in src and os.path.exists(src)):
            with open(src) as f:
                texts.append(f.read())
        else:
            texts.append(src)
    n0 = (len(ni.st), len(ni.hb), len(ni.tst))
    new_st, new_hb, new_tst = set(), set(), set()

    def pick(g, ng, loc, off, line):
        # ALL_IN_ONE: the imp columns plus the unit offset (0 for NINFO(all/all));
        # ONE_BY_ONE: the unit-local imp*un columns plus the offset
        out = [(g[k] if all_in_one else loc[k]) + off[k] for k in range(ng)]
        for v in out:
            if not (1 <= v <= st.nmp):
                raise NinfoError(f"bead {v} out of range 1..{st.nmp} =>{line}")
        return out

    # ---- first pass (read_nativeinfo.F90:111-700)
    for text in texts:
        for raw in text.splitlines():
            line = raw[:256]
            head = line.split()[0] if line.split() else ""
            if head in _OTHER_MODELS:
                raise NinfoError(f"'{head}' records belong to a model outside the DT15 path =>{line}")
            if line[:4] == "bond":
                v = _items(line, "i" * 7 + "rrrr" + "c", 11)
                imp = pick(v[3:5], 2, v[5:7], (ii, ii), line)
                ni.ibd2mp.append(imp)
                ni.bd_nat.append(v[7]); ni.factor_bd.append(v[8]); ni.coef_bd.append(v[10])
                ni.bd_type.append(v[11] or "")
            elif line[:4] == "fene":
                v = _items(line, "i" * 7 + "rrr" + "c", 10)
                ni.ifene2mp.append(pick(v[3:5], 2, v[5:7], (ii, ii), line))
                ni.fene_nat.append(v[7]); ni.dist2_fene.append(v[8]); ni.coef_fene.append(v[9])
            elif line[:4] == "angl":
                v = _items(line, "i" * 9 + "rrrr" + "c", 13)
                ni.iba2mp.append(pick(v[3:6], 3, v[6:9], (ii, ii, ii), line))
                ni.ba_nat.append(_deg_angl(v[9])); ni.factor_ba.append(v[10]); ni.coef_ba.append(v[12])
                ni.ba_type.append(v[13] or "")
            elif line[:3] == "wca":
                v = _items(line, "i" * 7 + "rrr", 10)
                ni.iwca2mp.append(pick(v[3:5], 2, v[5:7], (ii, jj), line))
                ni.wca_nat.append(v[7]); ni.coef_wca.append((v[8], v[9]))
            elif line[:7] == "bs-dist":
                v = _items(line, "i" * 7 + "rrrrr" + "c", 12)
                ist = v[0]
                if ist < 1:
                    raise NinfoError(f"ibs of bs-dist is out of range =>{line}")
                b1, b2 = pick(v[3:5], 2, v[5:7], (ii, jj), line)
                ni.st[ist] = dict(mp=[b1, b2, b1 - 2, b1 - 1, b1 + 1, b1 + 2, b1 + 4],
                                  nat=[v[10], 0.0, 0.0], coef=[v[11], 0.0, 0.0], hsTm=[v[7], v[8], v[9]],
                                  check=[False, False], line=line)
                new_st.add(ist)
            elif line[:7] == "hb-dist":
                v = _items(line, "i" * 7 + "rrr" + "c" + "i", 12)
                nhb_atoms = v[11]
                if nhb_atoms not in (1, 2, 3):
                    raise NinfoError(f"invalid nHB or atom names:{line}")
                tok = _tokens(line)[13:13 + 2 * nhb_atoms]
                if len(tok) < 2 * nhb_atoms:
                    raise NinfoError(f"read error =>{line}")
                ihb = v[0]
                if ihb < 1:
                    raise NinfoError(f"ihb of hb-dist is out of range =>{line}")
                imp1, imp2 = pick(v[3:5], 2, v[5:7], (ii, jj), line)
                mp = [min(imp1, imp2), max(imp1, imp2), 0, 0, 0, 0]
                a = [[tok[2 * k][:4], tok[2 * k + 1][:4]] for k in range(nhb_atoms)]
                # read_nativeinfo.F90:582-603: the atom columns list the
                # lower-numbered bead's atom first; they are swapped when
                # imp2 < imp1, so that side 1 of slot k is imp1's site of
                # atom a(k,1) and side 2 imp2's site of atom a(k,2)
                if imp2 < imp1:
                    a = [[q[1], q[0]] for q in a]
                off1 = int(site_tab[imp1 - 1, 0]) - 1
                off2 = int(site_tab[imp2 - 1, 0]) - 1
                sites = np.zeros((2, 3), dtype=np.int32)
                for k in range(nhb_atoms):
                    sites[0, k] = off1 + site_local(st.cmp2seq[imp1 - 1], a[k][0])
                    sites[1, k] = off2 + site_local(st.cmp2seq[imp2 - 1], a[k][1])
                    for sd, b in ((0, imp1), (1, imp2)):
                        if not (site_tab[b - 1, 0] <= sites[sd, k] <= site_tab[b - 1, 1]):
                            raise NinfoError(f"hydrogen-bond atom {a[k][sd]} is not a site of bead {b} =>{line}")
                if v[10][:1] == "S":
                    tert = False
                elif v[10][:1] == "T":
                    tert = True
                else:
                    raise NinfoError(f"read error =>{line}")
                ni.hb[ihb] = dict(mp=mp, nat=[v[8], 0.0, 0.0, 0.0, 0.0, 0.0],
                                  coef=[v[7], v[9], 0.0, 0.0, 0.0, 0.0, 0.0], sites=sites, tertiary=tert,
                                  check_angl=[False, False], check_dihd=[False, False, False], line=line)
                new_hb.add(ihb)
            elif line[:8] == "tbs-dist":
                v = _items(line, "i" * 7 + "rrr" + "ii", 12)
                itst = v[0]
                if itst < 1:
                    raise NinfoError(f"ist of st-dist is out of range =>{line}")
                imp1, imp2 = pick(v[3:5], 2, v[5:7], (ii, jj), line)
                t1, t2 = v[10], v[11]
                if imp1 > imp2:
                    imp1, imp2, t1, t2 = imp2, imp1, t2, t1
                side, excl = [], []
                for t in (t1, t2):
                    side.append(1 if t < 0 else 2)
                    if abs(t) == 1:
                        excl.append(0)
                    elif abs(t) == 2:
                        excl.append(1)
                    else:
                        raise NinfoError(f"read error =>{line}")
                ni.tst[itst] = dict(mp=[imp1, imp2, imp1 - 1, imp2 - 1, imp1 + 1, imp2 + 1],
                                    nat=[v[8], 0.0, 0.0, 0.0, 0.0, 0.0],
                                    coef=[v[7], v[9], 0.0, 0.0, 0.0, 0.0, 0.0], side=side, excl=excl,
                                    check_angl=[False, False], check_dihd=[False, False, False], line=line)
                new_tst.add(itst)
    for name, new, n_before in (("bs-dist", new_st, n0[0]), ("hb-dist", new_hb, n0[1]),
                                ("tbs-dist", new_tst, n0[2])):
        if new and sorted(new) != list(range(n_before + 1, n_before + len(new) + 1)):
            raise NinfoError(f"{name} record numbers must run {n_before + 1}..{n_before + len(new)}")

    def need(table, key, kind, line):
        rec = table.get(key)
        if rec is None:
            raise NinfoError(f"{kind} record {key} has no distance record =>{line}")
        return rec

    def assign(rec, slot, value, line):
        # read_nativeinfo.F90:866-872 and the like: keep a matching bead,
        # fill an empty slot, stop on a conflicting one
        if rec["mp"][slot] == value:
            return
        if rec["mp"][slot] == 0:
            rec["mp"][slot] = value
            return
        raise NinfoError(f"read error =>{line}")

    # ---- second pass (read_nativeinfo.F90:727-1105)
    for text in texts:
        for raw in text.splitlines():
            line = raw[:256]
            if line[:7] == "bs-dihd":
                v = _items(line, "i" * 12 + "rr" + "c", 14)
                rec = need(ni.st, v[0], "bs-dihd", line)
                imp = pick(v[4:8], 4, v[8:12], (ii,) * 4, line)
                dih = _deg_dih(v[12])
                m = rec["mp"]
                ctype = (v[14] or "")[:4]
                if ctype == "PSPS":
                    if not (imp == m[2:6] or imp[::-1] == m[2:6]):
                        m[2:6] = imp
                    rec["nat"][1] = dih; rec["coef"][1] = v[13]; rec["check"][0] = True
                elif ctype == "SPSP":
                    if not (imp == m[3:7] or imp[::-1] == m[3:7]):
                        m[6] = imp[3]
                    rec["nat"][2] = dih; rec["coef"][2] = v[13]; rec["check"][1] = True
                else:
                    raise NinfoError(f"read error =>{line}")
            elif line[:7] == "hb-angl":
                v = _items(line, "i" * 10 + "rr", 12)
                rec = need(ni.hb, v[0], "hb-angl", line)
                i1, i2, i3 = pick(v[4:7], 3, v[7:10], (ii,) * 3, line)
                if i1 > i3:
                    i1, i3 = i3, i1
                m = rec["mp"]
                ba = _deg_dih(v[10])
                if i2 == m[0] and i3 == m[1]:
                    assign(rec, 2, i1, line)
                    rec["nat"][1] = ba; rec["coef"][2] = v[11]; rec["check_angl"][0] = True
                elif i1 == m[0] and i2 == m[1]:
                    assign(rec, 3, i3, line)
                    rec["nat"][2] = ba; rec["coef"][3] = v[11]; rec["check_angl"][1] = True
                else:
                    raise NinfoError(f"read error =>{line}")
            elif line[:7] == "hb-dihd":
                v = _items(line, "i" * 12 + "rr", 14)
                rec = need(ni.hb, v[0], "hb-dihd", line)
                i1, i2, i3, i4 = pick(v[4:8], 4, v[8:12], (ii,) * 4, line)
                if i1 > i4:
                    i1, i2, i3, i4 = i4, i3, i2, i1
                m = rec["mp"]
                dih = _deg_dih(v[12])
                if i2 == m[0] and i3 == m[1]:
                    assign(rec, 2, i1, line)
                    assign(rec, 3, i4, line)
                    rec["nat"][3] = dih; rec["coef"][4] = v[13]; rec["check_dihd"][0] = True
                elif i3 == m[0] and i4 == m[1]:
                    assign(rec, 2, i2, line)
                    m[4] = i1
                    rec["nat"][4] = dih; rec["coef"][5] = v[13]; rec["check_dihd"][1] = True
                elif i1 == m[0] and i2 == m[1]:
                    assign(rec, 3, i3, line)
                    m[5] = i4
                    rec["nat"][5] = dih; rec["coef"][6] = v[13]; rec["check_dihd"][2] = True
                else:
                    raise NinfoError(f"read error =>{line}")
            elif line[:8] == "tbs-angl":
                v = _items(line, "i" * 10 + "rr", 12)
                rec = need(ni.tst, v[0], "tbs-angl", line)
                i1, i2, i3 = pick(v[4:7], 3, v[7:10], (ii,) * 3, line)
                if i1 > i3:
                    i1, i3 = i3, i1
                m = rec["mp"]
                ba = _deg_dih(v[10])
                if i1 == m[2] and i2 == m[0] and i3 == m[1]:
                    rec["nat"][1] = ba; rec["coef"][2] = v[11]; rec["check_angl"][0] = True
                elif i1 == m[0] and i2 == m[1] and i3 == m[3]:
                    rec["nat"][2] = ba; rec["coef"][3] = v[11]; rec["check_angl"][1] = True
                else:
                    raise NinfoError(f"read error =>{line}")
            elif line[:8] == "tbs-dihd":
                v = _items(line, "i" * 12 + "rr", 14)
                rec = need(ni.tst, v[0], "tbs-dihd", line)
                i1, i2, i3, i4 = pick(v[4:8], 4, v[8:12], (ii,) * 4, line)
                if i1 > i4:
                    i1, i2, i3, i4 = i4, i3, i2, i1
                m = rec["mp"]
                dih = _deg_dih(v[12])
                if [i1, i2, i3, i4] == [m[2], m[0], m[1], m[3]]:
                    rec["nat"][3] = dih; rec["coef"][4] = v[13]; rec["check_dihd"][0] = True
                elif [i1, i2, i3, i4] == [m[4], m[2], m[0], m[1]]:
                    rec["nat"][4] = dih; rec["coef"][5] = v[13]; rec["check_dihd"][1] = True
                elif [i1, i2, i3, i4] == [m[0], m[1], m[3], m[5]]:
                    rec["nat"][5] = dih; rec["coef"][6] = v[13]; rec["check_dihd"][2] = True
                else:
                    raise NinfoError(f"read error =>{line}")
    # ---- completeness (read_nativeinfo.F90:1107-1150)
    for ihb in sorted(new_hb):
        r = ni.hb[ihb]
        if not all(r["check_angl"]):
            raise NinfoError(f"Error in ninfo: following ihb does not have angle: {ihb}")
        if not all(r["check_dihd"]):
            raise NinfoError(f"Error in ninfo: following ihb does not have dihedral: {ihb}")
    for ist in sorted(new_st):
        if not all(ni.st[ist]["check"]):
            raise NinfoError(f"Error in ninfo: following ist does not have dihedral: {ist}")
    for itst in sorted(new_tst):
        r = ni.tst[itst]
        if not all(r["check_angl"]):
            raise NinfoError(f"Error in ninfo: following itst does not have angle: {itst}")
        if not all(r["check_dihd"]):
            raise NinfoError(f"Error in ninfo: following itst does not have dihedral: {itst}")
    return ni


# -------------------------------------------------------------------- PMF
def read_pmf(source) -> dict:
    """The Mg-P potential of mean force file of the DT19 model
    (setp_pmf.F90:31-105): lines "r V(r)" on a uniform grid.  Returns the
    tis_params fields pmf_nbin, pmf_rmin, pmf_rbin (second r minus the
    first), pmf_rmax (the last r read) and pmf_mg_p.  A spacing that departs
    from the first by more than 1e-4 stops the reference, and raises here."""
    text = source
    if isinstance(source, os.PathLike) or (isinstance(source, str) and "\n" not in source and os.path.exists(source)):
        with open(source) as f:
            text = f.read()
    rs, vs = [], []
    for raw in text.splitlines():
        tok = _tokens(raw)
        if not tok:
            continue
        if len(tok) < 2:
            raise NinfoError(f"Error: cannot read a line of PMF file: {raw}")
        rs.append(_to_real(tok[0], raw)); vs.append(_to_real(tok[1], raw))
    if len(rs) < 2:
        raise NinfoError("Error: cannot read the second line of PMF file")
    rbin = rs[1] - rs[0]
    for k in range(2, len(rs)):
        if abs(rs[k] - rs[k - 1] - rbin) > 0.0001:
            raise NinfoError(f"Error: bin width is not uniform in PMF file (line {k + 1})")
    if len(rs) > 3000:
        raise NinfoError("Error: Nbin > MXPMFBIN in setp_pmf")
    return dict(pmf_nbin=len(rs), pmf_rmin=rs[0], pmf_rbin=rbin, pmf_rmax=rs[-1],
                pmf_mg_p=np.array(vs, dtype=np.float64))


# ------------------------------------------------------------------ set-up
def _chemical(st: Structure, b: int) -> str:
    """imp2chemicaltype (setp_mass_fric.F90:283-330) for RNA beads and ions."""
    a = st.cmp2atom[b]
    if a in _ATOM_CHEM:
        return _ATOM_CHEM[a]
    r = st.cmp2seq[b]
    if r in _ION_CHEM:
        return _ION_CHEM[r]
    raise NinfoError(f"Error: unknown chemical type in setp_mass_fric; imp= {b + 1}")


def build_system(st: Structure, ni: NativeInfo, *, i_mass: int = 1, i_fric: int = 0,
                 fric_const: float = FRIC_CONST_DEFAULT, viscosity: float = VISCOSITY_DEFAULT,
                 i_simulate_type: int = 1, charge_change: dict | None = None,
                 ele_units=None, i_dtrna_model: int = 2015) -> dict:
    """The topology dict of ``st`` + ``ni`` (see tis_b200.abi.make_topology).

    i_mass 1: masses by chemical type; 0: general.para rmass for every bead
    (setp_mass_fric.F90:40-54).  i_fric 1: Stokes friction
    6 pi eta r (/ m for Langevin) with eta in (Da)(A^-1)(tau^-1)
    (setp_mass_fric.F90:58-113); 0: fric_const.  charge_change maps a
    1-based bead to its charge (CHARGE_CHANGE lines; flg_charge_fixed marks
    them, so that i_charge = 1 keeps them); ele_units, when given, lists the
    1-based units whose beads carry charges (flag_ele), default all units
    (setp_native_charge.F90:82-112).  i_dtrna_model 2019 takes the NHT19
    excluded-volume table (setp_dtrna15.F90:25-28)."""
    n = st.nmp
    chem = [_chemical(st, b) for b in range(n)]
    if i_mass == 1:
        cmass = np.array([MASS[c] for c in chem])
    elif i_mass == 0:
        cmass = np.full(n, RMASS_DEFAULT)
    else:
        raise NinfoError("i_mass must be 0 or 1")
    fric = np.full(n, float(fric_const))
    if i_fric == 1:
        if i_simulate_type == 1:      # SIM%LANGEVIN
            visc = viscosity * math.sqrt(1.0e3 * JOUL2KCAL) * N_AVO * 1.0e-20
            fric = np.array([6.0 * F_PI * visc * STOKES_RADIUS[c] / MASS[c] for c in chem])
        elif i_simulate_type == 6:    # SIM%BROWNIAN_HI keeps fric_const
            pass
        else:
            raise NinfoError("i_fric = 1 is set up here for Langevin and Brownian-HI runs")
    elif i_fric != 0:
        raise NinfoError("i_fric must be 0 or 1")
    if i_dtrna_model == 2019:
        missing = sorted({c for c in chem if c not in NHT19_EXV})
        if missing:
            raise NinfoError(f"the DT19 exv table (NHT19_exv_param) has no entry for {missing}")
        table = NHT19_EXV
    elif i_dtrna_model in (0, 2015):
        table = DT15_EXV
    else:
        raise NinfoError("i_dtrna_model must be 2015 or 2019")
    exv_radius = np.array([table[c][0] for c in chem])
    exv_epsilon = np.sqrt(np.array([table[c][1] for c in chem]))

    # charges in bead order, unit by unit (setp_native_charge.F90:82-112)
    change = dict(charge_change or {})
    units = range(1, st.nunit + 1) if ele_units is None else sorted(ele_units)
    qb, qv, qfix = [], [], []
    for u in units:
        a, b = st.lunit2mp[u - 1]
        for imp in range(a, b + 1):
            if imp in change:
                qb.append(imp); qv.append(float(change[imp])); qfix.append(1)
            elif st.iclass_unit[u - 1] == CLASS_RNA and st.imp2type[imp - 1] == MP_RNA_PHOS:
                qb.append(imp); qv.append(CHARGE_TYPE["P"]); qfix.append(0)
            elif st.iclass_unit[u - 1] == CLASS_ION:
                qb.append(imp); qv.append(CHARGE_TYPE[chem[imp - 1]]); qfix.append(0)
    site_tab, nsite, valence = hbsite_table(st)

    def arr(x, dt, k):
        return np.array(x, dtype=dt).reshape(-1, k)

    st_ids = sorted(ni.st)
    hb_ids = sorted(ni.hb)
    tst_ids = sorted(ni.tst)
    sysd = dict(
        nmp=n, nunit=st.nunit, lunit2mp=st.lunit2mp.astype(np.int32),
        iclass_unit=np.array(st.iclass_unit, dtype=np.int32), imp2type=st.imp2type.astype(np.int32),
        cmass=cmass, fric=fric, exv_radius=exv_radius, exv_epsilon=exv_epsilon,
        ncharge=len(qb), icharge2mp=np.array(qb, dtype=np.int32), coef_charge=np.array(qv),
        flg_charge_fixed=np.array(qfix, dtype=np.int32),
        nbd=len(ni.ibd2mp), ibd2mp=arr(ni.ibd2mp, np.int32, 2), bd_nat=np.array(ni.bd_nat),
        coef_bd=np.array(ni.coef_bd),
        nba=len(ni.iba2mp), iba2mp=arr(ni.iba2mp, np.int32, 3), ba_nat=np.array(ni.ba_nat),
        coef_ba=np.array(ni.coef_ba),
        nfene=len(ni.ifene2mp), ifene2mp=arr(ni.ifene2mp, np.int32, 2), fene_nat=np.array(ni.fene_nat),
        coef_fene=np.array(ni.coef_fene), dist2_fene=np.array(ni.dist2_fene),
        nwca=len(ni.iwca2mp), iwca2mp=arr(ni.iwca2mp, np.int32, 2), wca_nat=np.array(ni.wca_nat),
        coef_wca=np.array(ni.coef_wca, dtype=np.float64).reshape(-1, 2).T.copy(),
        nst=len(st_ids), idtrna_st2mp=arr([ni.st[i]["mp"] for i in st_ids], np.int32, 7),
        dtrna_st_nat=arr([ni.st[i]["nat"] for i in st_ids], np.float64, 3),
        coef_dtrna_st=arr([ni.st[i]["coef"] for i in st_ids], np.float64, 3),
        dtrna_st_hsTm=arr([ni.st[i]["hsTm"] for i in st_ids], np.float64, 3),
        nhb=len(hb_ids), idtrna_hb2mp=arr([ni.hb[i]["mp"] for i in hb_ids], np.int32, 6),
        dtrna_hb_nat=arr([ni.hb[i]["nat"] for i in hb_ids], np.float64, 6),
        coef_dtrna_hb=arr([ni.hb[i]["coef"] for i in hb_ids], np.float64, 7),
        idtrna_hb2hbsite=arr([ni.hb[i]["sites"].ravel() for i in hb_ids], np.int32, 6),
        flg_hb_tertiary=np.array([1 if ni.hb[i]["tertiary"] else 0 for i in hb_ids], dtype=np.int32),
        nhbsite=nsite, nvalence_hbsite=valence,
        ntst=len(tst_ids), idtrna_tst2mp=arr([ni.tst[i]["mp"] for i in tst_ids], np.int32, 6),
        dtrna_tst_nat=arr([ni.tst[i]["nat"] for i in tst_ids], np.float64, 6),
        coef_dtrna_tst=arr([ni.tst[i]["coef"] for i in tst_ids], np.float64, 7),
        idtrna_tst2side=arr([ni.tst[i]["side"] for i in tst_ids], np.int32, 2),
        flg_tst_exclusive=arr([ni.tst[i]["excl"] for i in tst_ids], np.int32, 2),
        xyz=st.xyz.copy(),
    )
    _check_indices(sysd)
    return sysd


def _check_indices(s: dict):
    """Every bead number of every record lies in 1..nmp (the reference
    would index out of its arrays otherwise)."""
    n = s["nmp"]
    for k in ("ibd2mp", "iba2mp", "ifene2mp", "iwca2mp", "idtrna_st2mp", "idtrna_hb2mp", "idtrna_tst2mp"):
        a = np.asarray(s[k])
        if a.size and (a.min() < 1 or a.max() > n):
            bad = int(np.argwhere((a < 1) | (a > n))[0][0]) + 1
            raise NinfoError(f"{k}: record {bad} refers to a bead outside 1..{n}")
    h = np.asarray(s["idtrna_hb2hbsite"])
    if h.size and (h.min() < 0 or h.max() > s["nhbsite"]):
        raise NinfoError("idtrna_hb2hbsite refers to a site outside 1..nhbsite")


def load(pdb, ninfo, **setup) -> dict:
    """read_pdb_cg + read_ninfo (NINFO(all/all)) + build_system."""
    st = read_pdb_cg(pdb)
    return build_system(st, read_ninfo(ninfo, st), **setup)


# ----------------------------------------------------------------- writers
_BASE_ATOM = {"A": " Ab ", "G": " Gb ", "C": " Cb ", "U": " Ub "}
_ION_PDB = {MP_ION_MG: ("MG  ", "Mg "), MP_ION_CA2: ("CA  ", "CA2"), MP_ION_NA: ("NA  ", "Na "),
            MP_ION_K: ("K   ", "K  "), MP_ION_CL: ("CL  ", "Cl ")}


def _rna_names(sysd: dict, u0: int, u1: int):
    """Atom and residue names of the beads u0..u1 (0-based, inclusive) of an
    RNA unit: the residue of each bead is its nucleotide's base, taken
    from sysd['seq'] in nucleotide order (a nucleotide starts at each
    sugar or phosphate that follows a base)."""
    seq = sysd["seq"]
    typ = sysd["imp2type"]
    names, res, resnum = [], [], []
    k = 0
    seen_base = False
    for b in range(u0, u1 + 1):
        t = int(typ[b])
        if t in (MP_RNA_PHOS, MP_RNA_SUGAR) and seen_base:
            k += 1
            seen_base = False
        if t == MP_RNA_BASE:
            seen_base = True
        base = seq[k]
        names.append(" P  " if t == MP_RNA_PHOS else " S  " if t == MP_RNA_SUGAR else _BASE_ATOM[base])
        res.append("R" + base + " ")
        resnum.append(k + 1)
    return names, res, resnum


def write_pdb_cg(sysd: dict, chains: str = "ABCDEFGHIJKLMNOPQRSTUVWXYZ") -> str:
    """CG PDB text of a topology dict (one TER-terminated block per unit),
    in the columns read_pdb_cg reads."""
    out = []
    xyz = np.asarray(sysd["xyz"], dtype=np.float64)
    iatom = 0
    for u, (a, b) in enumerate(np.asarray(sysd["lunit2mp"]).reshape(-1, 2)):
        ch = " " + chains[u % len(chains)]
        if int(sysd["iclass_unit"][u]) == CLASS_RNA:
            names, res, resnum = _rna_names(sysd, a - 1, b - 1)
        else:
            names = [_ION_PDB[int(sysd["imp2type"][i])][0] for i in range(a - 1, b)]
            res = [_ION_PDB[int(sysd["imp2type"][i])][1] for i in range(a - 1, b)]
            resnum = list(range(1, b - a + 2))
        for k, i in enumerate(range(a - 1, b)):
            iatom += 1
            x, y, z = xyz[i]
            out.append(f"ATOM  {iatom % 100000:5d} {names[k]} {res[k]}{ch}{resnum[k] % 10000:4d}    "
                       f"{x:8.3f}{y:8.3f}{z:8.3f}")
        out.append("TER")
    return "\n".join(out) + "\n"


def _deg(r: float) -> float:
    return r * 180.0 / F_PI


def write_ninfo(sysd: dict, hb_atoms=None) -> str:
    """NINFO(all/all) text of a topology dict: bond, angl, bs-dist/-dihd,
    hb-dist/-angl/-dihd and tbs-dist/-angl/-dihd records in the reference's
    columns, natural values with 17 significant digits.  hb_atoms[k] lists
    the (atom of bead 1, atom of bead 2) pairs of hydrogen bond k; by
    default they are recovered from its site numbers."""
    r = []
    g = lambda v: repr(float(v))   # noqa: E731  shortest round-trip decimal
    ibd = np.asarray(sysd.get("ibd2mp", np.zeros((0, 2)))).reshape(-1, 2)
    for k, (i, j) in enumerate(ibd):
        r.append(f"bond {k + 1} 1 1 {i} {j} {i} {j} {g(sysd['bd_nat'][k])} 1.0 1.0 {g(sysd['coef_bd'][k])}")
    iba = np.asarray(sysd.get("iba2mp", np.zeros((0, 3)))).reshape(-1, 3)
    for k, (i, j, l) in enumerate(iba):
        r.append(f"angl {k + 1} 1 1 {i} {j} {l} {i} {j} {l} {g(_deg(sysd['ba_nat'][k]))} 1.0 1.0 "
                 f"{g(sysd['coef_ba'][k])}")
    for k in range(int(sysd.get("nst", 0))):
        m = [int(x) for x in sysd["idtrna_st2mp"][k]]
        nat, cf, hs = sysd["dtrna_st_nat"][k], sysd["coef_dtrna_st"][k], sysd["dtrna_st_hsTm"][k]
        r.append(f"bs-dist {k + 1} 1 1 {m[0]} {m[1]} {m[0]} {m[1]} {g(hs[0])} {g(hs[1])} {g(hs[2])} "
                 f"{g(nat[0])} {g(cf[0])}")
        p = m[2:6]
        r.append(f"bs-dihd {k + 1} 1 1 1 {p[0]} {p[1]} {p[2]} {p[3]} {p[0]} {p[1]} {p[2]} {p[3]} "
                 f"{g(_deg(nat[1]))} {g(cf[1])} PSPS")
        p = m[3:7]
        r.append(f"bs-dihd {k + 1} 2 1 1 {p[0]} {p[1]} {p[2]} {p[3]} {p[0]} {p[1]} {p[2]} {p[3]} "
                 f"{g(_deg(nat[2]))} {g(cf[2])} SPSP")
    nhb = int(sysd.get("nhb", 0))
    if nhb:
        st = read_pdb_cg(write_pdb_cg(sysd))
        tab, _, _ = hbsite_table(st)
        tert = sysd.get("flg_hb_tertiary")
    for k in range(nhb):
        m = [int(x) for x in sysd["idtrna_hb2mp"][k]]
        nat, cf = sysd["dtrna_hb_nat"][k], sysd["coef_dtrna_hb"][k]
        sites = np.asarray(sysd["idtrna_hb2hbsite"][k]).reshape(2, 3)
        if hb_atoms is not None:
            pairs = hb_atoms[k]
        else:
            pairs = []
            for q in range(3):
                if sites[0, q] <= 0:
                    break
                pairs.append((_site_atom(st, tab, m[0], sites[0, q]), _site_atom(st, tab, m[1], sites[1, q])))
        kind = "T" if (tert is not None and tert[k]) else "S"
        at = " ".join(f"{x} {y}" for x, y in pairs)
        r.append(f"hb-dist {k + 1} 1 1 {m[0]} {m[1]} {m[0]} {m[1]} {g(cf[0])} {g(nat[0])} {g(cf[1])} "
                 f"{kind} {len(pairs)} {at}")
        r.append(f"hb-angl {k + 1} 1 1 1 {m[2]} {m[0]} {m[1]} {m[2]} {m[0]} {m[1]} {g(_deg(nat[1]))} {g(cf[2])}")
        r.append(f"hb-angl {k + 1} 2 1 1 {m[0]} {m[1]} {m[3]} {m[0]} {m[1]} {m[3]} {g(_deg(nat[2]))} {g(cf[3])}")
        r.append(f"hb-dihd {k + 1} 1 1 1 {m[2]} {m[0]} {m[1]} {m[3]} {m[2]} {m[0]} {m[1]} {m[3]} "
                 f"{g(_deg(nat[3]))} {g(cf[4])}")
        r.append(f"hb-dihd {k + 1} 2 1 1 {m[4]} {m[2]} {m[0]} {m[1]} {m[4]} {m[2]} {m[0]} {m[1]} "
                 f"{g(_deg(nat[4]))} {g(cf[5])}")
        r.append(f"hb-dihd {k + 1} 3 1 1 {m[0]} {m[1]} {m[3]} {m[5]} {m[0]} {m[1]} {m[3]} {m[5]} "
                 f"{g(_deg(nat[5]))} {g(cf[6])}")
    for k in range(int(sysd.get("ntst", 0))):
        m = [int(x) for x in sysd["idtrna_tst2mp"][k]]
        nat, cf = sysd["dtrna_tst_nat"][k], sysd["coef_dtrna_tst"][k]
        t = [(1 if sysd["flg_tst_exclusive"][k][q] == 0 else 2) * (-1 if sysd["idtrna_tst2side"][k][q] == 1 else 1)
             for q in range(2)]
        r.append(f"tbs-dist {k + 1} 1 1 {m[0]} {m[1]} {m[0]} {m[1]} {g(cf[0])} {g(nat[0])} {g(cf[1])} "
                 f"{t[0]:+d} {t[1]:+d}")
        r.append(f"tbs-angl {k + 1} 1 1 1 {m[2]} {m[0]} {m[1]} {m[2]} {m[0]} {m[1]} {g(_deg(nat[1]))} {g(cf[2])}")
        r.append(f"tbs-angl {k + 1} 2 1 1 {m[0]} {m[1]} {m[3]} {m[0]} {m[1]} {m[3]} {g(_deg(nat[2]))} {g(cf[3])}")
        r.append(f"tbs-dihd {k + 1} 1 1 1 {m[2]} {m[0]} {m[1]} {m[3]} {m[2]} {m[0]} {m[1]} {m[3]} "
                 f"{g(_deg(nat[3]))} {g(cf[4])}")
        r.append(f"tbs-dihd {k + 1} 2 1 1 {m[4]} {m[2]} {m[0]} {m[1]} {m[4]} {m[2]} {m[0]} {m[1]} "
                 f"{g(_deg(nat[4]))} {g(cf[5])}")
        r.append(f"tbs-dihd {k + 1} 3 1 1 {m[0]} {m[1]} {m[3]} {m[5]} {m[0]} {m[1]} {m[3]} {m[5]} "
                 f"{g(_deg(nat[5]))} {g(cf[6])}")
    return "\n".join(r) + "\n"


# atom names by (bead atom field, local site) for the writer: the inverse of
# site_local on the atoms each bead carries (setp_dtrna15.F90:114-161)
_SITE_ATOMS = {" S  ": ("O2'", "O4'", "O3'", "O5'"), " P  ": ("OP1", "OP2"),
               " Ab ": ("N1", "N3", "N6", "N7"), " Cb ": ("O2", "N3", "N4"),
               " Gb ": ("N1", "N2", "N3", "O6", "N7"), " Ub ": ("O2", "N3", "O4")}


def _site_atom(st: Structure, tab, bead: int, site: int) -> str:
    lo, hi = tab[bead - 1]
    if not (lo <= site <= hi):
        raise NinfoError(f"site {site} is not on bead {bead}")
    return _SITE_ATOMS[st.cmp2atom[bead - 1]][site - lo]

"""Seeded synthetic DT15 systems with the reference's parameter values.

There is no network and no structure files, so every system here is built
from a seeded random walk and the DT15 force-field tables of the reference:

* bonds / angles: natural values and force constants of the DT15 native-info
  convention (ninfo/dtrna15.ninfo "bond"/"angl" records: SP 3.8157 k=64,
  PS 4.6010 k=23, SB per base k=10; PSP/SPS k=20, PSB/BSP k=5),
* stacks: bs-dist coef 1.4, bs-dihd coef 4.0 with the PSPS/SPSP natural
  dihedrals -148.22/175.98 deg and h, s, Tm of para/rna.para:379-400
  (DT15_stack_param),
* hydrogen bonds: hb-dist coef 5.0, hb-angl 1.5, hb-dihd 0.15,
  U0 = -2.93168175 per hydrogen bond (para/rna.para:366-372),
* masses (para/general.para:76-87), excluded-volume radius and epsilon
  (para/rna.para:402-416, DT15_exv_param; exv_epsilon_mp = sqrt(eps),
  src/setp_dtrna15.F90:98-160), hbond sites and valences
  (src/setp_dtrna15.F90:46-161, src/read_nativeinfo.F90:1286-1336).

Bead order of a linear-S chain of n nucleotides (1-based): nt 1 = S1 B1,
nt k >= 2 = P_k S_k B_k, so N = 3n - 1, P_k = 3k-3, S_k = 3k-2, B_k = 3k-1.

Every array is record-major (nrec, k) = the Fortran (k, nrec) layout with
1-based bead numbers, ready for ``tis_b200.abi.make_topology``.
"""
from __future__ import annotations

import math

import numpy as np

from .abi import (CLASS_ION, CLASS_LIG, CLASS_RNA, MP_ION_CA2, MP_ION_CL, MP_ION_K, MP_ION_MG,
                  MP_ION_NA, MP_RNA_BASE, MP_RNA_PHOS, MP_RNA_SUGAR)

DEG = math.pi / 180.0

# para/general.para:76-87
MASS = {"P": 62.972561, "S": 131.10668, "A": 134.11876, "G": 150.11816, "C": 110.09406,
        "U": 111.07882, "Mg": 24.3050, "Cl": 35.4500, "K": 39.1000, "Na": 22.9900, "Ca": 40.078}
# para/rna.para:402-416 (radius, epsilon)
EXV = {"P": (2.1, 0.2), "S": (2.9, 0.2), "A": (2.8, 0.2), "G": (3.0, 0.2), "C": (2.7, 0.2),
       "U": (2.7, 0.2), "Mg": (0.7926, 0.894700), "Ca": (1.7131, 0.459789),
       "Cl": (1.9480, 0.265000), "K": (2.6580, 0.000328), "Na": (1.8680, 0.002770)}
# para/rna.para:379-400 (DT15_stack_param): h, s, Tm
STACK_HST = {
    "AA": (3.99578, -0.319, 299.058), "AC": (3.96314, -0.319, 299.058),
    "AG": (4.75714, 5.301, 341.349), "AU": (3.96314, -0.319, 299.058),
    "CA": (3.92173, -0.319, 299.058), "CC": (3.65726, -1.567, 285.968),
    "CG": (4.23498, 0.774, 315.673), "CU": (3.62896, -1.567, 285.968),
    "GA": (4.71668, 5.301, 341.349), "GC": (4.71997, 4.370, 343.363),
    "GG": (5.19674, 7.346, 366.523), "GU": (4.61901, 2.924, 338.329),
    "UA": (3.92173, -0.319, 299.058), "UC": (3.62234, -1.567, 285.968),
    "UG": (4.67613, 2.924, 338.329), "UU": (2.99569, -3.563, 251.733),
}
# natural SB bond lengths and PSB / BSP angles by base (ninfo/dtrna15.ninfo)
SB_NAT = {"A": 4.8515, "G": 4.9659, "C": 4.2738, "U": 4.2733}
PSB_NAT = {"A": 97.5690, "G": 101.3562, "C": 90.5445, "U": 90.1549}
BSP_NAT = {"A": 110.3459, "G": 109.7214, "C": 112.6149, "U": 112.6607}
# A-form stacking distances by dinucleotide class (purine/pyrimidine); synthetic
STACK_DIST = {"RR": 4.25, "RY": 4.00, "YR": 4.60, "YY": 4.35}
# hbond sites per bead type (src/setp_dtrna15.F90:52-76) and valences (:116-160)
NSITE = {"S": 4, "P": 2, "A": 4, "C": 3, "G": 5, "U": 3}
VALENCE = {"S": [2, 1, 1, 1], "P": [1, 1], "A": [1, 1, 2, 1], "C": [2, 1, 2],
           "G": [1, 2, 1, 2, 1], "U": [2, 1, 1]}
COMPLEMENT = {"A": "U", "U": "A", "G": "C", "C": "G"}
# Watson-Crick / wobble hydrogen-bond atom pairs (base i atom, base j atom)
HB_ATOMS = {
    ("G", "C"): [("N1", "N3"), ("N2", "O2"), ("O6", "N4")],
    ("A", "U"): [("N1", "N3"), ("N6", "O4")],
    ("G", "U"): [("N1", "O2"), ("O6", "N3")],
}
HB_U0_PER_BOND = -2.93168175
ION_TYPE = {"Mg": MP_ION_MG, "Ca": MP_ION_CA2, "Na": MP_ION_NA, "K": MP_ION_K, "Cl": MP_ION_CL}
ION_CHARGE = {"Mg": 2.0, "Ca": 2.0, "Na": 1.0, "K": 1.0, "Cl": -1.0}


def site_local(res: str, atom: str) -> int:
    """src/read_nativeinfo.F90:1286-1336 (the base atoms used here)."""
    if atom == "N1" or atom == "O2":
        return 1
    if atom == "N2":
        return 2
    if atom == "N3":
        return 3 if res == "G" else 2
    if atom in ("O4", "N4", "N6"):
        return 3
    if atom == "O6":
        return 4
    if atom == "N7":
        return 4 if res == "A" else 5
    raise ValueError(atom)


def _bead_index(k: int, kind: str) -> int:
    """1-based bead number of P/S/B of nucleotide k (1-based)."""
    if kind == "S":
        return 1 if k == 1 else 3 * k - 2
    if kind == "B":
        return 2 if k == 1 else 3 * k - 1
    if kind == "P":
        assert k >= 2
        return 3 * k - 3
    raise ValueError(kind)


def random_sequence(n: int, rng) -> str:
    return "".join(rng.choice(list("ACGU"), size=n))


def _walk(kinds, parents, lengths, rng, min_dist=3.2, tries=200, persist=0.55, confine=None):
    """Self-avoiding random walk: bead b is placed at parent(b) + length*u with
    a random direction u biased towards the previous backbone direction, and
    resampled until it is >= min_dist from every earlier bead (the best of
    `tries` draws is kept otherwise).  confine=R keeps beads inside a sphere
    of radius R (dense test systems)."""
    n = len(kinds)
    X = np.zeros((n, 3))
    last_dir = rng.normal(size=3)
    last_dir /= np.linalg.norm(last_dir)
    for b in range(1, n):
        p = parents[b]
        best, best_d = None, -1.0
        for _ in range(tries):
            u = rng.normal(size=3)
            u /= np.linalg.norm(u)
            if kinds[b] != "B":
                u = u + persist * last_dir
                u /= np.linalg.norm(u)
            cand = X[p] + lengths[b] * u
            if confine is not None and np.linalg.norm(cand) > confine:
                continue
            if b > 1:
                d = np.sqrt(((X[:b] - cand) ** 2).sum(axis=1))
                d[p] = np.inf
                dm = d.min()
            else:
                dm = np.inf
            if dm > best_d:
                best, best_d = cand, dm
                if dm >= min_dist:
                    break
        if best is None:   # confinement rejected every draw: step inwards
            u = -X[p] / max(np.linalg.norm(X[p]), 1e-9)
            best = X[p] + lengths[b] * u
        X[b] = best
        if kinds[b] != "B":
            dv = X[b] - X[p]
            last_dir = dv / np.linalg.norm(dv)
    return X


def dt15_chain(n: int, seed: int, seq: str | None = None, hb_pairs=None,
               stem: int | None = None, hb_fraction: float | None = None,
               jitter: float = 0.1, min_dist: float = 3.2, confine: float | None = None):
    """One linear-S DT15 chain of n nucleotides with a seeded random-walk start.

    hb_pairs: explicit list of (i, j) nucleotide pairs (1-based, i < j);
    stem: pair nt i with nt (n+1-i) for i = 1..stem;
    hb_fraction: pair that fraction of residues at random (|i-j| >= 4).
    Paired bases are made complementary (the base of j follows the base of i).
    """
    rng = np.random.default_rng(seed)
    seq = list(seq) if seq is not None else list(random_sequence(n, rng))
    assert len(seq) == n
    pairs = list(hb_pairs or [])
    if stem:
        pairs += [(i, n + 1 - i) for i in range(1, stem + 1)]
    if hb_fraction:
        k = int(round(hb_fraction * n / 2.0))
        free = list(range(1, n + 1))
        rng.shuffle(free)
        used = set(i for p in pairs for i in p)
        for i in free:
            if len(pairs) >= k + (stem or 0) + len(hb_pairs or []):
                break
            if i in used:
                continue
            cands = [j for j in free if j not in used and j != i and abs(j - i) >= 4]
            if not cands:
                continue
            j = cands[int(rng.integers(len(cands)))]
            a, b = (i, j) if i < j else (j, i)
            pairs.append((a, b))
            used.update((a, b))
    for i, j in pairs:
        seq[j - 1] = COMPLEMENT[seq[i - 1]] if (seq[i - 1], seq[j - 1]) not in (("G", "U"), ("U", "G")) else seq[j - 1]

    N = 3 * n - 1
    kinds = [""] * N
    res = [""] * N
    for k in range(1, n + 1):
        kinds[_bead_index(k, "S") - 1] = "S"
        kinds[_bead_index(k, "B") - 1] = "B"
        res[_bead_index(k, "S") - 1] = seq[k - 1]
        res[_bead_index(k, "B") - 1] = seq[k - 1]
        if k >= 2:
            kinds[_bead_index(k, "P") - 1] = "P"
            res[_bead_index(k, "P") - 1] = seq[k - 1]
    # walk: S1 root; B_k from S_k; P_{k+1} from S_k; S_k from P_k
    parents = [0] * N
    lengths = np.zeros(N)
    for k in range(1, n + 1):
        s, b = _bead_index(k, "S") - 1, _bead_index(k, "B") - 1
        parents[b], lengths[b] = s, 4.7 + rng.uniform(-jitter, jitter)
        if k >= 2:
            p = _bead_index(k, "P") - 1
            parents[p], lengths[p] = _bead_index(k - 1, "S") - 1, 3.8 + rng.uniform(-jitter, jitter)
            parents[s], lengths[s] = p, 3.9 + rng.uniform(-jitter, jitter)
    order = sorted(range(N))  # parents always precede children in bead order
    assert all(parents[b] < b for b in order[1:])
    X = _walk(kinds, parents, lengths, rng, min_dist=min_dist, confine=confine)

    typ = {"P": MP_RNA_PHOS, "S": MP_RNA_SUGAR, "B": MP_RNA_BASE}
    imp2type = np.array([typ[k] for k in kinds], dtype=np.int32)
    mkey = [("P" if k == "P" else "S" if k == "S" else r) for k, r in zip(kinds, res)]
    cmass = np.array([MASS[m] for m in mkey])
    exv_radius = np.array([EXV[m][0] for m in mkey])
    exv_epsilon = np.sqrt(np.array([EXV[m][1] for m in mkey]))

    bonds, bnat, bk = [], [], []
    for k in range(1, n + 1):  # SB
        bonds.append((_bead_index(k, "S"), _bead_index(k, "B"))); bnat.append(SB_NAT[seq[k - 1]]); bk.append(10.0)
    for k in range(1, n):      # SP
        bonds.append((_bead_index(k, "S"), _bead_index(k + 1, "P"))); bnat.append(3.8157); bk.append(64.0)
    for k in range(2, n + 1):  # PS
        bonds.append((_bead_index(k, "P"), _bead_index(k, "S"))); bnat.append(4.6010); bk.append(23.0)

    angs, anat, ak = [], [], []
    for k in range(1, n):      # BSP
        angs.append((_bead_index(k, "B"), _bead_index(k, "S"), _bead_index(k + 1, "P")))
        anat.append(BSP_NAT[seq[k - 1]] * DEG); ak.append(5.0)
    for k in range(2, n + 1):  # PSB
        angs.append((_bead_index(k, "P"), _bead_index(k, "S"), _bead_index(k, "B")))
        anat.append(PSB_NAT[seq[k - 1]] * DEG); ak.append(5.0)
    for k in range(2, n):      # PSP
        angs.append((_bead_index(k, "P"), _bead_index(k, "S"), _bead_index(k + 1, "P")))
        anat.append(82.7351 * DEG); ak.append(20.0)
    for k in range(1, n):      # SPS
        angs.append((_bead_index(k, "S"), _bead_index(k + 1, "P"), _bead_index(k + 1, "S")))
        anat.append(87.4104 * DEG); ak.append(20.0)

    st, stnat, stk, sths = [], [], [], []
    pur = set("AG")
    for k in range(2, n - 1):  # needs P_k and P_{k+2}
        b1 = _bead_index(k, "B")
        st.append((b1, b1 + 3, b1 - 2, b1 - 1, b1 + 1, b1 + 2, b1 + 4))
        cls = ("R" if seq[k - 1] in pur else "Y") + ("R" if seq[k] in pur else "Y")
        stnat.append((STACK_DIST[cls] + rng.uniform(-0.2, 0.2), -148.22 * DEG, 175.98 * DEG))
        stk.append((1.4, 4.0, 4.0))
        sths.append(STACK_HST[seq[k - 1] + seq[k]])

    # hbond sites (setp_dtrna15.F90:46-80)
    imp2hbsite = np.zeros(N, dtype=np.int64)
    off = 0
    nval = []
    for b in range(N):
        key = "P" if kinds[b] == "P" else "S" if kinds[b] == "S" else res[b]
        imp2hbsite[b] = off + 1
        off += NSITE[key]
        nval += VALENCE[key]
    hb, hbnat, hbcoef, hbsite = [], [], [], []
    for i, j in pairs:
        assert 1 <= i < j <= n and i < n and j >= 2
        bi, bj = _bead_index(i, "B"), _bead_index(j, "B")
        six = bj + 1 if j < n else bj - 2
        hb.append((bi, bj, bi - 1, bj - 1, bi + 1, six))
        key = (seq[i - 1], seq[j - 1])
        flip = False
        if key not in HB_ATOMS:
            key, flip = (key[1], key[0]), True
        atoms = HB_ATOMS[key]
        nhb_atoms = len(atoms)
        g = rng.uniform(-1.0, 1.0, size=6)
        hbnat.append((5.66 + 0.26 * (nhb_atoms == 2) + 0.05 * g[0], (142.31 + 2 * g[1]) * DEG,
                      (161.75 + 2 * g[2]) * DEG, (79.65 + 5 * g[3]) * DEG, (69.75 + 5 * g[4]) * DEG,
                      (43.65 + 5 * g[5]) * DEG))
        hbcoef.append((HB_U0_PER_BOND * nhb_atoms, 5.0, 1.5, 1.5, 0.15, 0.15, 0.15))
        s = np.zeros((2, 3), dtype=np.int32)  # (side, slot) -> Fortran (3, 2)
        for a, (ai, aj) in enumerate(atoms):
            if flip:
                ai, aj = aj, ai
            s[0, a] = imp2hbsite[bi - 1] - 1 + site_local(seq[i - 1], ai)
            s[1, a] = imp2hbsite[bj - 1] - 1 + site_local(seq[j - 1], aj)
        hbsite.append(s)

    charges = [b + 1 for b in range(N) if kinds[b] == "P"]
    sysd = dict(
        nmp=N, nunit=1, lunit2mp=np.array([[1, N]], dtype=np.int32),
        iclass_unit=np.array([CLASS_RNA], dtype=np.int32), imp2type=imp2type,
        cmass=cmass, fric=np.zeros(N), exv_radius=exv_radius, exv_epsilon=exv_epsilon,
        ncharge=len(charges), icharge2mp=np.array(charges, dtype=np.int32),
        coef_charge=-np.ones(len(charges)),
        nbd=len(bonds), ibd2mp=np.array(bonds, dtype=np.int32).reshape(-1, 2),
        bd_nat=np.array(bnat), coef_bd=np.array(bk),
        nba=len(angs), iba2mp=np.array(angs, dtype=np.int32).reshape(-1, 3),
        ba_nat=np.array(anat), coef_ba=np.array(ak),
        nst=len(st), idtrna_st2mp=np.array(st, dtype=np.int32).reshape(-1, 7),
        dtrna_st_nat=np.array(stnat).reshape(-1, 3), coef_dtrna_st=np.array(stk).reshape(-1, 3),
        dtrna_st_hsTm=np.array(sths).reshape(-1, 3),
        nhb=len(hb), idtrna_hb2mp=np.array(hb, dtype=np.int32).reshape(-1, 6),
        dtrna_hb_nat=np.array(hbnat).reshape(-1, 6), coef_dtrna_hb=np.array(hbcoef).reshape(-1, 7),
        idtrna_hb2hbsite=np.array(hbsite, dtype=np.int32).reshape(-1, 6),
        nhbsite=off, nvalence_hbsite=np.array(nval, dtype=np.int32),
        xyz=X, seq="".join(seq), pairs=pairs,
    )
    return sysd


def set_friction(sysd: dict, fric_const: float):
    """i_fric = 0: fric_mp = fric_const for every bead (setp_mass_fric.F90:44)."""
    sysd["fric"] = np.full(sysd["nmp"], float(fric_const))
    return sysd


def add_ions(sysd: dict, box: float, counts: dict, seed: int, clash: float = 10.0):
    """Appends one ION unit with the given counts, placed uniformly in the box
    centred at the origin with clash rejection (src/simu_initial_ion.F90:21-40)."""
    rng = np.random.default_rng(seed)
    X = sysd["xyz"]
    N0 = sysd["nmp"]
    placed = []
    allpos = [p for p in X]
    names = []
    for name in ("Mg", "Ca", "K", "Na", "Cl"):
        names += [name] * int(counts.get(name, 0))
    grid = {}
    cell = clash

    def key(p):
        return tuple(np.floor(p / cell).astype(int))

    for p in allpos:
        grid.setdefault(key(p), []).append(p)
    for name in names:
        for _ in range(100000):
            cand = rng.uniform(-box / 2, box / 2, size=3)
            k = key(cand)
            ok = True
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        for q in grid.get((k[0] + dx, k[1] + dy, k[2] + dz), ()):
                            if np.sum((q - cand) ** 2) < clash * clash:
                                ok = False
                                break
                        if not ok:
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                break
        else:
            raise RuntimeError("ion placement failed")
        grid.setdefault(k, []).append(cand)
        placed.append(cand)
    nI = len(names)
    N = N0 + nI
    sysd = dict(sysd)
    sysd["xyz"] = np.vstack([X, np.array(placed).reshape(-1, 3)])
    sysd["nmp"] = N
    sysd["nunit"] = 2
    sysd["lunit2mp"] = np.array([[1, N0], [N0 + 1, N]], dtype=np.int32)
    sysd["iclass_unit"] = np.array([CLASS_RNA, CLASS_ION], dtype=np.int32)
    sysd["imp2type"] = np.concatenate([sysd["imp2type"], np.array([ION_TYPE[n] for n in names], dtype=np.int32)])
    sysd["cmass"] = np.concatenate([sysd["cmass"], [MASS[n] for n in names]])
    sysd["fric"] = np.concatenate([sysd["fric"], np.full(nI, sysd["fric"][0] if N0 else 0.0)])
    sysd["exv_radius"] = np.concatenate([sysd["exv_radius"], [EXV[n][0] for n in names]])
    sysd["exv_epsilon"] = np.concatenate([sysd["exv_epsilon"], np.sqrt([EXV[n][1] for n in names])])
    sysd["icharge2mp"] = np.concatenate([sysd["icharge2mp"], np.arange(N0 + 1, N + 1, dtype=np.int32)]).astype(np.int32)
    sysd["coef_charge"] = np.concatenate([sysd["coef_charge"], [ION_CHARGE[n] for n in names]])
    sysd["ncharge"] = len(sysd["icharge2mp"])
    sysd["ion_names"] = names
    return sysd


# ------------------------------------------------------------- parameters
def dt15_params(**over):
    """tis_params defaults: para/rna.para:325-370 (DT15), general.para
    (neigh_margin 8.0), the electrostatic defaults and the configuration
    of the workload (set by the caller)."""
    p = dict(i_periodic=0, psize=(0.0, 0.0, 0.0), neigh_margin=8.0, n_step_neighbor=10,
             exv_dist=3.2, exv_dist_PS=3.2, exv_adjust=1.5852, exv_inf=0.2,
             n_sep_nlocal_P=3, n_sep_nlocal_S=3, n_sep_nlocal_B=2, hb_cutoff_dist=2.0,
             i_ele=1, i_diele=1, diele_water=78.0, ionic_strength=0.15, cutoff_ele=20.0,
             i_DH_cutoff_type=0, ewld_alpha=0.05, ewld_hmax=10.0,
             i_simulate_type=1, tstep=0.05, viscosity=0.0, wca_coef_cutoff=1.0,
             precision=0, hb_beta_global=1, seed=12345, hi_radius=2.0, n_step_hydro=1)
    p.update(over)
    return p


# ------------------------------------------------------------- workloads
def workload_c1(seed: int = 1):
    """Plain FP64 single system: 22-nt chain (65 beads), 6-bp stem (nt i with
    nt 23-i), DH 150 mM, 300 K, dt 0.05, friction 0.5, rebuild every 10."""
    s = set_friction(dt15_chain(22, seed, stem=6), 0.5)
    par = dt15_params(ionic_strength=0.150, precision=0)
    return [s], par, [300.0]


def workload_c2(seed: int = 2):
    """Explicit ions + Ewald: 51-nt chain in a 150 A periodic cube, Mg 5 mM,
    K 150 mM, Cl to neutrality, alpha 0.05, r_c 20, |h| <= 10, 300 K."""
    box = 150.0
    s = set_friction(dt15_chain(51, seed, stem=8), 0.5)
    vol_l = box ** 3 * 1e-27
    n_mg = int(round(0.005 * vol_l * 6.022140857e23))
    n_k = int(round(0.150 * vol_l * 6.022140857e23))
    n_cl = int(2 * n_mg + n_k - s["ncharge"])
    s = add_ions(s, box, {"Mg": n_mg, "K": n_k, "Cl": n_cl}, seed + 100)
    par = dt15_params(i_periodic=1, psize=(box, box, box), i_ele=2, cutoff_ele=20.0,
                      ewld_alpha=0.05, ewld_hmax=10.0, ionic_strength=0.150 + 3 * 0.005, precision=1)
    return [s], par, [300.0]


def bead_chain(n: int, seed: int, bond: float = 3.8, sigma: float = 4.0, min_dist: float = 4.2,
               k_fene: float = 20.0, r2_fene: float = 2.0, eps_wca: float = 1.0, mass: float = 100.0):
    """Brownian-HI bead chain: one LIG-class unit of n beads (no DT15 terms:
    zero excluded-volume radius), FENE bonds between consecutive beads
    (fene_nat = bond, coef_fene = k_fene, dist2_fene = r2_fene, the column
    meaning of read_nativeinfo.F90:153-176) and a WCA record for every
    non-bonded pair j >= i + 2 (wca_nat = sigma, coef_wca = (eps, eps):
    read_nativeinfo.F90:306-332).  Coordinates: seeded self-avoiding walk."""
    rng = np.random.default_rng(seed)
    kinds = ["S"] * n
    parents = [0] + list(range(n - 1))
    lengths = [0.0] + list(bond + rng.uniform(-0.05, 0.05, n - 1))
    X = _walk(kinds, parents, lengths, rng, min_dist=min_dist, persist=0.3)
    X = X - X.mean(axis=0)
    ii, jj = np.triu_indices(n, k=2)
    nw = len(ii)
    return dict(
        nmp=n, nunit=1, lunit2mp=np.array([[1, n]], dtype=np.int32),
        iclass_unit=np.array([CLASS_LIG], dtype=np.int32),
        imp2type=np.full(n, MP_RNA_SUGAR, dtype=np.int32),
        cmass=np.full(n, mass), fric=np.full(n, 0.5),
        exv_radius=np.zeros(n), exv_epsilon=np.zeros(n),
        ncharge=0, icharge2mp=np.zeros(0, dtype=np.int32), coef_charge=np.zeros(0),
        nbd=0, nba=0, nst=0, nhb=0, nhbsite=0,
        nfene=n - 1,
        ifene2mp=np.stack([np.arange(1, n), np.arange(2, n + 1)], axis=1).astype(np.int32),
        fene_nat=np.full(n - 1, bond), coef_fene=np.full(n - 1, k_fene), dist2_fene=np.full(n - 1, r2_fene),
        nwca=nw,
        iwca2mp=np.stack([ii + 1, jj + 1], axis=1).astype(np.int32),
        wca_nat=np.full(nw, sigma),
        coef_wca=np.stack([np.full(nw, eps_wca), np.full(nw, eps_wca)], axis=0),
        xyz=X,
    )


def bdhi_params(**over):
    """Brownian dynamics with hydrodynamic interactions (i_simulate_type 6,
    HI_TENSOR%RPY): water viscosity 1e-3 Pa s in the internal units of
    setp_mass_fric.F90:67 (x sqrt(1e3 JOUL2KCAL) N_AVO 1e-20 = 2.944), RPY
    radius 2 A, dt 0.01, no electrostatics, WCA cut at sigma."""
    visc = 1.0e-3 * np.sqrt(1.0e3 / 4184.0) * 6.022140857e23 * 1.0e-20
    p = dt15_params(i_simulate_type=6, i_ele=0, tstep=0.01, viscosity=visc, hi_radius=2.0,
                    n_step_hydro=1, wca_coef_cutoff=1.0, n_step_neighbor=10)
    p.update(over)
    return p


def workload_c5(seed: int = 5, nchain: int = 32):
    """Brownian-HI batch: nchain bead chains, N uniform in 100..1000, FENE
    bonds, WCA between all non-bonded pairs, RPY radius 2 A, dt 0.01, D and
    its Cholesky factor refreshed every 10 steps, 300 K; mixed precision
    (tensor-core trailing updates, FP32 D and L in the step)."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(100, 1001, size=nchain)
    systems = [bead_chain(int(n), seed * 1000 + k) for k, n in enumerate(ns)]
    return systems, bdhi_params(n_step_hydro=10, precision=1), [300.0] * nchain


def temperature_ladder(n=64, tlo=280.0, thi=400.0):
    return [tlo * (thi / tlo) ** (k / (n - 1)) for k in range(n)]


def workload_c3(seed: int = 3, nrep: int = 64):
    """64-replica temperature REMD of one 76-nt chain (227 beads), 20 random
    stem hbond pairs, DH 100 mM, ladder 280-400 K, exchange every 1000 steps."""
    rng = np.random.default_rng(seed)
    n = 76
    pairs = []
    used = set()
    while len(pairs) < 20:
        i, j = sorted(int(x) for x in rng.integers(1, n + 1, size=2))
        if j - i < 4 or i in used or j in used:
            continue
        pairs.append((i, j)); used.update((i, j))
    s = set_friction(dt15_chain(n, seed, hb_pairs=sorted(pairs)), 0.5)
    par = dt15_params(ionic_strength=0.100, precision=1)
    return [s], par, temperature_ladder(nrep)


def workload_c4(seed: int = 4, nchain: int = 256):
    """256 independent chains, n ~ exp(U(ln 20, ln 400)), 30% of residues in
    random hbond pairs, DH 150 mM, 300 K."""
    rng = np.random.default_rng(seed)
    lens = np.exp(rng.uniform(np.log(20), np.log(400), size=nchain)).round().astype(int)
    systems = [set_friction(dt15_chain(int(n), seed * 1000 + k, hb_fraction=0.3), 0.5)
               for k, n in enumerate(lens)]
    par = dt15_params(ionic_strength=0.150, precision=1)
    return systems, par, [300.0] * nchain


# ------------------------------------------------------------- test geometry
def hairpin_coords(sysd: dict, stem: int, seed: int = 0, D: float = 15.2, dx: float = 6.5, zjit: float = 0.6):
    """Replaces the coordinates of a chain built with ``stem`` by a hairpin
    ladder: nt k and nt n+1-k face each other with their bases ~5.8 A apart
    (inside the 2 A window of every stem hydrogen bond); the loop runs on a
    half ellipse.  Random z jitter avoids planar (degenerate) dihedrals."""
    rng = np.random.default_rng(seed)
    n = (sysd["nmp"] + 1) // 3
    X = np.zeros((sysd["nmp"], 3))

    def put(k, sx, sy, bdir):
        s_ = _bead_index(k, "S") - 1
        b_ = _bead_index(k, "B") - 1
        X[s_] = (sx, sy, 0.0)
        X[b_] = (sx + 0.3 * bdir[0] * 0, sy + 4.7 * bdir[1], 0.0) if bdir[0] == 0 else (sx + 4.7 * bdir[0], sy + 4.7 * bdir[1], 0.0)
        if k >= 2:
            X[_bead_index(k, "P") - 1] = (0, 0, 0)

    m = stem
    L = n - 2 * m
    # stem strands
    S = {}
    for k in range(1, m + 1):
        S[k] = (dx * (k - 1), 0.0, (0.0, 1.0))
        S[n + 1 - k] = (dx * (k - 1), D, (0.0, -1.0))
    # loop on a half ellipse from (x_m + dx, 0) to (x_m + dx, D)
    x0 = dx * m
    a = max(2.0 * dx * (L + 1) / np.pi - D / 2.0, dx)
    for q, k in enumerate(range(m + 1, n - m + 1)):
        th = np.pi * (q + 1) / (L + 1)
        sx, sy = x0 + a * np.sin(th), D / 2.0 - (D / 2.0) * np.cos(th)
        cx, cy = x0, D / 2.0
        v = np.array([sx - cx, sy - cy])   # loop bases point outwards
        v /= np.linalg.norm(v)
        S[k] = (sx, sy, (v[0], v[1]))
    for k in range(1, n + 1):
        sx, sy, bd = S[k]
        X[_bead_index(k, "S") - 1] = (sx, sy, 0.0)
        X[_bead_index(k, "B") - 1] = (sx + 4.7 * bd[0], sy + 4.7 * bd[1], 0.0)
    for k in range(2, n + 1):   # P_k between S_{k-1} and S_k, pushed outwards
        a_ = X[_bead_index(k - 1, "S") - 1]
        b_ = X[_bead_index(k, "S") - 1]
        mid = 0.5 * (a_ + b_)
        out = np.array([0.0, 0.0, 1.5])
        X[_bead_index(k, "P") - 1] = mid + out
    X[:, 2] += rng.uniform(-zjit, zjit, size=sysd["nmp"])
    X[:, :2] += rng.uniform(-0.15, 0.15, size=(sysd["nmp"], 2))
    sysd = dict(sysd)
    sysd["xyz"] = X
    return sysd


def _tst_geometry(x, m):
    """Distance, 2 angles and 3 dihedrals of one tertiary stack (beads m,
    0-based B1 B2 S1 S2 P1' P2') as energy_dtrna_stack_nlocal.F90 defines them."""
    v12, v13, v53, v42, v46 = x[m[0]] - x[m[1]], x[m[0]] - x[m[2]], x[m[4]] - x[m[2]], x[m[3]] - x[m[1]], x[m[3]] - x[m[5]]
    a12, a13, a42 = (np.linalg.norm(v) for v in (v12, v13, v42))
    t1 = np.arccos(np.dot(v13, v12) / (a13 * a12))
    t2 = np.arccos(np.dot(v12, v42) / (a12 * a42))
    c4212, c1213 = np.cross(v42, v12), np.cross(v12, v13)
    p0 = np.arctan2(np.dot(v42, c1213) * a12, np.dot(c4212, c1213))
    n1 = -c1213
    p1 = np.arctan2(np.dot(v53, n1) * a13, np.dot(np.cross(v53, v13), n1))
    m2, n2 = -c4212, np.cross(v42, v46)
    p2 = np.arctan2(np.dot(v12, n2) * a42, np.dot(m2, n2))
    return np.array([a12, t1, t2, p0, p1, p2])


def add_tertiary_stacks(sysd: dict, pairs, sides, exclusive, seed: int = 0, dist_shift=None,
                        u0: float = -5.0, coef=(5.0, 1.5, 1.5, 0.15, 0.15, 0.15)):
    """Appends tertiary stacks (tbs-dist/-angl/-dihd records) between the
    bases of nucleotides (i, j) of a dt15_chain: beads B_i, B_j, S_i, S_j,
    P_{i+1}, P_{j+1} (read_nativeinfo.F90:666-671).  Natural values are the
    current geometry plus small seeded offsets; dist_shift[k], when given,
    is added to record k's natural distance (a large negative shift puts the
    stack more than 10 A from native, so it excludes nothing).  sides[k] =
    (side of B_i, side of B_j): 1 = its stack with B - 3, 2 = with B + 3;
    exclusive[k] = (flag, flag)."""
    rng = np.random.default_rng(seed)
    s = dict(sysd)
    x = np.asarray(s["xyz"], dtype=np.float64)
    idx, nat = [], []
    for k, (i, j) in enumerate(pairs):
        bi, bj = _bead_index(i, "B"), _bead_index(j, "B")
        m = (bi, bj, bi - 1, bj - 1, bi + 1, bj + 1)
        g = _tst_geometry(x, [b - 1 for b in m])
        g = g + rng.uniform(-1.0, 1.0, size=6) * np.array([0.2, 0.05, 0.05, 0.1, 0.1, 0.1])
        if dist_shift is not None:
            g[0] += dist_shift[k]
        idx.append(m)
        nat.append(g)
    s["ntst"] = len(pairs)
    s["idtrna_tst2mp"] = np.array(idx, dtype=np.int32).reshape(-1, 6)
    s["dtrna_tst_nat"] = np.array(nat).reshape(-1, 6)
    s["coef_dtrna_tst"] = np.tile(np.array((u0,) + tuple(coef)), (len(pairs), 1))
    s["idtrna_tst2side"] = np.array(sides, dtype=np.int32).reshape(-1, 2)
    s["flg_tst_exclusive"] = np.array(exclusive, dtype=np.int32).reshape(-1, 2)
    return s


def hairpin_tertiary(seed: int = 1):
    """22-nt hairpin with three tertiary stacks across the stem: two within
    10 A of their native distance (their exclusive sides turn secondary
    stacks off), one 15 A short of it (excludes nothing)."""
    s = hairpin_coords(set_friction(dt15_chain(22, seed, stem=6), 0.5), 6, seed=seed)
    return add_tertiary_stacks(s, [(3, 19), (5, 17), (8, 14)], sides=[(2, 1), (1, 2), (2, 2)],
                               exclusive=[(1, 1), (1, 0), (1, 1)], seed=seed + 2, dist_shift=[0.0, 0.0, -15.0])


def duplicate_hbonds(sysd: dict, seed: int = 0, shift: float = 0.3):
    """Appends a second record for every hydrogen bond (same beads and sites,
    shifted natural values), so every hbond site is over its valence and the
    valence pruning (force_dtrna_hbond15.F90:373-509) must act."""
    rng = np.random.default_rng(seed)
    s = dict(sysd)
    nhb = s["nhb"]
    nat = s["dtrna_hb_nat"].copy()
    nat2 = nat + rng.uniform(-shift, shift, size=nat.shape) * np.array([1, 0.1, 0.1, 0.3, 0.3, 0.3])
    s["idtrna_hb2mp"] = np.vstack([s["idtrna_hb2mp"], s["idtrna_hb2mp"]])
    s["dtrna_hb_nat"] = np.vstack([nat, nat2])
    s["coef_dtrna_hb"] = np.vstack([s["coef_dtrna_hb"], s["coef_dtrna_hb"]])
    s["idtrna_hb2hbsite"] = np.vstack([s["idtrna_hb2hbsite"], s["idtrna_hb2hbsite"]])
    s["nhb"] = 2 * nhb
    return s


# ----------------------------------------------------- DT19 semi-explicit
# para/rna.para:495-507 (NHT19_exv_param): radius, epsilon of the DT19 model
NHT19_EXV = {"P": (1.8900, 0.2), "S": (2.6100, 0.2), "A": (2.5200, 0.2), "G": (2.7000, 0.2),
             "C": (2.4300, 0.2), "U": (2.4300, 0.2), "Mg": (2.0000, 0.894700)}


def mg_p_pmf(seed: int = 0, rmin: float = 1.775, rbin: float = 0.025, nbin: int = 1930):
    """A seeded synthetic Mg-P potential of mean force on the grid of the
    reference's RISM table (1.775 A in steps of 0.025 A, 1930 points): a
    steep repulsive wall, contact and solvent-separated wells and a screened
    1/r tail, with seeded depths and positions.  It stands in for the RISM
    table, which is not shipped with this code.  Returns the tis_params
    fields of tis_b200.ninfo.read_pmf."""
    rng = np.random.default_rng(seed)
    r = rmin + rbin * np.arange(nbin)
    w1, w2 = rng.uniform(0.7, 1.1), rng.uniform(0.8, 1.2)
    c1, c2 = rng.uniform(2.6, 3.2), rng.uniform(6.0, 7.0)
    v = (360.0 * np.exp(-(r - rmin) / 0.12) - w1 * np.exp(-((r - c1) / 0.45) ** 2)
         - w2 * np.exp(-((r - c2) / 1.6) ** 2) - 4.7 / r * (1.0 - np.exp(-r / 3.0)))
    return dict(pmf_nbin=nbin, pmf_rmin=rmin, pmf_rbin=rbin, pmf_rmax=float(r[-1]), pmf_mg_p=v)


def dt19_params(**over):
    """tis_params of the DT19 model: para/rna.para:423-470 (para_NHT19_rna:
    n_sep_nlocal P/S 4, exv_inf 0), Manning phosphate charges with
    LENGTH_PER_UNIT P 4.38178046 (para/electrostatic.para:42), pmf_merge 5 A
    and the synthetic Mg-P table of mg_p_pmf."""
    p = dt15_params(n_sep_nlocal_P=4, n_sep_nlocal_S=4, n_sep_nlocal_B=2, exv_inf=0.0,
                    i_dtrna_model=2019, i_charge=1, length_per_unit_P=4.38178046, pmf_rmerge=5.0)
    p.update(mg_p_pmf())
    p.update(over)
    return p


def dt19_mg_system(seed: int = 11, n: int = 16, stem: int = 4, box: float = 80.0, n_near: int = 5, n_far: int = 3):
    """A DT19 chain in a periodic box with Mg ions: n_near of them 2.4-5.5 A
    from phosphates (inside the PMF table, some within pmf_merge), one next
    to a phosphate whose charge is fixed at 0 (a CHARGE_CHANGE line: that
    pair keeps its excluded volume), n_far elsewhere.  The chain is a
    self-avoiding walk with 5.2 A between non-bonded beads (the NHT19 radii
    are larger than the DT15 contact distance); radii and epsilons from the
    NHT19 table; phosphate charges are replaced by -Zp of each temperature
    (i_charge = 1)."""
    rng = np.random.default_rng(seed)
    s = set_friction(dt15_chain(n, seed, stem=stem, min_dist=5.2), 0.5)
    kinds = []
    typ = s["imp2type"]
    seq = s["seq"]
    k = 0
    for b in range(s["nmp"]):
        if typ[b] == MP_RNA_PHOS:
            kinds.append("P")
        elif typ[b] == MP_RNA_SUGAR:
            kinds.append("S")
        else:
            kinds.append(seq[k]); k += 1
    s["exv_radius"] = np.array([NHT19_EXV[q][0] for q in kinds])
    s["exv_epsilon"] = np.sqrt(np.array([NHT19_EXV[q][1] for q in kinds]))
    X = s["xyz"] - s["xyz"].mean(axis=0)
    phos = [b for b in range(s["nmp"]) if typ[b] == MP_RNA_PHOS]
    fixed_p = phos[-1]
    picks = list(rng.choice(phos[:-1], size=n_near, replace=False)) + [fixed_p]
    ions = []
    for b in picks:
        for _ in range(1000):
            u = rng.normal(size=3)
            u /= np.linalg.norm(u)
            # the Mg of the uncharged phosphate sits inside their exv contact distance (3.89 A)
            cand = X[b] + (rng.uniform(3.4, 3.8) if b == fixed_p else rng.uniform(2.4, 5.5)) * u
            d_p = np.linalg.norm(X[phos] - cand, axis=1)
            non_p = [q for q in range(len(X)) if typ[q] != MP_RNA_PHOS]
            d_o = np.linalg.norm(np.vstack([X[non_p]] + ([np.array(ions)] if ions else [])) - cand, axis=1)
            if d_p.min() > 2.4 and d_o.min() > 4.7:
                ions.append(cand)
                break
        else:
            raise RuntimeError("Mg placement failed")
    while len(ions) < n_near + 1 + n_far:
        cand = rng.uniform(-box / 2, box / 2, size=3)
        if np.min(np.linalg.norm(np.vstack([X, np.array(ions)]) - cand, axis=1)) > 12.0:
            ions.append(cand)
    nI = len(ions)
    N0 = s["nmp"]
    N = N0 + nI
    s["xyz"] = np.vstack([X, np.array(ions)])
    s["nmp"] = N
    s["nunit"] = 2
    s["lunit2mp"] = np.array([[1, N0], [N0 + 1, N]], dtype=np.int32)
    s["iclass_unit"] = np.array([CLASS_RNA, CLASS_ION], dtype=np.int32)
    s["imp2type"] = np.concatenate([typ, np.full(nI, MP_ION_MG, dtype=np.int32)]).astype(np.int32)
    s["cmass"] = np.concatenate([s["cmass"], np.full(nI, MASS["Mg"])])
    s["fric"] = np.concatenate([s["fric"], np.full(nI, s["fric"][0])])
    s["exv_radius"] = np.concatenate([s["exv_radius"], np.full(nI, NHT19_EXV["Mg"][0])])
    s["exv_epsilon"] = np.concatenate([s["exv_epsilon"], np.full(nI, math.sqrt(NHT19_EXV["Mg"][1]))])
    q_idx = list(s["icharge2mp"]) + list(range(N0 + 1, N + 1))
    q_val = [0.0 if b - 1 == fixed_p else v for b, v in zip(s["icharge2mp"], s["coef_charge"])] + [2.0] * nI
    s["icharge2mp"] = np.array(q_idx, dtype=np.int32)
    s["coef_charge"] = np.array(q_val)
    s["flg_charge_fixed"] = np.array([1 if b - 1 == fixed_p else 0 for b in q_idx], dtype=np.int32)
    s["ncharge"] = len(q_idx)
    return s

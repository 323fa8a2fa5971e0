"""The DT19 semi-explicit ion model and Manning phosphate charges in the
CPU restatement (oracle/), CPU only: the charge of simu_ele_set.F90:107-166,
the Mg-P table of :231-253, the list rules of neighbor_assign.F90:524-537 and
neighbor_list_ele.F90:167-174, F = -grad E for the table and the NHT19
excluded volume, and the PMF file reader of setp_pmf.F90."""
import math
import os

import numpy as np
import pytest

from tis_b200 import ninfo, synth
from tis_b200.abi import MP_ION_MG, MP_RNA_PHOS
from oracle.oracle import Oracle

# the reference source tree (Hori-Lab/TIS), when present: its input files
# are read as test data; the tests that need it skip otherwise
REF = os.environ.get("TIS_REFERENCE_DIR", "")
ELE, EPSI_0, BOLTZ_J, N_AVO = 1.6021766208e-19, 8.854187817e-12, 1.38064852e-23, 6.022140857e23
JOUL2KCAL_MOL = 1.0 / 4184.0 * N_AVO
BOX = 80.0


def dt19(**over):
    return synth.dt19_params(i_periodic=1, psize=(BOX, BOX, BOX), ionic_strength=0.1, **over)


def ek_of(T):
    tc = T - 273.15
    return 87.740 - 0.4008 * tc + 9.398e-4 * tc * tc - 1.410e-6 * tc ** 3


def zp_expected(T, ionic, n_mg, b=4.38178046, dt19_model=True):
    """simu_ele_set.F90:107-151 restated."""
    ek = ek_of(T)
    lb = ELE * ELE / (4.0 * math.pi * EPSI_0 * ek * BOLTZ_J * T) * 1.0e10
    if not (dt19_model and n_mg > 0):
        return b / lb
    xi = lb / b
    conc = n_mg / (N_AVO * 1e-27 * BOX ** 3)
    v1 = 4 * math.pi * b ** 3 * (xi - 1.0) * 2
    v2 = 4 * math.pi * b ** 3 * (xi - 0.5) * 3
    c1, c2 = N_AVO * 1e-27 * ionic * v1, N_AVO * 1e-27 * conc * v2
    theta = (-c1 ** 2 + math.sqrt(c1 ** 4 + 8 * c1 ** 2 * c2 * (1 - 1 / xi))) / (4 * c2)
    return 1.0 - theta


@pytest.fixture(scope="module")
def system():
    return synth.dt19_mg_system()


def test_manning_charge_and_table(oracle_lib, system):
    s = system
    n_mg = int(np.sum(s["imp2type"] == MP_ION_MG))
    par = dt19()
    temps = [290.0, 330.0]
    o = Oracle(s, par, temps)
    for lab, T in enumerate(temps, start=1):
        zp, e, f = o.label_pmf(lab)
        assert zp == pytest.approx(zp_expected(T, 0.1, n_mg), rel=1e-13)
        assert 0.5 < zp < 1.0
        # the table: PMF switched to DH(+2, -Zp) below pmf_merge, finite-difference force
        p = o.label_params(lab)
        r = par["pmf_rmin"] + par["pmf_rbin"] * np.arange(par["pmf_nbin"])
        dh = p["coef"] * 2.0 * (-zp) * np.exp(-r / p["cdist"]) / r
        v = par["pmf_mg_p"]
        e_ref = v + (dh - v) * np.exp(-(par["pmf_rmerge"] ** 2) / (r * r))
        assert np.allclose(e, e_ref, rtol=1e-13, atol=1e-13)
        assert np.allclose(f[:-1], -(e[1:] - e[:-1]) / par["pmf_rbin"], rtol=1e-10, atol=1e-12) and f[-1] == 0.0
    o.close()
    # without Mg, or in the DT15 model, Zp = b / l_B
    s2 = synth.set_friction(synth.dt15_chain(8, 3), 0.5)
    for model in (2015, 2019):
        o = Oracle(s2, dt19(i_dtrna_model=model), [300.0])
        zp, e, _ = o.label_pmf(1)
        assert zp == pytest.approx(zp_expected(300.0, 0.1, 0, dt19_model=False), rel=1e-13) and len(e) == 0
        o.close()


def test_lists(oracle_lib, system):
    s = system
    o = Oracle(s, dt19(), [300.0])
    o.set_state(s["xyz"][None])
    o.neighbor()
    typ = s["imp2type"]
    n_rna = int(s["lunit2mp"][0][1])
    fixed = {int(b) for b, fx in zip(s["icharge2mp"], s["flg_charge_fixed"]) if fx}
    ex = o.exv_list()
    p_ion = [(i, j) for i, j, _ in ex if j > n_rna and typ[i - 1] == MP_RNA_PHOS]
    # neighbor_assign.F90:524-537: only the uncharged phosphate keeps its exv with an ion
    assert p_ion and all(i in fixed for i, _ in p_ion)
    lst, coef = o.ele_list()
    for (i, j, _, ipmf), c in zip(lst, coef):
        pair = {typ[i - 1], typ[j - 1]}
        assert ipmf == (1 if pair == {MP_RNA_PHOS, MP_ION_MG} else 0)
    assert (lst[:, 3] == 1).sum() > 10
    # with the DT15 rules every phosphate-ion pair in range is an exv pair
    o2 = Oracle(s, dt19(i_dtrna_model=2015), [300.0])
    o2.set_state(s["xyz"][None])
    o2.neighbor()
    ex2 = o2.exv_list()
    assert len([1 for i, j, _ in ex2 if j > n_rna and typ[i - 1] == MP_RNA_PHOS]) > len(p_ion)
    assert (o2.ele_list()[0][:, 3] == 0).all()
    o.close(); o2.close()


def fd_term(o, x0, k, h):
    g = np.zeros_like(x0)
    for i in range(x0.shape[0]):
        for d in range(3):
            e = []
            for sgn in (1, -1):
                xp = x0.copy()
                xp[i, d] += sgn * h
                o.set_state(xp[None])
                o.neighbor()
                e.append(o.energy()[k - 1])
            g[i, d] = -(e[0] - e[1]) / (2 * h)
    return g


def test_force_is_minus_energy_gradient(oracle_lib, system):
    """The table energy is linear within a bin, so central differences with
    a step far below the bin width (0.025 A) reproduce the bin force; the
    NHT19 excluded volume (base-base 3.2 A, else the radius sum) likewise."""
    s = system
    o = Oracle(s, dt19(), [300.0])
    x0 = s["xyz"].copy()
    o.set_state(x0[None])
    o.neighbor()
    f_ele, f_exv = o.force_term("dh"), o.force_term("exv")
    o.force()
    assert o.nclamp() == 0 and o.pmf_range() == 0
    g_ele = fd_term(o, x0, 8, 1e-6)
    g_exv = fd_term(o, x0, 18, 1e-5)
    for f, g in ((f_ele, g_ele), (f_exv, g_exv)):
        assert np.abs(f).max() > 0.05
        assert np.abs(f - g).max() <= 1e-5 * max(np.abs(f).max(), 1.0), np.abs(f - g).max()
    o.close()


def test_pair_below_the_table_is_reported(oracle_lib, system):
    """force_ele_DH.F90:90-93 stops when a Mg-P pair is closer than the
    table's first point; the restatement records it."""
    s = dict(system)
    x = s["xyz"].copy()
    n_rna = int(s["lunit2mp"][0][1])
    phos = [b for b in range(n_rna) if s["imp2type"][b] == MP_RNA_PHOS]
    x[n_rna] = x[phos[0]] + np.array([1.5, 0.0, 0.0])
    o = Oracle(s, dt19(), [300.0])
    o.set_state(x[None])
    o.neighbor()
    o.force()
    assert o.pmf_range() == 1
    o.close()


def test_read_pmf_text():
    r = 1.775 + 0.025 * np.arange(5)
    text = "".join(f"{a:.8E} {b}\n" for a, b in zip(r, [363.9, 299.5, 246.3, 202.2, 165.7]))
    d = ninfo.read_pmf(text)
    assert d["pmf_nbin"] == 5 and d["pmf_rmin"] == 1.775 and d["pmf_rmax"] == float(f"{r[-1]:.8E}")
    assert abs(d["pmf_rbin"] - 0.025) < 1e-12 and d["pmf_mg_p"].tolist() == [363.9, 299.5, 246.3, 202.2, 165.7]
    bad = text.replace(f"{r[3]:.8E}", f"{r[3] + 0.001:.8E}")
    with pytest.raises(ninfo.NinfoError, match="not uniform"):
        ninfo.read_pmf(bad)


@pytest.mark.skipif(not REF or not os.path.isdir(REF), reason="TIS_REFERENCE_DIR not set")
def test_read_reference_pmf_file():
    d = ninfo.read_pmf(f"{REF}/para/PMF_RISM/pmf_Mg_P_1264")
    assert d["pmf_nbin"] == 1930 and d["pmf_rmin"] == 1.775 and d["pmf_rmax"] == 50.0
    assert abs(d["pmf_rbin"] - 0.025) < 1e-12 and d["pmf_mg_p"][0] == 363.922


def test_synthetic_table_matches_reference_grid():
    d = synth.mg_p_pmf()
    assert d["pmf_nbin"] == 1930 and d["pmf_rmin"] == 1.775 and abs(d["pmf_rmax"] - 50.0) < 1e-9
    v = d["pmf_mg_p"]
    assert v[0] > 300 and v.min() < -0.5 and abs(v[-1]) < 0.2


@pytest.mark.skipif(not REF or not os.path.isdir(REF), reason="TIS_REFERENCE_DIR not set")
def test_reference_bwyv19_force_check_input(oracle_lib):
    """The reference's DT19 force-check input (inp/bwyv19_force_check.inp:
    bwyv19.ninfo on the RNA and 206-Mg PDBs, the RISM Mg-P table,
    CHARGE_CHANGE 85 0.0, 700 A box, 57 mM, DH cutoff type 1 at 50 A,
    310.15 K) read through tis_b200.ninfo and evaluated by the
    restatement: the table forces are -grad E of the table energies."""
    st = ninfo.read_pdb_cg([f"{REF}/pdb/bwyv19_force_check.rna.pdb", f"{REF}/pdb/bwyv19_force_check.ion.pdb"])
    s = ninfo.build_system(st, ninfo.read_ninfo(f"{REF}/ninfo/bwyv19.ninfo", st), i_fric=1, viscosity=0.000015,
                           charge_change={85: 0.0}, i_dtrna_model=2019)
    par = synth.dt19_params(i_periodic=1, psize=(700.0, 700.0, 700.0), ionic_strength=0.057, i_DH_cutoff_type=1,
                            cutoff_ele=50.0)
    par.update(ninfo.read_pmf(f"{REF}/para/PMF_RISM/pmf_Mg_P_1264"))
    o = Oracle(s, par, [310.15])
    x0 = s["xyz"].copy()
    o.set_state(x0[None])
    o.neighbor()
    e = o.energy()
    f = o.force_term("dh")
    assert np.all(np.isfinite(e)) and o.pmf_range() == 0
    assert (o.ele_list()[0][:, 3] == 1).sum() > 1000
    zp, _, _ = o.label_pmf(1)
    # Zp of 206 Mg in the 700 A box at 57 mM
    ek = ek_of(310.15)
    lb = ELE * ELE / (4.0 * math.pi * EPSI_0 * ek * BOLTZ_J * 310.15) * 1.0e10
    xi, b = lb / 4.38178046, 4.38178046
    conc = 206 / (N_AVO * 1e-27 * 700.0 ** 3)
    c1 = N_AVO * 1e-27 * 0.057 * 4 * math.pi * b ** 3 * (xi - 1.0) * 2
    c2 = N_AVO * 1e-27 * conc * 4 * math.pi * b ** 3 * (xi - 0.5) * 3
    theta = (-c1 ** 2 + math.sqrt(c1 ** 4 + 8 * c1 ** 2 * c2 * (1 - 1 / xi))) / (4 * c2)
    assert zp == pytest.approx(1.0 - theta, rel=1e-13)
    # -grad E of the electrostatic term on the beads with the largest forces
    top = np.argsort(-np.linalg.norm(f, axis=1))[:12]
    h = 1e-6
    for i in top:
        for d in range(3):
            ev = []
            for sgn in (1, -1):
                xp = x0.copy()
                xp[i, d] += sgn * h
                o.set_state(xp[None])
                o.neighbor()
                ev.append(o.energy()[7])
            g = -(ev[0] - ev[1]) / (2 * h)
            assert abs(f[i, d] - g) <= 1e-5 * max(np.abs(f).max(), 1.0), (i, d, f[i, d], g)
    o.close()

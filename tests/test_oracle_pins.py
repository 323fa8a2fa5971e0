"""Pins of the CPU restatement (oracle/) -- CPU only.

The reference is Fortran and ships no golden vectors for this path, so the
restatement is pinned by the checks the reference itself relies on:

* F = -grad E by central differences with h = 1e-4
  (src/simu_checkforce.F90:99-133), term by term;
* Ewald energy against a direct lattice sum (utility/coulomb_energy_exact.F90),
  with the surface term 2 pi |M|^2 / 3V that separates spherical summation
  from the tin-foil Ewald sum;
* the Ewald k-vector table of src/mloop_ewld.F90:56-156 (4168 vectors for
  |h| <= 10, sorted by |h|^2, both signs of every h);
* the dielectric constant, Debye length and Coulomb prefactor of
  src/simu_ele_set.F90 at 280/300/400 K and 100/150 mM;
* the neighbour list of src/neighbor_list.F90:49-90 restated in numpy;
* one Langevin step (src/time_integral.F90:152-183 with the constants of
  src/time_integral_pre.F90:160-171) restated in numpy;
* the odd/even pair alternation of the replica exchange
  (src/simu_replica_exchange.F90:121-267, src/var_replica.F90:134,165-183).
"""
import numpy as np
import pytest

from tis_b200 import synth
from oracle.oracle import Oracle, boltz

E_IDX = {"bond": 3, "angle": 4, "stack": 16, "hbond": 17, "exv": 18, "dh": 8, "tstack": 19}


def hairpin():
    s = synth.set_friction(synth.dt15_chain(22, 1, stem=6), 0.5)
    return synth.hairpin_coords(s, 6, seed=1), {}


def dense_noclamp():
    # pairs inside the excluded-volume range, none at the DE_MAX clamp
    return synth.set_friction(synth.dt15_chain(30, 5, min_dist=3.0, confine=10.0), 0.5), {}


def periodic_ions():
    s = synth.set_friction(synth.dt15_chain(12, 7, stem=3), 0.5)
    s = synth.add_ions(s, 40.0, {"Mg": 2, "K": 12, "Cl": 5}, 8, clash=6.0)
    return s, dict(i_periodic=1, psize=(40.0, 40.0, 40.0))


def hairpin_tertiary():
    return synth.hairpin_tertiary(1), {}


FD_SYSTEMS = {"hairpin": hairpin, "dense_noclamp": dense_noclamp, "periodic_ions": periodic_ions,
              "hairpin_tertiary": hairpin_tertiary}


def fd_forces(o, x0, h=1e-4):
    fd = {t: np.zeros_like(x0) for t in E_IDX}
    for i in range(x0.shape[0]):
        for d in range(3):
            xp = x0.copy()
            xp[i, d] += h
            o.set_state(xp[None])
            o.neighbor()
            ep = o.energy()
            xm = x0.copy()
            xm[i, d] -= h
            o.set_state(xm[None])
            o.neighbor()
            em = o.energy()
            for t, k in E_IDX.items():
                fd[t][i, d] = -(ep[k - 1] - em[k - 1]) / (2 * h)
    return fd


@pytest.fixture(scope="module")
def fd_cache():
    out = {}
    for name, fn in FD_SYSTEMS.items():
        s, extra = fn()
        par = synth.dt15_params(ionic_strength=0.15, **extra)
        o = Oracle(s, par, [300.0])
        x0 = s["xyz"].copy()
        o.set_state(x0[None])
        o.neighbor()
        forces = {t: o.force_term(t) for t in E_IDX}
        o.force()
        clamped = o.nclamp() > 0
        out[name] = (forces, fd_forces(o, x0), clamped)
        o.close()
    return out


@pytest.mark.parametrize("term", list(E_IDX))
@pytest.mark.parametrize("name", list(FD_SYSTEMS))
def test_force_is_minus_energy_gradient(fd_cache, name, term):
    forces, fd, clamped = fd_cache[name]
    if term == "exv" and clamped:
        pytest.skip("pair forces clamped at DE_MAX: F is not -grad E there by construction")
    f, g = forces[term], fd[term]
    scale = max(np.abs(f).max(), 1.0)
    assert np.abs(f - g).max() <= 1e-5 * scale, (name, term, np.abs(f - g).max(), scale)


def test_fd_systems_exercise_every_term(fd_cache):
    for term in E_IDX:
        assert any(np.abs(v[0][term]).max() > 0.1 for v in fd_cache.values()), term
    assert not fd_cache["dense_noclamp"][2]


def test_tertiary_stacks_turn_off_secondary_stacks():
    """force_dtrna_stack_nlocal.F90:83-92 with mloop_dtrna.F90:74-140: a
    tertiary stack within 10 A of its native distance turns off the
    secondary stacks of its exclusive sides; the others stay on."""
    s = synth.hairpin_tertiary(1)
    par = synth.dt15_params(ionic_strength=0.15)
    o = Oracle(s, par, [300.0])
    o.set_state(s["xyz"][None])
    o.neighbor()
    e = o.energy()
    st = s["idtrna_st2mp"]
    expect_off = set()
    for k in range(s["ntst"]):
        m = s["idtrna_tst2mp"][k]
        d = np.linalg.norm(s["xyz"][m[0] - 1] - s["xyz"][m[1] - 1]) - s["dtrna_tst_nat"][k, 0]
        if d >= 10.0:
            continue
        for sd in range(2):
            b = m[sd]
            b2 = b - 3 if s["idtrna_tst2side"][k, sd] == 1 else b + 3
            for ist in range(s["nst"]):
                if {st[ist, 0], st[ist, 1]} == {b, b2} and s["flg_tst_exclusive"][k, sd]:
                    expect_off.add(ist)
    assert expect_off
    # the stack energy equals the sum over the stacks left on
    s_on = dict(s, ntst=0)
    o2 = Oracle(s_on, par, [300.0])
    per = []
    for ist in range(s["nst"]):
        keep = dict(s_on, nst=1, idtrna_st2mp=st[ist:ist + 1], dtrna_st_nat=s["dtrna_st_nat"][ist:ist + 1],
                    coef_dtrna_st=s["coef_dtrna_st"][ist:ist + 1], dtrna_st_hsTm=s["dtrna_st_hsTm"][ist:ist + 1])
        ok = Oracle(keep, par, [300.0])
        ok.set_state(s["xyz"][None])
        ok.neighbor()
        per.append(ok.energy()[15])
        ok.close()
    want = sum(v for ist, v in enumerate(per) if ist not in expect_off)
    assert abs(e[15] - want) <= 1e-12 * max(1.0, abs(want))
    assert e[18] < 0.0
    o.close(); o2.close()


def test_coulomb_force_is_minus_energy_gradient():
    """force_ele_coulomb.F90 against the central differences of
    energy_ele_coulomb.F90 (cutoff 200 A: no pair near it)."""
    s, _ = hairpin()
    par = synth.dt15_params(ionic_strength=0.15, i_ele=3, cutoff_ele=200.0)
    o = Oracle(s, par, [300.0])
    x0 = s["xyz"].copy()
    o.set_state(x0[None])
    o.neighbor()
    f = o.force_term("coulomb")
    h = 1e-4
    g = np.zeros_like(x0)
    for i in range(x0.shape[0]):
        for d in range(3):
            e = []
            for sgn in (1, -1):
                xp = x0.copy()
                xp[i, d] += sgn * h
                o.set_state(xp[None])
                o.neighbor()
                e.append(o.energy()[7])
            g[i, d] = -(e[0] - e[1]) / (2 * h)
    assert np.abs(f).max() > 0.1
    assert np.abs(f - g).max() <= 1e-5 * max(np.abs(f).max(), 1.0)
    o.close()


def neutral_ion_box():
    s = synth.set_friction(synth.dt15_chain(8, 3, stem=0), 0.5)
    return synth.add_ions(s, 40.0, {"Mg": 1, "K": 6, "Cl": 1}, 9, clash=6.0)


def test_ewald_matches_direct_lattice_sum():
    s = neutral_ion_box()
    q = np.zeros(s["nmp"])
    q[np.asarray(s["icharge2mp"]) - 1] = s["coef_charge"]
    assert abs(q.sum()) < 1e-12
    L = 40.0
    par = synth.dt15_params(i_periodic=1, psize=(L, L, L), i_ele=2, ewld_alpha=0.2, ewld_hmax=10.0,
                            cutoff_ele=19.9)
    o = Oracle(s, par, [300.0])
    o.set_state(s["xyz"][None])
    o.neighbor()
    e_ewald = o.energy()[7]
    p = o.get_pxyz().reshape(-1, 3)
    M = (q[:, None] * p).sum(0)
    coef = o.label_params(1)["coef"]
    surface = coef * 2.0 * np.pi / (3.0 * L ** 3) * (M @ M)
    e_direct = o.coulomb_direct(1, 20)
    assert abs(e_direct - (e_ewald + surface)) < 1e-5 * abs(e_direct)


def test_ewald_kvector_table():
    s = neutral_ion_box()
    L, alpha = 150.0, 0.05
    par = synth.dt15_params(i_periodic=1, psize=(L, L, L), i_ele=2, ewld_alpha=alpha, ewld_hmax=10.0)
    o = Oracle(s, par, [300.0])
    rlv, coef = o.ewald_table()
    assert len(rlv) == 4168
    h = rlv * L / (2 * np.pi)
    assert np.allclose(h, np.round(h), atol=1e-9)
    h2 = np.round((h * h).sum(1)).astype(int)
    assert (np.diff(h2) >= 0).all() and h2.max() <= 100 and h2.min() >= 1
    keys = {tuple(v) for v in np.round(h).astype(int)}
    assert all(tuple(-np.array(k)) in keys for k in keys)
    k2 = (rlv * rlv).sum(1)
    ref = 2 * np.pi / L ** 3 * np.exp(-k2 / (4 * alpha * alpha)) / k2
    assert np.allclose(coef, ref, rtol=1e-12)


@pytest.mark.parametrize("T,ionic,ek,cdist", [
    (300.0, 0.15, 77.63, 7.835), (300.0, 0.10, 77.63, 9.596),
    (280.0, 0.10, 85.04, 9.70), (400.0, 0.10, 49.14, 8.82)])
def test_debye_hueckel_constants(T, ionic, ek, cdist):
    s = neutral_ion_box()
    o = Oracle(s, synth.dt15_params(ionic_strength=ionic), [T])
    lp = o.label_params(1)
    nd = len(str(cdist).split(".")[1])
    assert round(lp["ek"], 2) == pytest.approx(ek, abs=0.011)
    assert round(lp["cdist"], nd) == pytest.approx(cdist, abs=1.1 * 10 ** -nd)
    if T == 300.0:
        assert lp["coef"] == pytest.approx(4.278, abs=5e-4)


def numpy_exv_list(s, par):
    """neighbor_list.F90:49-90 for one RNA chain: pairs i < j with
    j >= i + nsep(type_i) and |r_ij|^2 < (3.2 + neigh_margin)^2."""
    x = s["xyz"]
    n = s["nmp"]
    nsep = {synth_type: k for synth_type, k in ((2, par["n_sep_nlocal_P"]), (4, par["n_sep_nlocal_S"]),
                                                 (3, par["n_sep_nlocal_B"]))}
    typ = np.asarray(s["imp2type"])
    cut2 = (max(par["exv_dist"], par["exv_dist_PS"]) + par["neigh_margin"]) ** 2
    out = []
    for i in range(n):
        for j in range(i + nsep[int(typ[i])], n):
            d = x[j] - x[i]
            if d @ d < cut2:
                out.append((i + 1, j + 1, 1))
    return np.array(out, dtype=np.int32).reshape(-1, 3)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_exv_list_matches_numpy_restatement(seed):
    s = synth.set_friction(synth.dt15_chain(40, seed, min_dist=3.0, confine=14.0), 0.5)
    par = synth.dt15_params()
    o = Oracle(s, par, [300.0])
    o.set_state(s["xyz"][None])
    o.neighbor()
    got = o.exv_list()
    ref = numpy_exv_list(s, par)
    got_sorted = got[np.lexsort((got[:, 1], got[:, 0]))]
    assert len(got) > 100
    assert np.array_equal(got_sorted, ref)


def test_langevin_step_matches_numpy_restatement():
    s, _ = hairpin()
    par = synth.dt15_params(ionic_strength=0.15)
    T = 300.0
    o = Oracle(s, par, [T])
    n = s["nmp"]
    rng = np.random.default_rng(3)
    x0 = s["xyz"].copy()
    v0 = rng.normal(0, 0.3, (n, 3))
    noise = rng.normal(size=(2, 1, n, 3))
    o.set_state(x0[None], v0[None], np.zeros((1, n, 3)))
    o.set_noise(noise)
    o.time_integral_pre()
    _, _, a0 = (z.reshape(n, 3) for z in o.get_state())
    o.step(1)
    x1, v1, a1 = (z.reshape(n, 3) for z in o.get_state())
    dt = par["tstep"]
    g = np.asarray(s["fric"])[:, None]
    m = np.asarray(s["cmass"])[:, None]
    kb = boltz()
    u = 1.0 - 0.5 * g * dt
    c1 = np.sqrt(2.0 * g * kb * T / (dt * m))
    c2 = u * (1.0 - 0.5 * g * dt + (0.5 * g * dt) ** 2)
    c3 = 0.5 * dt * u
    c4 = dt * u
    assert np.allclose(x1, x0 + c4 * v0 + 0.5 * dt * dt * a0, rtol=0, atol=1e-12)
    q = Oracle(s, par, [T])
    q.set_state(x1[None])
    q.neighbor()
    f1, _ = q.force()
    a1_ref = f1 / m + c1 * noise[1, 0]
    assert np.allclose(a1, a1_ref, rtol=1e-12, atol=1e-12)
    assert np.allclose(v1, c2 * v0 + c3 * (a0 + a1_ref), rtol=1e-12, atol=1e-12)


def test_replica_exchange_pair_alternation():
    s, _ = hairpin()
    temps = list(synth.temperature_ladder(6, 300.0, 330.0))
    o = Oracle(s, synth.dt15_params(), temps)
    o.set_state(np.tile(s["xyz"], (6, 1, 1)))
    o.neighbor()
    for r in range(1, 7):
        o.force(r)
    assert list(o.labels()) == [1, 2, 3, 4, 5, 6]
    # u = 0 accepts every attempted swap: first the (1,2),(3,4),(5,6) pairs ...
    o.replica_exchange(np.zeros(6))
    assert list(o.labels()) == [2, 1, 4, 3, 6, 5]
    for r in range(1, 7):
        o.force(r)
    # ... then (2,3),(4,5) of the temperature labels
    o.replica_exchange(np.zeros(6))
    lab = list(o.labels())
    assert sorted(lab) == [1, 2, 3, 4, 5, 6]
    assert lab == [3, 1, 5, 2, 6, 4]

"""The diffusion tensors of simu_hydro_tensors.F90 in the oracle, pinned on CPU.

* Against a vectorised numpy restatement of each HI_TENSOR variant
  (const_index.F90:39-45): RPY (:139-182), RPY_OVER (:187-236), ERMAK_OVER
  (:241-290) with the radius of bead 1, and Zuk et al.'s RPY with per-bead
  radii (:50-124), on chains with overlapping beads and, for Zuk-RPY, a bead
  inside another: relative 1e-14.
* Continuity of each overlap formula at its switch distance (r = 2a for
  RPY_OVER; r = a_i + a_j and r = |a_i - a_j| for Zuk-RPY), a property of the
  published tensors that the code does not use.
* The overlap-corrected RPY tensors (RPY_OVER, Zuk-RPY) stay positive
  definite where the plain RPY tensor does not (the Ermak-McCammon variant
  carries no such guarantee and is not checked for it).
"""
import numpy as np
import pytest

from tis_b200 import synth
from oracle.oracle import Oracle

BOLTZ = 1.38064852e-23 / 4184.0 * 6.022140857e23


def tensor_np(x, radii, kind, T, visc):
    N = len(x)
    c6 = BOLTZ * T / (6.0 * np.pi * visc)
    c8 = BOLTZ * T / (8.0 * np.pi * visc)
    D = np.zeros((3 * N, 3 * N))
    a = radii[0]
    for i in range(N):
        for j in range(i + 1, N):
            r = x[j] - x[i]
            rs = r @ r
            ra = np.sqrt(rs)
            if kind == 4:
                ai, aj = radii[i], radii[j]
                if ai + aj < ra:
                    p1 = c8 / ra * (1 + (ai * ai + aj * aj) / (3 * rs))
                    p2 = c8 / ra * (1 - (ai * ai + aj * aj) / rs) / rs
                elif abs(ai - aj) < ra:
                    rc = rs * ra
                    p1 = c6 / ai / aj * (16 * rc * (ai + aj) - ((ai - aj) ** 2 + 3 * rs) ** 2) / 32 / rc
                    p2 = c6 / ai / aj * 3 * ((ai - aj) ** 2 - rs) ** 2 / 32 / rc / rs
                else:
                    D[3 * i:3 * i + 3, 3 * j:3 * j + 3] = c6 / max(ai, aj) * np.eye(3)
                    continue
            elif kind == 1 or 2 * a < ra:
                p1 = c8 / ra * (1 + 2 * a * a / (3 * rs))
                p2 = c8 / ra * (1 - 2 * a * a / rs) / rs
            elif kind == 2:
                p1 = c6 / a * (1 - 9 / 32 * ra / a)
                p2 = c6 / a * 3 / 32 / a / ra
            else:
                p1 = c8 / 2 / a * 7 / 6
                p2 = c8 / 2 / 2 / rs
            D[3 * i:3 * i + 3, 3 * j:3 * j + 3] = p1 * np.eye(3) + p2 * np.outer(r, r)
    D = D + D.T
    diag = np.repeat(radii if kind == 4 else np.full(N, a), 3)
    D[np.diag_indices(3 * N)] = c6 / diag
    return D


def chain(n, seed, radii=None, nest=False):
    s = dict(synth.bead_chain(n, seed))
    x = s["xyz"] * 0.85                      # consecutive beads overlap (3.2 A < 2 x 2 A)
    if nest:
        x = x.copy()
        x[n // 2] = x[n // 2 - 3] + np.array([0.3, 0.1, -0.2])   # a small bead inside a large one
    s["xyz"] = x
    if radii is not None:
        s["radius"] = radii
    return s


@pytest.mark.parametrize("kind", [1, 2, 3, 4])
def test_oracle_tensor_matches_numpy(kind):
    n = 24
    rng = np.random.default_rng(kind)
    radii = rng.uniform(1.2, 2.8, n) if kind == 4 else None
    if kind == 4:
        radii[n // 2], radii[n // 2 - 3] = 1.0, 2.6
    s = chain(n, 5, radii, nest=(kind == 4))
    par = synth.bdhi_params(i_hydro_tensor=kind)
    orc = Oracle(s, par, [300.0])
    orc.set_state(s["xyz"][None])
    D, _, _ = orc.hydro_tensors(cholesky=False)
    ref = tensor_np(s["xyz"], radii if radii is not None else np.full(n, par["hi_radius"]), kind, 300.0,
                    par["viscosity"])
    assert np.abs(D - ref).max() <= 1e-14 * np.abs(ref).max()
    assert np.array_equal(D, D.T)


def _pair_pre(kind, r, ai, aj, a=2.0):
    x = np.array([[0.0, 0.0, 0.0], [r, 0.0, 0.0]])
    D = tensor_np(x, np.array([ai, aj]) if kind == 4 else np.array([a, a]), kind, 300.0, 2.944)
    blk = D[0:3, 3:6]
    return blk[1, 1], blk[0, 0] - blk[1, 1]      # pre1, pre2 r^2


@pytest.mark.parametrize("kind,r0,ai,aj", [(2, 4.0, 2.0, 2.0), (4, 3.5, 1.5, 2.0), (4, 1.0, 1.5, 2.5)])
def test_overlap_formulas_are_continuous(kind, r0, ai, aj):
    lo = _pair_pre(kind, r0 * (1 - 1e-9), ai, aj)
    hi = _pair_pre(kind, r0 * (1 + 1e-9), ai, aj)
    assert lo[0] == pytest.approx(hi[0], rel=1e-7)
    assert lo[1] == pytest.approx(hi[1], rel=1e-6, abs=1e-9)


@pytest.mark.parametrize("kind", [2, 4])
def test_overlap_tensors_stay_positive_definite(kind):
    n = 30
    s = chain(n, 11)
    s["xyz"] = s["xyz"] * 0.5                # pairs well inside 2a
    par = synth.bdhi_params(i_hydro_tensor=kind)
    orc = Oracle(s, par, [300.0])
    orc.set_state(s["xyz"][None])
    _, L, rc = orc.hydro_tensors()
    assert rc == 0
    assert np.linalg.eigvalsh(tensor_np(s["xyz"], np.full(n, 2.0), 1, 300.0, par["viscosity"])).min() < 0

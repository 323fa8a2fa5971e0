"""ctypes wrapper of oracle/libtis_oracle.so, the CPU FP64 restatement of the
reference path.  TEST INFRASTRUCTURE: imported only by tests/, by
__graft_entry__.smoke() as the checker, and by bench.py's cpu_baseline leg.

Parity status: unpinned against reference outputs (no Fortran compiler and
no golden vectors for this path ship with the reference); pinned by
F = -grad E, Ewald vs direct lattice sum and analytic cases (see tests).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from tis_b200.abi import (ETYPE_MAX, Params, Topology, make_params, make_topology,
                          ptr_f64, ptr_i32)

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}


def _host_tag() -> str:
    """The host CPU's model and feature flags, hashed: a -march=native build
    is used only on the kind of CPU it was built on."""
    import hashlib
    info = ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith(("model name", "flags")):
                    info += line
                if line.startswith("flags"):
                    break
    except OSError:
        pass
    return hashlib.sha1(info.encode()).hexdigest()[:12]


# the checker (-O2, built with the package) and the copy timed as the CPU
# baseline (-O3 -march=native, built on the host that runs it)
_FILES = {"checker": "libtis_oracle.so", "native": f"libtis_oracle_native-{_host_tag()}.so"}


def build(quiet: bool = True):
    cmd = ["make", "-C", _HERE]
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL if quiet else None)


def build_native() -> bool:
    """Builds the timing copy for this host; False when that fails."""
    r = subprocess.run(["make", "-C", _HERE, "native", f"NATIVE_SO={_FILES['native']}"],
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    return r.returncode == 0 and os.path.exists(os.path.join(_HERE, _FILES["native"]))


def lib(variant: str = "checker"):
    if variant not in _LIBS:
        path = os.path.join(_HERE, _FILES[variant])
        if not os.path.exists(path):
            build() if variant == "checker" else build_native()
        L = C.CDLL(path)
        vp = C.c_void_p
        i32p, f64p = C.POINTER(C.c_int32), C.POINTER(C.c_double)
        L.orc_create.argtypes = [C.POINTER(Topology), C.POINTER(Params), C.c_int, f64p]
        L.orc_create.restype = vp
        L.orc_destroy.argtypes = [vp]
        L.orc_destroy.restype = None
        L.orc_set_state.argtypes = [vp, f64p, f64p, f64p]
        L.orc_get_state.argtypes = [vp, f64p, f64p, f64p]
        L.orc_get_pxyz.argtypes = [vp, f64p]
        L.orc_set_noise.argtypes = [vp, f64p, C.c_int, f64p, C.c_int]
        L.orc_neighbor.argtypes = [vp, C.c_int]
        L.orc_get_exv_list.argtypes = [vp, C.c_int, i32p, C.c_int]
        L.orc_get_ele_list.argtypes = [vp, C.c_int, i32p, f64p, C.c_int]
        L.orc_get_hb_list.argtypes = [vp, C.c_int, i32p, C.c_int]
        L.orc_get_hb_status.argtypes = [vp, C.c_int, i32p, f64p]
        L.orc_force_sumup.argtypes = [vp, C.c_int, f64p]
        L.orc_force_term.argtypes = [vp, C.c_int, C.c_int, f64p]
        L.orc_energy_sumup.argtypes = [vp, C.c_int, f64p, C.c_int]
        L.orc_time_integral_pre.argtypes = [vp]
        L.orc_step.argtypes = [vp, C.c_long]
        L.orc_replica_exchange.argtypes = [vp, f64p, i32p]
        L.orc_get_labels.argtypes = [vp, i32p]
        L.orc_label_params.argtypes = [vp, C.c_int, f64p]
        L.orc_ewald_table.argtypes = [vp, f64p, f64p, C.c_int]
        L.orc_coulomb_direct.argtypes = [vp, C.c_int, C.c_int]
        L.orc_coulomb_direct.restype = C.c_double
        L.orc_hydro_tensors.argtypes = [vp, C.c_int, f64p, f64p]
        L.orc_not_spd.argtypes = [vp]
        L.orc_nclamp.argtypes = [vp]
        L.orc_replica_energy.argtypes = [vp, C.c_int, f64p]
        L.orc_rex_apply.argtypes = [vp, i32p, f64p]
        L.orc_rebuild_info.argtypes = [vp, C.c_int, C.POINTER(C.c_long), C.POINTER(C.c_long)]
        L.orc_rebuild_info.restype = None
        L.orc_pmf_range.argtypes = [vp]
        L.orc_pmf_range.restype = C.c_int
        L.orc_label_pmf.argtypes = [vp, C.c_int, f64p, f64p, f64p, C.c_int]
        L.orc_label_pmf.restype = C.c_int
        L.orc_nclamp.restype = C.c_long
        L.orc_boltz_kcal_mol.restype = C.c_double
        _LIBS[variant] = L
    return _LIBS[variant]


TERMS = {"bond": 0, "angle": 1, "stack": 2, "hbond": 3, "exv": 4, "dh": 5, "ewald": 6, "fene": 7, "wca": 8,
         "tstack": 9, "coulomb": 10}


class Oracle:
    """One topology, nrep replicas (labels = temperatures tempk)."""

    def __init__(self, sysd: dict, par: dict, tempk, variant: str = "checker"):
        self.L = lib(variant)
        self.sysd = sysd
        self.nmp = int(sysd["nmp"])
        self.nrep = len(tempk)
        self._t, self._keep = make_topology(sysd)
        self._p = make_params(**par)
        self._T = np.ascontiguousarray(np.asarray(tempk, dtype=np.float64))
        self.h = self.L.orc_create(C.byref(self._t), C.byref(self._p), self.nrep, ptr_f64(self._T))

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _arr(self, *shape):
        return np.zeros(shape, dtype=np.float64)

    def set_state(self, xyz, velo=None, accel=None):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        v = None if velo is None else np.ascontiguousarray(velo, dtype=np.float64)
        a = None if accel is None else np.ascontiguousarray(accel, dtype=np.float64)
        self.L.orc_set_state(self.h, ptr_f64(xyz), None if v is None else ptr_f64(v), None if a is None else ptr_f64(a))

    def get_state(self):
        x, v, a = (self._arr(self.nrep, self.nmp, 3) for _ in range(3))
        self.L.orc_get_state(self.h, ptr_f64(x), ptr_f64(v), ptr_f64(a))
        return x, v, a

    def get_pxyz(self):
        p = self._arr(self.nrep, self.nmp, 3)
        self.L.orc_get_pxyz(self.h, ptr_f64(p))
        return p

    def set_noise(self, noise, uniforms=None):
        noise = np.ascontiguousarray(noise, dtype=np.float64)
        nsteps = noise.shape[0]
        if uniforms is not None:
            u = np.ascontiguousarray(uniforms, dtype=np.float64)
            self.L.orc_set_noise(self.h, ptr_f64(noise), nsteps, ptr_f64(u), u.shape[-1])
        else:
            self.L.orc_set_noise(self.h, ptr_f64(noise), nsteps, None, 0)

    def neighbor(self, irep=-1):
        self.L.orc_neighbor(self.h, irep)

    def exv_list(self, irep=1):
        n = self.L.orc_get_exv_list(self.h, irep, None, 0)
        out = np.zeros((max(n, 1), 3), dtype=np.int32)
        self.L.orc_get_exv_list(self.h, irep, ptr_i32(out), n)
        return out[:n]

    def ele_list(self, irep=1):
        n = self.L.orc_get_ele_list(self.h, irep, None, None, 0)
        out = np.zeros((max(n, 1), 4), dtype=np.int32)
        coef = np.zeros(max(n, 1))
        self.L.orc_get_ele_list(self.h, irep, ptr_i32(out), ptr_f64(coef), n)
        return out[:n], coef[:n]

    def hb_list(self, irep=1):
        n = self.L.orc_get_hb_list(self.h, irep, None, 0)
        out = np.zeros(max(n, 1), dtype=np.int32)
        self.L.orc_get_hb_list(self.h, irep, ptr_i32(out), n)
        return out[:n]

    def hb_status(self, irep=1):
        nhb = max(int(self.sysd.get("nhb", 0)), 1)
        st = np.zeros(nhb, dtype=np.int32)
        ene = np.zeros(nhb)
        self.L.orc_get_hb_status(self.h, irep, ptr_i32(st), ptr_f64(ene))
        return st, ene

    def force(self, irep=1):
        f = self._arr(self.nmp, 3)
        rc = self.L.orc_force_sumup(self.h, irep, ptr_f64(f))
        return f, rc

    def force_term(self, term, irep=1):
        f = self._arr(self.nmp, 3)
        self.L.orc_force_term(self.h, irep, TERMS[term], ptr_f64(f))
        return f

    def energy(self, irep=1, reuse_hb=False):
        e = np.zeros(ETYPE_MAX)
        self.L.orc_energy_sumup(self.h, irep, ptr_f64(e), 1 if reuse_hb else 0)
        return e

    def time_integral_pre(self):
        return self.L.orc_time_integral_pre(self.h)

    def step(self, n):
        return self.L.orc_step(self.h, int(n))

    def replica_exchange(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        na = C.c_int32(0)
        self.L.orc_replica_exchange(self.h, ptr_f64(u), C.byref(na))
        return na.value

    def replica_energy(self, irep):
        """(E at the own label, E at the exchange partner's label or 0)."""
        out = np.zeros(2)
        self.L.orc_replica_energy(self.h, irep, ptr_f64(out))
        return out

    def rex_apply(self, rep2lab, vscale):
        r = np.ascontiguousarray(rep2lab, dtype=np.int32)
        v = np.ascontiguousarray(vscale, dtype=np.float64)
        self.L.orc_rex_apply(self.h, ptr_i32(r), ptr_f64(v))

    def labels(self):
        out = np.zeros(self.nrep, dtype=np.int32)
        self.L.orc_get_labels(self.h, ptr_i32(out))
        return out

    def label_params(self, label):
        out = np.zeros(4)
        self.L.orc_label_params(self.h, label, ptr_f64(out))
        return dict(ek=out[0], coef=out[1], cdist=out[2], beta_hbond15=out[3])

    def ewald_table(self):
        n = self.L.orc_ewald_table(self.h, None, None, 0)
        rlv = np.zeros((n, 3))
        coef = np.zeros(n)
        self.L.orc_ewald_table(self.h, ptr_f64(rlv), ptr_f64(coef), n)
        return rlv, coef

    def coulomb_direct(self, irep=1, nlat=10):
        return self.L.orc_coulomb_direct(self.h, irep, nlat)

    def hydro_tensors(self, irep=1, cholesky=True):
        """(D, L, rc) of replica irep at its current coordinates: the
        tensor tis_params.i_hydro_tensor selects, with the bead radii."""
        n = 3 * self.nmp
        D = np.zeros((n, n))
        Lm = np.zeros((n, n)) if cholesky else None
        rc = self.L.orc_hydro_tensors(self.h, irep, ptr_f64(D), None if Lm is None else ptr_f64(Lm))
        # column-major (3N, 3N) buffers: transpose to row-major views
        return D.T.copy(), (None if Lm is None else Lm.T.copy()), rc

    def not_spd(self):
        return self.L.orc_not_spd(self.h)

    def nclamp(self):
        return self.L.orc_nclamp(self.h)

    def rebuild_info(self, irep=1):
        """(neighbour rebuilds of replica irep, istep of the last one)."""
        n, last = C.c_long(0), C.c_long(0)
        self.L.orc_rebuild_info(self.h, irep, C.byref(n), C.byref(last))
        return n.value, last.value

    def pmf_range(self):
        return self.L.orc_pmf_range(self.h)

    def label_pmf(self, label):
        """(Zp, PMF+DH energy table, force table) of a label."""
        zp = C.c_double(0.0)
        n = self.L.orc_label_pmf(self.h, label, C.byref(zp), None, None, 0)
        e, f = np.zeros(max(n, 1)), np.zeros(max(n, 1))
        self.L.orc_label_pmf(self.h, label, C.byref(zp), ptr_f64(e), ptr_f64(f), n)
        return zp.value, e[:n], f[:n]


BOLTZ_KCAL_MOL = None


def boltz():
    return lib().orc_boltz_kcal_mol()

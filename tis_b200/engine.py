"""Python mirror of the C-ABI (include/tis_b200.h) over ctypes.

``Engine`` owns one ``tis_ctx``: a batch of replicas (lanes) of one or more
topologies on cuda:0.  Method names follow the reference routines they
replace (neighbor, force_sumup, energy_sumup, time_integral_pre,
time_integral, replica exchange).  Every call goes through the in-tree
``libtis_b200.so``; a missing library raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .abi import (ETYPE_MAX, Params, Status, Topology, load_library, make_params,
                  make_topology, ptr_f64, ptr_i32)


class TisError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"tis error {code}: {msg}")
        self.code = code


class Engine:
    def __init__(self, systems, par: dict, tempk, nrep=None, ladder=None):
        """systems: list of topology dicts (tis_b200.synth); nrep[k] replicas of
        systems[k] (default 1 each) with temperatures tempk (one per lane).
        ladder=(tempk_all, irep_first): this engine holds replicas irep_first
        .. irep_first + len(tempk) - 1 (1-based) of the ladder tempk_all of one
        system split over ranks (tis_init_ladder); tempk are their starting
        temperatures."""
        self.L = load_library()
        if isinstance(systems, dict):
            systems = [systems]
        self.systems = list(systems)
        if nrep is None:
            nrep = [1] * len(self.systems) if len(self.systems) > 1 else [len(tempk)]
        self.nrep = list(int(n) for n in nrep)
        self.tempk = np.ascontiguousarray(np.asarray(tempk, dtype=np.float64))
        assert sum(self.nrep) == len(self.tempk)
        self._keep = []
        tops = (Topology * len(self.systems))()
        for k, s in enumerate(self.systems):
            t, keep = make_topology(s)
            tops[k] = t
            self._keep.append(keep)
        self._tops = tops
        self._par = make_params(**par)
        self.par = dict(par)
        nr = np.ascontiguousarray(np.asarray(self.nrep, dtype=np.int32))
        self._nr = nr
        h = C.c_void_p()
        self.ladder = None
        if ladder is not None:
            tall = np.ascontiguousarray(np.asarray(ladder[0], dtype=np.float64))
            self.ladder = (tall, int(ladder[1]))
            assert len(self.systems) == 1
            rc = self.L.tis_init_ladder(tops, C.byref(self._par), len(tall), ptr_f64(tall), int(ladder[1]),
                                        len(self.tempk), C.byref(h))
        else:
            rc = self.L.tis_init_batch(len(self.systems), tops, C.byref(self._par), ptr_i32(nr),
                                       ptr_f64(self.tempk), C.byref(h))
        if rc != 0 or not h.value:
            raise TisError(rc, "tis_init_batch failed")
        self.h = h
        self.nlane = self.L.tis_nrep(self.h)
        self.lane_nmp = [self.L.tis_nmp(self.h, i + 1) for i in range(self.nlane)]
        self.systems_of_lane = [s for s, r in zip(self.systems, self.nrep) for _ in range(r)]
        self.nbead = int(sum(self.lane_nmp))
        self.offsets = np.concatenate([[0], np.cumsum(self.lane_nmp)]).astype(int)

    # ------------------------------------------------------------------
    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.tis_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc < 0:
            msg = self.L.tis_last_error(self.h)
            raise TisError(rc, f"{what}: {msg.decode() if msg else ''}")
        return rc

    # state: arrays of shape (nbead_total, 3) with lanes concatenated
    def set_state(self, xyz, velo=None, accel=None):
        x = np.ascontiguousarray(xyz, dtype=np.float64).reshape(self.nbead, 3)
        v = None if velo is None else np.ascontiguousarray(velo, dtype=np.float64).reshape(self.nbead, 3)
        a = None if accel is None else np.ascontiguousarray(accel, dtype=np.float64).reshape(self.nbead, 3)
        self._check(self.L.tis_set_state(self.h, ptr_f64(x), None if v is None else ptr_f64(v),
                                         None if a is None else ptr_f64(a)), "set_state")

    def get_state(self):
        x, v, a = (np.zeros((self.nbead, 3)) for _ in range(3))
        self._check(self.L.tis_get_state(self.h, ptr_f64(x), ptr_f64(v), ptr_f64(a)), "get_state")
        return x, v, a

    def get_pxyz(self):
        p = np.zeros((self.nbead, 3))
        self._check(self.L.tis_get_pxyz(self.h, ptr_f64(p)), "get_pxyz")
        return p

    def set_noise(self, noise=None, uniforms=None):
        if noise is not None:
            n = np.ascontiguousarray(noise, dtype=np.float64)
            nsteps = n.shape[0]
            np_ = ptr_f64(n)
        else:
            nsteps, np_ = 0, None
        if uniforms is not None:
            u = np.ascontiguousarray(uniforms, dtype=np.float64)
            nu = u.shape[-1]
            up = ptr_f64(u)
        else:
            nu, up = 0, None
        self._keep_noise = (noise, uniforms)
        self._check(self.L.tis_set_noise(self.h, np_, nsteps, up, nu), "set_noise")

    def neighbor(self, irep=-1):
        return self._check(self.L.tis_neighbor(self.h, irep), "neighbor")

    def exv_list(self, irep=1):
        n = C.c_int32(0)
        self.L.tis_get_exv_list(self.h, irep, None, 0, C.byref(n))
        out = np.zeros((max(n.value, 1), 3), dtype=np.int32)
        self._check(self.L.tis_get_exv_list(self.h, irep, ptr_i32(out), n.value, C.byref(n)), "exv_list")
        return out[:n.value]

    def ele_list(self, irep=1):
        n = C.c_int32(0)
        self.L.tis_get_ele_list(self.h, irep, None, None, 0, C.byref(n))
        out = np.zeros((max(n.value, 1), 4), dtype=np.int32)
        coef = np.zeros(max(n.value, 1))
        self._check(self.L.tis_get_ele_list(self.h, irep, ptr_i32(out), ptr_f64(coef), n.value, C.byref(n)), "ele_list")
        return out[:n.value], coef[:n.value]

    def hb_list(self, irep=1):
        n = C.c_int32(0)
        self.L.tis_get_hb_list(self.h, irep, None, 0, C.byref(n))
        out = np.zeros(max(n.value, 1), dtype=np.int32)
        self._check(self.L.tis_get_hb_list(self.h, irep, ptr_i32(out), n.value, C.byref(n)), "hb_list")
        return out[:n.value]

    def force(self, irep=1):
        f = np.zeros((self.lane_nmp[irep - 1], 3))
        rc = self._check(self.L.tis_force_sumup(self.h, irep, ptr_f64(f)), "force_sumup")
        return f, rc

    def energy(self, irep=1):
        e = np.zeros(ETYPE_MAX)
        self._check(self.L.tis_energy_sumup(self.h, irep, ptr_f64(e)), "energy_sumup")
        return e

    def time_integral_pre(self):
        return self._check(self.L.tis_time_integral_pre(self.h), "time_integral_pre")

    def step(self, n):
        return self._check(self.L.tis_step(self.h, int(n)), "step")

    def run(self, nperiod, nstep, exchange=True):
        """nperiod periods of nstep steps of every replica, each followed by
        a replica exchange with counter-based uniforms when exchange is set,
        replayed from one recorded CUDA graph; one host wait at the end."""
        return self._check(self.L.tis_run(self.h, int(nperiod), int(nstep), 1 if exchange else 0), "run")

    def time_integral(self, n, flags, exchange_step=None):
        """n calls of time_integral(flg_step_each_replica): flags (nrep int32,
        updated in place) freeze replicas; exchange_step (nrep int64) stops
        a replica there and sets its flag."""
        assert flags.dtype == np.int32 and flags.shape == (self.nlane,)
        ex = None
        if exchange_step is not None:
            ex = np.ascontiguousarray(exchange_step, dtype=np.int64)
            self._keep_ex = ex
        return self._check(self.L.tis_time_integral(self.h, int(n), ptr_i32(flags),
                                                    None if ex is None else ex.ctypes.data_as(C.POINTER(C.c_int64))),
                           "time_integral")

    def random_number(self, istep, nstep):
        """(nstep, nbead, 3) Gaussian noise of the counter-based generator at
        steps istep .. istep + nstep - 1."""
        out = np.zeros((nstep, self.nbead, 3))
        self._check(self.L.tis_get_random_number(self.h, int(istep), int(nstep), ptr_f64(out)), "random_number")
        return out

    def steps(self):
        out = np.zeros(self.nlane, dtype=np.int64)
        self._check(self.L.tis_get_steps(self.h, out.ctypes.data_as(C.POINTER(C.c_int64))), "get_steps")
        return out

    def rebuild_info(self, irep=1):
        """(neighbour rebuilds of replica irep, step of the last one)."""
        n, last = C.c_int64(0), C.c_int64(0)
        self._check(self.L.tis_get_rebuild_info(self.h, irep, C.byref(n), C.byref(last)), "rebuild_info")
        return n.value, last.value

    def last_step_ms(self):
        return self.L.tis_last_step_ms(self.h)

    def timer_start(self):
        self._check(self.L.tis_timer(self.h, 0, None), "timer")

    def timer_stop(self) -> float:
        ms = C.c_double(0.0)
        self._check(self.L.tis_timer(self.h, 1, C.byref(ms)), "timer")
        return ms.value

    def replica_exchange(self, u=None, count=True):
        """One exchange; returns the number of accepted swaps.  count=False
        skips that count, so the exchange stays on the device stream with no
        host wait (returns None)."""
        na = C.c_int32(0)
        up = None
        if u is not None:
            uu = np.ascontiguousarray(u, dtype=np.float64)
            up = ptr_f64(uu)
        self._check(self.L.tis_replica_exchange(self.h, up, C.byref(na) if count else None), "replica_exchange")
        return na.value if count else None

    def rex_energies(self):
        """(nrep_local, 2): energy at the own label and at the exchange
        partner's label of this ladder engine's replicas."""
        out = np.zeros((self.nlane, 2))
        self._check(self.L.tis_rex_energies(self.h, ptr_f64(out)), "rex_energies")
        return out

    def rex_exchange_all(self, energies_all, u=None):
        """The exchange of the whole ladder from the gathered (nrep_all, 2)
        energies; returns the number of accepted swaps."""
        e = np.ascontiguousarray(energies_all, dtype=np.float64)
        na = C.c_int32(0)
        up = None if u is None else ptr_f64(np.ascontiguousarray(u, dtype=np.float64))
        self._check(self.L.tis_rex_exchange_all(self.h, ptr_f64(e), up, C.byref(na)), "rex_exchange_all")
        return na.value

    def hydro_tensors(self, irep=1):
        """(D, L) of the last Brownian-HI refresh, row-major (3N, 3N) arrays."""
        n = 3 * self.lane_nmp[irep - 1]
        D = np.zeros((n, n))
        Lm = np.zeros((n, n))
        self._check(self.L.tis_get_hydro_tensors(self.h, irep, ptr_f64(D), ptr_f64(Lm)), "hydro_tensors")
        # column-major buffers: transpose to row-major views
        return D.T.copy(), Lm.T.copy()

    def launch_count(self) -> int:
        return int(self.L.tis_launch_count(self.h))

    def set_step(self, istep: int):
        self._check(self.L.tis_set_step(self.h, int(istep)), "set_step")

    def dtrna_status(self, irep=1):
        """(hb_status, st_status) of replica irep as 0/1 int32 arrays."""
        t = self.systems_of_lane[irep - 1]
        hb = np.zeros(max(int(t.get("nhb", 0)), 1), dtype=np.int32)
        st = np.ones(max(int(t.get("nst", 0)), 1), dtype=np.int32)
        self._check(self.L.tis_get_dtrna_status(self.h, irep, ptr_i32(hb), ptr_i32(st)), "dtrna_status")
        return hb[:int(t.get("nhb", 0))], st[:int(t.get("nst", 0))]

    def labels(self):
        out = np.zeros(self.nlane, dtype=np.int32)
        self._check(self.L.tis_get_labels(self.h, ptr_i32(out)), "labels")
        return out

    def status(self):
        st = Status()
        self._check(self.L.tis_status(self.h, C.byref(st)), "status")
        return {k: getattr(st, k) for k, _ in Status._fields_}

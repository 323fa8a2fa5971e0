"""ctypes mirror of include/tis_b200.h (structs, enums) and the loader of the
in-tree CUDA library ``tis_b200/libtis_b200.so``.

The struct layouts must match the header field for field; ``tests`` check
the sizes against the compiled library (``tis_sizeof_*`` exports).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

# ---- enums (values of src/const_index.F90 in the reference) -------------
CLASS_RNA, CLASS_LIG, CLASS_ION = 2, 3, 4
MP_RNA_PHOS, MP_RNA_BASE, MP_RNA_SUGAR = 2, 3, 4
MP_ION_MG, MP_ION_CA2, MP_ION_NA, MP_ION_K, MP_ION_CL = 5, 6, 7, 8, 9
E_TOTAL, E_VELO, E_BOND, E_BANGLE, E_ELE = 1, 2, 3, 4, 8
E_STACK_DTRNA, E_HBOND_DTRNA, E_EXV_DT15 = 16, 17, 18
E_TSTACK_DTRNA, E_THBOND_DTRNA, E_WCA_REP, E_WCA_ATT = 19, 20, 23, 24
ETYPE_MAX = 25
SIM_LANGEVIN, SIM_BROWNIAN_HI = 1, 6
HI_RPY, HI_RPY_OVER, HI_ERMAK_OVER, HI_ZUK_RPY = 1, 2, 3, 4
ELE_NONE, ELE_DH, ELE_EWALD = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1

TIS_OK = 0
TIS_E_ARG = -1
TIS_E_CUDA = -2
TIS_E_LIST_OVERFLOW = -3
TIS_E_NOT_SPD = -4
TIS_E_TIMEOUT = -5
TIS_E_NOISE_EXHAUSTED = -6
TIS_E_UNSUPPORTED = -7
TIS_E_NAN = -8
TIS_E_PMF_RANGE = -9

_i32p = C.POINTER(C.c_int32)
_f64p = C.POINTER(C.c_double)


class Topology(C.Structure):
    _fields_ = [
        ("nmp", C.c_int32), ("nunit", C.c_int32),
        ("lunit2mp", _i32p), ("iclass_unit", _i32p), ("imp2type", _i32p),
        ("cmass", _f64p), ("fric", _f64p), ("exv_radius", _f64p), ("exv_epsilon", _f64p),
        ("ncharge", C.c_int32), ("icharge2mp", _i32p), ("coef_charge", _f64p),
        ("nbd", C.c_int32), ("ibd2mp", _i32p), ("bd_nat", _f64p), ("coef_bd", _f64p),
        ("nba", C.c_int32), ("iba2mp", _i32p), ("ba_nat", _f64p), ("coef_ba", _f64p),
        ("nst", C.c_int32), ("idtrna_st2mp", _i32p), ("dtrna_st_nat", _f64p),
        ("coef_dtrna_st", _f64p), ("dtrna_st_hsTm", _f64p),
        ("nhb", C.c_int32), ("idtrna_hb2mp", _i32p), ("dtrna_hb_nat", _f64p),
        ("coef_dtrna_hb", _f64p), ("idtrna_hb2hbsite", _i32p),
        ("nhbsite", C.c_int32), ("nvalence_hbsite", _i32p),
        ("nfene", C.c_int32), ("ifene2mp", _i32p), ("fene_nat", _f64p),
        ("coef_fene", _f64p), ("dist2_fene", _f64p),
        ("nwca", C.c_int32), ("iwca2mp", _i32p), ("wca_nat", _f64p), ("coef_wca", _f64p),
        ("ntst", C.c_int32), ("idtrna_tst2mp", _i32p), ("dtrna_tst_nat", _f64p),
        ("coef_dtrna_tst", _f64p), ("idtrna_tst2side", _i32p), ("flg_tst_exclusive", _i32p),
        ("flg_hb_tertiary", _i32p), ("flg_charge_fixed", _i32p), ("radius", _f64p),
    ]


class Params(C.Structure):
    _fields_ = [
        ("i_periodic", C.c_int32), ("psize", C.c_double * 3),
        ("neigh_margin", C.c_double), ("n_step_neighbor", C.c_int32),
        ("exv_dist", C.c_double), ("exv_dist_PS", C.c_double),
        ("exv_adjust", C.c_double), ("exv_inf", C.c_double),
        ("n_sep_nlocal_P", C.c_int32), ("n_sep_nlocal_S", C.c_int32), ("n_sep_nlocal_B", C.c_int32),
        ("hb_cutoff_dist", C.c_double),
        ("i_ele", C.c_int32), ("i_diele", C.c_int32), ("diele_water", C.c_double),
        ("ionic_strength", C.c_double), ("cutoff_ele", C.c_double),
        ("i_DH_cutoff_type", C.c_int32), ("ewld_alpha", C.c_double), ("ewld_hmax", C.c_double),
        ("i_simulate_type", C.c_int32), ("tstep", C.c_double),
        ("viscosity", C.c_double), ("wca_coef_cutoff", C.c_double),
        ("precision", C.c_int32), ("hb_beta_global", C.c_int32), ("seed", C.c_uint64),
        ("hi_radius", C.c_double), ("n_step_hydro", C.c_int32),
        ("i_dtrna_model", C.c_int32), ("i_charge", C.c_int32), ("length_per_unit_P", C.c_double),
        ("pmf_nbin", C.c_int32), ("pmf_rmin", C.c_double), ("pmf_rbin", C.c_double), ("pmf_rmax", C.c_double),
        ("pmf_rmerge", C.c_double), ("pmf_mg_p", _f64p), ("hi_refine", C.c_int32), ("i_hydro_tensor", C.c_int32),
        ("launch_threads", C.c_int32), ("launch_group", C.c_int32), ("launch_ctas", C.c_int32),
        ("launch_noise_sweep", C.c_int32), ("launch_order", C.c_int32), ("launch_table", C.c_char_p),
        ("launch_sweep", C.c_int32),
    ]


class Status(C.Structure):
    _fields_ = [
        ("step", C.c_int64), ("n_rebuild", C.c_int64), ("n_clamp", C.c_int64),
        ("list_overflow", C.c_int32), ("nan_seen", C.c_int32), ("wait_timeout", C.c_int32),
        ("not_spd", C.c_int32), ("last_error", C.c_int32),
        ("exv_pairs_max", C.c_int32), ("ele_pairs_max", C.c_int32), ("ctas_per_lane", C.c_int32),
        ("threads_per_cta", C.c_int32), ("group", C.c_int32), ("noise_sweep", C.c_int32),
        ("lane_order", C.c_int32), ("launch_source", C.c_int32), ("sweep", C.c_int32),
    ]


def ptr_f64(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_f64p)


def ptr_i32(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_i32p)


# Fields of Topology that carry arrays, with their dtype.
_TOPO_ARRAYS = {
    "lunit2mp": np.int32, "iclass_unit": np.int32, "imp2type": np.int32,
    "cmass": np.float64, "fric": np.float64, "exv_radius": np.float64, "exv_epsilon": np.float64,
    "icharge2mp": np.int32, "coef_charge": np.float64,
    "ibd2mp": np.int32, "bd_nat": np.float64, "coef_bd": np.float64,
    "iba2mp": np.int32, "ba_nat": np.float64, "coef_ba": np.float64,
    "idtrna_st2mp": np.int32, "dtrna_st_nat": np.float64, "coef_dtrna_st": np.float64,
    "dtrna_st_hsTm": np.float64,
    "idtrna_hb2mp": np.int32, "dtrna_hb_nat": np.float64, "coef_dtrna_hb": np.float64,
    "idtrna_hb2hbsite": np.int32, "nvalence_hbsite": np.int32,
    "ifene2mp": np.int32, "fene_nat": np.float64, "coef_fene": np.float64, "dist2_fene": np.float64,
    "iwca2mp": np.int32, "wca_nat": np.float64, "coef_wca": np.float64,
    "idtrna_tst2mp": np.int32, "dtrna_tst_nat": np.float64, "coef_dtrna_tst": np.float64,
    "idtrna_tst2side": np.int32, "flg_tst_exclusive": np.int32,
    "flg_hb_tertiary": np.int32, "flg_charge_fixed": np.int32, "radius": np.float64,
}
# Arrays the library accepts as NULL (their absence has a meaning of its own).
_TOPO_OPTIONAL = ("flg_hb_tertiary", "flg_charge_fixed", "radius")
_TOPO_COUNTS = ("nmp", "nunit", "ncharge", "nbd", "nba", "nst", "nhb", "nhbsite", "nfene", "nwca", "ntst")


def make_topology(sysd: dict):
    """Builds a ``Topology`` from a dict of numpy arrays (see tis_b200.synth).
    Index tables are record-major, shape (nrec, k), i.e. the Fortran (k, nrec)
    layout; ``coef_wca`` is (2, nwca) like the Fortran (nwca, 2).
    Returns (struct, keepalive) -- keep ``keepalive`` referenced while the
    struct is in use."""
    keep = {}
    t = Topology()
    for k in _TOPO_COUNTS:
        setattr(t, k, int(sysd.get(k, 0)))
    for k, dt in _TOPO_ARRAYS.items():
        a = sysd.get(k)
        if k in _TOPO_OPTIONAL and a is None:
            continue
        if a is None or np.size(a) == 0:
            a = np.zeros(1, dtype=dt)
        # record-major (nrec, k) C-order arrays are the Fortran (k, nrec) layout
        a = np.ascontiguousarray(np.asarray(a, dtype=dt)).ravel()
        keep[k] = a
        setattr(t, k, a.ctypes.data_as(_i32p if dt == np.int32 else _f64p))
    return t, keep


def make_params(**kw) -> Params:
    """A ``Params`` from keyword values; ``pmf_mg_p`` takes an array, which
    the returned struct keeps referenced (``p._keep``)."""
    p = Params()
    p._keep = []
    for k, v in kw.items():
        if k == "psize":
            for i in range(3):
                p.psize[i] = float(v[i])
        elif k == "launch_table":
            if v is not None:
                b = str(v).encode()
                p._keep.append(b)
                p.launch_table = b
        elif k == "pmf_mg_p":
            if v is not None:
                a = np.ascontiguousarray(np.asarray(v, dtype=np.float64))
                p._keep.append(a)
                p.pmf_mg_p = a.ctypes.data_as(_f64p)
        else:
            setattr(p, k, v)
    return p


_LIB = None


def library_path() -> str:
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "libtis_b200.so")


def load_library():
    """Loads the in-tree CUDA library.  There is no CPU fallback: a missing
    or unloadable library is an error."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not os.path.exists(path):
        raise RuntimeError(f"libtis_b200.so not built ({path}); run python -c 'import __graft_entry__ as g; g.build()'")
    lib = C.CDLL(path)
    _declare(lib)
    _LIB = lib
    return lib


EXPORTED = [
    "tis_init", "tis_init_batch", "tis_destroy", "tis_nrep", "tis_nmp",
    "tis_set_state", "tis_get_state", "tis_get_pxyz", "tis_set_noise",
    "tis_neighbor", "tis_get_exv_list", "tis_get_ele_list", "tis_get_hb_list",
    "tis_force_sumup", "tis_energy_sumup", "tis_time_integral_pre", "tis_step", "tis_run",
    "tis_replica_exchange", "tis_get_labels", "tis_status", "tis_last_step_ms",
    "tis_last_error", "tis_timer", "tis_force_sumup_static", "tis_launch_count",
    "tis_get_hydro_tensors", "tis_set_step", "tis_get_dtrna_status",
    "tis_time_integral", "tis_get_steps", "tis_get_rebuild_info", "tis_get_random_number",
    "tis_init_ladder", "tis_rex_energies", "tis_rex_exchange_all", "tis_rex_decide",
]


def _declare(lib):
    vp = C.c_void_p
    lib.tis_init.argtypes = [C.POINTER(Topology), C.POINTER(Params), C.c_int32, _f64p, C.POINTER(vp)]
    lib.tis_init_batch.argtypes = [C.c_int32, C.POINTER(Topology), C.POINTER(Params), _i32p, _f64p, C.POINTER(vp)]
    lib.tis_destroy.argtypes = [vp]
    lib.tis_destroy.restype = None
    lib.tis_nrep.argtypes = [vp]
    lib.tis_nmp.argtypes = [vp, C.c_int32]
    lib.tis_set_state.argtypes = [vp, _f64p, _f64p, _f64p]
    lib.tis_get_state.argtypes = [vp, _f64p, _f64p, _f64p]
    lib.tis_get_pxyz.argtypes = [vp, _f64p]
    lib.tis_set_noise.argtypes = [vp, _f64p, C.c_int32, _f64p, C.c_int32]
    lib.tis_neighbor.argtypes = [vp, C.c_int32]
    lib.tis_get_exv_list.argtypes = [vp, C.c_int32, _i32p, C.c_int32, _i32p]
    lib.tis_get_ele_list.argtypes = [vp, C.c_int32, _i32p, _f64p, C.c_int32, _i32p]
    lib.tis_get_hb_list.argtypes = [vp, C.c_int32, _i32p, C.c_int32, _i32p]
    lib.tis_force_sumup.argtypes = [vp, C.c_int32, _f64p]
    lib.tis_energy_sumup.argtypes = [vp, C.c_int32, _f64p]
    lib.tis_time_integral_pre.argtypes = [vp]
    lib.tis_step.argtypes = [vp, C.c_int64]
    lib.tis_run.argtypes = [vp, C.c_int32, C.c_int64, C.c_int32]
    lib.tis_replica_exchange.argtypes = [vp, _f64p, _i32p]
    lib.tis_get_labels.argtypes = [vp, _i32p]
    lib.tis_status.argtypes = [vp, C.POINTER(Status)]
    lib.tis_last_step_ms.argtypes = [vp]
    lib.tis_last_step_ms.restype = C.c_double
    lib.tis_last_error.argtypes = [vp]
    lib.tis_last_error.restype = C.c_char_p
    lib.tis_timer.argtypes = [vp, C.c_int32, _f64p]
    lib.tis_force_sumup_static.argtypes = [vp, C.c_int32, vp, vp]
    lib.tis_get_hydro_tensors.argtypes = [vp, C.c_int32, _f64p, _f64p]
    lib.tis_set_step.argtypes = [vp, C.c_int64]
    lib.tis_get_dtrna_status.argtypes = [vp, C.c_int32, _i32p, _i32p]
    lib.tis_time_integral.argtypes = [vp, C.c_int64, _i32p, C.POINTER(C.c_int64)]
    lib.tis_init_ladder.argtypes = [C.POINTER(Topology), C.POINTER(Params), C.c_int32, _f64p, C.c_int32, C.c_int32,
                                    C.POINTER(vp)]
    lib.tis_rex_energies.argtypes = [vp, _f64p]
    lib.tis_rex_exchange_all.argtypes = [vp, _f64p, _f64p, _i32p]
    lib.tis_rex_decide.argtypes = [C.c_int32, _f64p, C.c_int32, _f64p, _f64p, _i32p, _f64p, _i32p]
    lib.tis_get_random_number.argtypes = [vp, C.c_int64, C.c_int32, _f64p]
    lib.tis_get_steps.argtypes = [vp, C.POINTER(C.c_int64)]
    lib.tis_get_rebuild_info.argtypes = [vp, C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    lib.tis_launch_count.argtypes = [vp]
    lib.tis_launch_count.restype = C.c_int64

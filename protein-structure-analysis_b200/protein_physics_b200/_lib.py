"""ctypes binding of libalma_b200.so (the C ABI in include/alma_b200.h).

Loading fails loudly: there is no fallback implementation.  Every call
checks the returned status and raises RuntimeError / ValueError with the
library's thread-local message.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libalma_b200.so")

ALMA_OK = 0
ALMA_EINVAL = -1
ALMA_ECUDA = -2
ALMA_ECAPACITY = -3
ALMA_EDEVICE = -4

PREC_MIXED = 0
PREC_FP64 = 1

ST_NL_OVERFLOW = 1
ST_CELL_OVERFLOW = 2
ST_BAD_INDEX = 4
ST_NONFINITE = 8
ST_SPEC_ABORT = 16

_p = C.c_void_p
_i32 = C.c_int32
_i64 = C.c_int64


class AlmaParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "coulomb", "eps_water", "eps_prot", "kappa", "gamma_sa", "beta_sa", "probe_r",
        "pair_cut2", "nl_rcut2", "half_skin2", "hard_scale", "hard_cap", "hard_frac",
        "k_ss", "r0_ss")]


class AlmaBatch(C.Structure):
    _fields_ = [("nsys", _i32), ("natoms", _i32), ("atom_off", _p), ("xyz", _p), ("prm", _p),
                ("prm64", _p), ("born", _p), ("status", _p), ("sasa", _p)]


class AlmaTopo(C.Structure):
    _fields_ = [("excl_ptr", _p), ("excl_cols", _p),
                ("nrb", _i32), ("rb_off", _p), ("rb_ij", _p), ("rb_kind", _p), ("rb_scale", _p),
                ("side_ptr", _p), ("side_idx", _p), ("side_lo", _p), ("side_hi", _p),
                ("ndih", _i32), ("dih_off", _p), ("dih_abcd", _p), ("term_off", _p), ("term_v2", _p),
                ("term_n", _p), ("term_gamma", _p),
                ("nss", _i32), ("ss_off", _p), ("ss_ij", _p),
                ("ncp", _i32), ("cp_off", _p), ("cp", _p),
                ("ncsp", _i32), ("csp_off", _p), ("csp", _p), ("excl_win", _p)]


class AlmaNL(C.Structure):
    _fields_ = [("full_ptr", _p), ("full_len", _p), ("full_cols", _p), ("full_base", _p),
                ("half_ptr", _p), ("half_len", _p), ("half_cols", _p), ("half_base", _p),
                ("ref_xyz", _p), ("need", _p),
                ("sfull_ptr", _p), ("sfull_len", _p), ("sfull_cols", _p), ("sfull_base", _p),
                ("shalf_ptr", _p), ("shalf_len", _p), ("shalf_cols", _p), ("shalf_base", _p),
                ("full_span", _p)]


class AlmaMCConfig(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("policy", _i32), ("tune_freq", _i32),
                ("target_lo", C.c_double), ("target_hi", C.c_double),
                ("scale_up", C.c_double), ("scale_down", C.c_double),
                ("angle_max", C.c_double), ("angle_min", C.c_double),
                ("sidechain_mult", C.c_double), ("crank_prob", C.c_double),
                ("concerted_prob", C.c_double), ("fixed_delta", C.c_double),
                ("moveset_off", _p), ("moveset", _p), ("threads_per_system", _i32), ("cluster_size", _i32),
                ("spec_teams", _i32), ("pad", _i32), ("rebuild_ws", _p), ("sys_order", _p),
                ("launch_systems", _i32), ("pad2", _i32)]


class AlmaChainState(C.Structure):
    _fields_ = [("cur_max", C.c_double), ("energy", C.c_double), ("temperature", C.c_double),
                ("step", _i64), ("n_proposed", _i64), ("n_accepted", _i64), ("n_rebuild", _i64),
                ("acc_win", _i32), ("tot_win", _i32), ("need_rebuild", _i32), ("parity", _i32)]


# numpy view of AlmaChainState (72 bytes)
STATE_DTYPE = np.dtype([("cur_max", "f8"), ("energy", "f8"), ("temperature", "f8"), ("step", "i8"),
                        ("n_proposed", "i8"), ("n_accepted", "i8"), ("n_rebuild", "i8"), ("acc_win", "i4"),
                        ("tot_win", "i4"), ("need_rebuild", "i4"), ("parity", "i4")])
assert STATE_DTYPE.itemsize == C.sizeof(AlmaChainState) == 72



class AlmaTorsionTree(C.Structure):
    _fields_ = [("rb_parent", _p), ("atom_rb", _p)]


class AlmaMalaState(C.Structure):
    _fields_ = [("energy", C.c_double), ("beta", C.c_double), ("scale", C.c_double), ("log_alpha", C.c_double),
                ("step", C.c_int64), ("n_proposed", C.c_int64), ("n_accepted", C.c_int64), ("acc_win", C.c_int32),
                ("tot_win", C.c_int32)]


class AlmaMalaConfig(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("drift_clip", C.c_double), ("tune_freq", C.c_int32), ("pad", C.c_int32),
                ("target_lo", C.c_double), ("target_hi", C.c_double), ("scale_up", C.c_double),
                ("scale_down", C.c_double), ("scale_min", C.c_double), ("scale_max", C.c_double)]


MALA_STATE_DTYPE = np.dtype([("energy", "f8"), ("beta", "f8"), ("scale", "f8"), ("log_alpha", "f8"), ("step", "i8"),
                             ("n_proposed", "i8"), ("n_accepted", "i8"), ("acc_win", "i4"), ("tot_win", "i4")])
assert MALA_STATE_DTYPE.itemsize == C.sizeof(AlmaMalaState) == 64

_lib = None


def lib():
    """The loaded library (raises if it is missing: no fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"protein_physics_b200: native library missing ({LIB_PATH}); build it with "
            "`python protein-structure-analysis_b200/build.py` (nvcc, sm_100a)")
    L = C.CDLL(LIB_PATH)
    L.alma_abi_version.restype = C.c_int
    L.alma_launch_count.restype = C.c_longlong
    L.alma_last_error.restype = C.c_char_p
    L.alma_params_reference.argtypes = [C.POINTER(AlmaParams)]
    L.alma_nl_workspace_bytes.restype = C.c_size_t
    L.alma_nl_workspace_bytes.argtypes = [_i32, _i32, _i64]
    L.alma_move_scratch_bytes.restype = C.c_size_t
    L.alma_move_scratch_bytes.argtypes = [_i32]
    L.alma_mc_scratch_bytes.restype = C.c_size_t
    L.alma_mc_scratch_bytes.argtypes = [_i32, _i32, _i32]
    L.alma_mc_rebuild_bytes.restype = C.c_size_t
    L.alma_mc_rebuild_bytes.argtypes = [_i32, _i32]
    L.alma_spec_round_bytes.restype = C.c_size_t
    L.alma_spec_round_bytes.argtypes = []
    L.alma_spec_wait_selftest.argtypes = [_p, _p, _p, _p]
    L.alma_topo_sides.argtypes = [_i32, _p, _p, _i32, _p, _p, _p, _i64]
    L.alma_topo_sides_compact.argtypes = [_i32, _p, _p, _i32, _p, _p, _p, _p, _p, _p, _i64]
    L.alma_nl_build.argtypes = [_p, _p, _p, _p, _p, _p, _i64, _p]
    L.alma_excl_window.argtypes = [_p, _p, _i32, _p, _p]
    L.alma_born_radii.argtypes = [_p, _p, _p, C.c_int, _p, _p]
    L.alma_energy.argtypes = [_p, _p, _p, _p, C.c_int, _p, _p, _p, _p]
    L.alma_forces_workspace_bytes.restype = C.c_size_t
    L.alma_forces_workspace_bytes.argtypes = [_i32]
    L.alma_forces.argtypes = [_p, _p, _p, _p, C.c_int, _p, _p, _p, _p]
    L.alma_torsion_tree.argtypes = [_i32, _i32, _p, _p, _p, _p, _p, _p, _p]
    L.alma_torsion_workspace_bytes.restype = C.c_size_t
    L.alma_torsion_workspace_bytes.argtypes = [_i32, _i32, _i32]
    L.alma_torsion_grad.argtypes = [_p, _p, _p, _p, _p, _p, _p]
    L.alma_torsion_apply.argtypes = [_p, _p, _p, _p, _p, _p, _p]
    L.alma_mala_propose.argtypes = [_p, _i32, _p, _p, _p, _p, _p, _p, _p]
    L.alma_mala_accept.argtypes = [_p, _i32, _p, _p, _p, _p, _p, _p, _p, _p, _p, _p]
    L.alma_mala_select.argtypes = [_p, _p, _p, _p, _p, _p, _p, _p, _p]
    L.alma_mean_dist_matrix.argtypes = [_p, _i32, _i32, _p, _p]
    L.alma_contact_freq_matrix.argtypes = [_p, _i32, _i32, C.c_double, _p, _p]
    L.alma_replica_exchange.argtypes = [_i32, _p, _p, _p, _p, C.c_uint64, _i64, _p, _p, _p]
    L.alma_mc_run.argtypes = [_p, _p, _p, _p, C.c_int, _p, _p, _p, _i64, _p]
    L.alma_mc_after_rebuild.argtypes = [_p, _p, _p, _i32, _p]
    L.alma_move_scratch_init.argtypes = [_p, _i32, _p]
    L.alma_move_counters.argtypes = [_p, _i32, _i32, _p, _p]
    L.alma_move_dE.argtypes = [_p, _p, _p, _p, C.c_int, _p, _p, _p, _p, C.c_int, _p, _p, _p]
    if L.alma_abi_version() != 1:
        raise RuntimeError("protein_physics_b200: ABI version mismatch")
    _lib = L
    return L


def check(rc: int, what: str = ""):
    if rc == ALMA_OK:
        return
    msg = lib().alma_last_error().decode(errors="replace")
    if rc == ALMA_EINVAL:
        raise ValueError(f"{what}: {msg}")
    raise RuntimeError(f"{what}: {msg} (code {rc})")


def reference_params() -> AlmaParams:
    p = AlmaParams()
    lib().alma_params_reference(C.byref(p))
    return p


def topo_sides(n, adj_ptr, adj_idx, bonds_ij):
    """j-side atom lists (DFS order) for each (i, j) bond — host call."""
    nb = len(bonds_ij)
    bonds = np.ascontiguousarray(np.asarray(bonds_ij, dtype=np.int32).reshape(-1, 2))
    adj_ptr = np.ascontiguousarray(adj_ptr, dtype=np.int64)
    adj_idx = np.ascontiguousarray(adj_idx, dtype=np.int32)
    side_ptr = np.zeros(nb + 1, dtype=np.int64)
    cap = max(16, 8 * n)
    while True:
        side_idx = np.zeros(cap, dtype=np.int32)
        rc = lib().alma_topo_sides(n, adj_ptr.ctypes.data, adj_idx.ctypes.data, nb, bonds.ctypes.data,
                                   side_ptr.ctypes.data, side_idx.ctypes.data, cap)
        if rc == ALMA_ECAPACITY:
            cap = int(side_ptr[-1])
            continue
        check(rc, "alma_topo_sides")
        break
    return [side_idx[side_ptr[k]:side_ptr[k + 1]].tolist() for k in range(nb)]


def topo_sides_compact(n, adj_ptr, adj_idx, bonds_ij):
    """Compact j-sides: (lo, hi, count, ex_ptr, ex_idx) numpy arrays."""
    nb = len(bonds_ij)
    bonds = np.ascontiguousarray(np.asarray(bonds_ij, dtype=np.int32).reshape(-1, 2))
    adj_ptr = np.ascontiguousarray(adj_ptr, dtype=np.int64)
    adj_idx = np.ascontiguousarray(adj_idx, dtype=np.int32)
    lo = np.zeros(nb, np.int32)
    hi = np.zeros(nb, np.int32)
    cnt = np.zeros(nb, np.int64)
    ex_ptr = np.zeros(nb + 1, np.int64)
    cap = max(16, 32 * nb)
    while True:
        ex_idx = np.zeros(cap, np.int32)
        rc = lib().alma_topo_sides_compact(n, adj_ptr.ctypes.data, adj_idx.ctypes.data, nb, bonds.ctypes.data,
                                           lo.ctypes.data, hi.ctypes.data, cnt.ctypes.data, ex_ptr.ctypes.data,
                                           ex_idx.ctypes.data, cap)
        if rc == ALMA_ECAPACITY:
            cap = int(ex_ptr[-1])
            continue
        check(rc, "alma_topo_sides_compact")
        break
    return lo, hi, cnt, ex_ptr, ex_idx[:int(ex_ptr[-1])].copy()

"""TEST INFRASTRUCTURE — Python wrappers of the two CPU checkers.

* ``Oracle``   : oracle/alma_oracle.so, the plain-C FP64 restatement of the
                 reference path (alma_oracle.c cites the reference lines).
* ``RefEngine``: oracle/_ref/protein_physics*.so, the reference engine
                 itself compiled from its own sources (oracle/Makefile),
                 reached through the ref_* C symbols of oracle/ref_shim.cpp.

Only the test suite, the smoke check and bench.py's CPU-baseline leg use
this module, and only as the checker / the baseline.  Parity of ``Oracle``
against the reference is pinned by tests/test_oracle_golden.py on the
golden vectors in tests/golden/ (generated by tests/golden/make_golden.py).
"""
from __future__ import annotations

import ctypes as C
import glob
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "alma_oracle.so")

_p = C.c_void_p


class OrTopo(C.Structure):
    _fields_ = [("n", C.c_int), ("excl_ptr", _p), ("excl_cols", _p), ("ndih", C.c_int), ("dih_abcd", _p),
                ("term_off", _p), ("term_v2", _p), ("term_n", _p), ("term_gamma", _p), ("nss", C.c_int),
                ("ss", _p)]


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


class TopoArrays:
    """Holds the arrays an OrTopo points into (keeps them alive)."""

    def __init__(self, flat):
        self.n = int(flat.n)
        self.excl_ptr = _c(flat.excl_ptr, np.int64)
        self.excl_cols = _c(flat.excl_cols, np.int32)
        self.dih_abcd = _c(flat.dih_abcd, np.int32).reshape(-1)
        self.term_off = _c(flat.term_off, np.int32)
        self.term_v2 = _c(flat.term_v2, np.float64)
        self.term_n = _c(flat.term_n, np.int32)
        self.term_gamma = _c(flat.term_gamma, np.float64)
        self.ss = _c(flat.ss, np.int32).reshape(-1)
        self.s = OrTopo(self.n, self.excl_ptr.ctypes.data, self.excl_cols.ctypes.data, int(flat.dih_abcd.shape[0]),
                        self.dih_abcd.ctypes.data, self.term_off.ctypes.data, self.term_v2.ctypes.data,
                        self.term_n.ctypes.data, self.term_gamma.ctypes.data, int(self.ss.size // 2),
                        self.ss.ctypes.data)

    @property
    def ref(self):
        return C.byref(self.s)


class Oracle:
    """FP64 C restatement (strict IEEE build)."""

    def __init__(self, path=ORACLE_SO):
        if not os.path.exists(path):
            raise RuntimeError(f"oracle not built: {path} (make -C oracle)")
        L = C.CDLL(path)
        d, i64 = C.c_double, C.c_int64
        L.or_nl_build.restype = i64
        L.or_nl_build.argtypes = [C.c_int, _p, _p, _p, i64]
        L.or_born_radii.argtypes = [C.c_int, _p, _p, _p, _p, _p]
        L.or_sasa.restype = d
        L.or_sasa.argtypes = [C.c_int, _p, _p, _p, _p, _p]
        L.or_energy.restype = d
        L.or_energy.argtypes = [C.c_int, _p, _p, _p, _p, _p, _p, _p, _p, _p]
        L.or_calculate_potential.restype = d
        L.or_calculate_potential.argtypes = [C.c_int, _p, _p, _p, _p, _p, _p]
        L.or_move_dE.restype = d
        L.or_move_dE.argtypes = [C.c_int, _p, _p, _p, _p, _p, _p, _p, _p, C.c_int, _p, _p, _p, _p, _p, _p,
                                 _p, _p]
        L.or_pair_e.restype = d
        L.or_pair_e.argtypes = [_p, _p, d, d]
        L.or_hct.restype = d
        L.or_hct.argtypes = [d, d, d, d]
        L.or_dihedral_e.restype = d
        L.or_dihedral_e.argtypes = [_p, _p]
        self.L = L

    def nl_build(self, xyz):
        xyz = _c(xyz, np.float64).reshape(-1, 3)
        n = xyz.shape[0]
        row_ptr = np.zeros(n + 1, np.int64)
        cap = 256 * n + 16
        cols = np.zeros(cap, np.int32)
        m = self.L.or_nl_build(n, xyz.ctypes.data, row_ptr.ctypes.data, cols.ctypes.data, cap)
        if m < 0:
            cap = -m
            cols = np.zeros(cap, np.int32)
            m = self.L.or_nl_build(n, xyz.ctypes.data, row_ptr.ctypes.data, cols.ctypes.data, cap)
        return row_ptr, cols[:m].copy()

    def born_radii(self, xyz, radius, nl):
        xyz = _c(xyz, np.float64).reshape(-1, 3)
        radius = _c(radius, np.float64)
        a = np.zeros(xyz.shape[0])
        self.L.or_born_radii(xyz.shape[0], xyz.ctypes.data, radius.ctypes.data, nl[0].ctypes.data,
                             nl[1].ctypes.data, a.ctypes.data)
        return a

    def sasa(self, xyz, radius, nl, per_atom=False):
        xyz = _c(xyz, np.float64).reshape(-1, 3)
        radius = _c(radius, np.float64)
        sa = np.zeros(xyz.shape[0])
        E = self.L.or_sasa(xyz.shape[0], xyz.ctypes.data, radius.ctypes.data, nl[0].ctypes.data,
                           nl[1].ctypes.data, sa.ctypes.data)
        return (E, sa) if per_atom else E

    def energy(self, xyz, q, radius, eps, nl, born, topo=None):
        """{sasa, dihedral, disulfide, pairs, total} with given NL and radii."""
        xyz = _c(xyz, np.float64).reshape(-1, 3)
        q, radius, eps, born = (_c(v, np.float64) for v in (q, radius, eps, born))
        terms = np.zeros(5)
        self.L.or_energy(xyz.shape[0], xyz.ctypes.data, q.ctypes.data, radius.ctypes.data, eps.ctypes.data,
                         nl[0].ctypes.data, nl[1].ctypes.data, born.ctypes.data,
                         topo.ref if topo is not None else None, terms.ctypes.data)
        return terms

    def calculate_potential(self, xyz, q, radius, eps, topo=None):
        xyz = _c(xyz, np.float64).reshape(-1, 3)
        q, radius, eps = (_c(v, np.float64) for v in (q, radius, eps))
        terms = np.zeros(5)
        self.L.or_calculate_potential(xyz.shape[0], xyz.ctypes.data, q.ctypes.data, radius.ctypes.data,
                                      eps.ctypes.data, topo.ref if topo is not None else None, terms.ctypes.data)
        return terms

    def move_dE(self, xyz, q, radius, eps, nl, born, topo, rotations, group):
        """rotations: list of (axis_i, axis_j, delta, atom_indices) applied in
        order; group: int8[n] move groups.  Returns (dE, terms[4], new_xyz,
        new_born)."""
        xyz = _c(xyz, np.float64).reshape(-1, 3)
        n = xyz.shape[0]
        q, radius, eps, born = (_c(v, np.float64) for v in (q, radius, eps, born))
        axis = _c([[r[0], r[1]] for r in rotations], np.int32).reshape(-1)
        delta = _c([r[2] for r in rotations], np.float64)
        ptr = np.zeros(len(rotations) + 1, np.int64)
        for k, r in enumerate(rotations):
            ptr[k + 1] = ptr[k] + len(r[3])
        idx = _c(np.concatenate([np.asarray(r[3], np.int32) for r in rotations]) if rotations else [], np.int32)
        group = _c(group, np.int8)
        terms = np.zeros(4)
        new_xyz = np.zeros((n, 3))
        new_born = np.zeros(n)
        dE = self.L.or_move_dE(n, xyz.ctypes.data, q.ctypes.data, radius.ctypes.data, eps.ctypes.data,
                               nl[0].ctypes.data, nl[1].ctypes.data, born.ctypes.data, topo.ref, len(rotations),
                               axis.ctypes.data, delta.ctypes.data, ptr.ctypes.data, idx.ctypes.data,
                               group.ctypes.data, terms.ctypes.data, new_xyz.ctypes.data, new_born.ctypes.data)
        return dE, terms, new_xyz, new_born


class OrMCState(C.Structure):
    _fields_ = [("cur_max", C.c_double), ("energy", C.c_double), ("temperature", C.c_double),
                ("step", C.c_int64), ("n_proposed", C.c_int64), ("n_accepted", C.c_int64), ("n_rebuild", C.c_int64),
                ("acc_win", C.c_int32), ("tot_win", C.c_int32), ("need_rebuild", C.c_int32), ("pad", C.c_int32)]


class OrMCCfg(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("policy", C.c_int), ("tune_freq", C.c_int)] + \
               [(n, C.c_double) for n in ("target_lo", "target_hi", "scale_up", "scale_down", "angle_max",
                                          "angle_min", "sidechain_mult", "crank_prob", "concerted_prob",
                                          "fixed_delta")] + [("nset", C.c_int), ("moveset", _p)]


class OrMCSys(C.Structure):
    _fields_ = [("n", C.c_int), ("xyz", _p), ("q", _p), ("radius", _p), ("eps", _p), ("born", _p), ("topo", _p),
                ("nrb", C.c_int), ("rb_ij", _p), ("rb_kind", _p), ("rb_scale", _p), ("side_ptr", _p),
                ("side_idx", _p), ("ncp", C.c_int), ("cp", _p), ("ncsp", C.c_int), ("csp", _p),
                ("sys_index", C.c_int)]


def oracle_mc(orc, flat, xyz, q, radius, eps, seed, steps, temperature=0.6, cur_max=0.12, policy=0,
              fixed_delta=0.0, moveset=None, sys_index=0, tune_freq=200):
    """Runs the oracle's MC chain (alma_oracle.c or_mc_run); returns
    (final xyz [n,3], state dict)."""
    L = orc.L
    L.or_mc_run.argtypes = [_p, _p, _p, C.c_int64]
    n = flat.n
    keep = []

    def arr(a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a.ctypes.data

    x = np.ascontiguousarray(np.asarray(xyz, np.float64).reshape(-1, 3).copy())
    born = np.zeros(n)
    TA = TopoArrays(flat)
    # full sorted j-sides from the compact form
    rows = []
    for k in range(flat.nrb):
        s = set(range(int(flat.side_lo[k]), int(flat.side_hi[k])))
        s.update(flat.side_idx[flat.side_ptr[k]:flat.side_ptr[k + 1]].tolist())
        rows.append(sorted(s))
    sp = np.zeros(flat.nrb + 1, np.int64)
    sp[1:] = np.cumsum([len(r) for r in rows])
    si = np.array([j for r in rows for j in r], np.int32) if sp[-1] else np.zeros(1, np.int32)
    S = OrMCSys(n, x.ctypes.data, arr(q, np.float64), arr(radius, np.float64), arr(eps, np.float64), born.ctypes.data,
                C.cast(C.pointer(TA.s), _p), flat.nrb, arr(np.stack([flat.rb_i, flat.rb_j], 1).reshape(-1), np.int32),
                arr(flat.rb_kind, np.int32), arr(flat.rb_scale, np.float64), arr(sp, np.int64), arr(si, np.int32),
                int(flat.crank.shape[0]), arr(flat.crank.reshape(-1), np.int32) if flat.crank.size else None,
                int(flat.conc_sc.shape[0]), arr(flat.conc_sc.reshape(-1), np.int32) if flat.conc_sc.size else None,
                int(sys_index))
    cfg = OrMCCfg(int(seed) & ((1 << 64) - 1), int(policy), int(tune_freq), 0.28, 0.52, 1.06, 0.94, 0.5, 0.004,
                  2.5, 0.25, 0.15, float(fixed_delta), len(moveset) if moveset is not None else 0,
                  arr(moveset, np.int32) if moveset is not None and len(moveset) else None)
    st = OrMCState(cur_max, 0.0, temperature, 0, 0, 0, 0, 0, 0, 0, 0)
    L.or_mc_run(C.byref(S), C.byref(cfg), C.byref(st), int(steps))
    return x, {f[0]: getattr(st, f[0]) for f in OrMCState._fields_}, born


def ref_so_path():
    hits = glob.glob(os.path.join(HERE, "_ref", "protein_physics*.so"))
    return hits[0] if hits else None


class RefEngine:
    """The reference engine compiled from its own sources (oracle/_ref)."""

    def __init__(self, path=None):
        path = path or ref_so_path()
        if not path or not os.path.exists(path):
            raise RuntimeError("reference build missing (make -C oracle ref, needs the reference sources)")
        L = C.CDLL(path)
        d, i64 = C.c_double, C.c_int64
        L.ref_topo_build.restype = _p
        L.ref_topo_build.argtypes = [C.c_int, _p, _p, _p]
        L.ref_topo_free.argtypes = [_p]
        L.ref_topo_add_disulfide.argtypes = [_p, C.c_int, C.c_int]
        L.ref_topo_concerted_sidechain.argtypes = [_p, C.c_int, _p, d]
        L.ref_nl.restype = i64
        L.ref_nl.argtypes = [C.c_int, _p, _p, _p, i64]
        L.ref_born_radii.argtypes = [C.c_int, _p, _p, _p, _p, _p]
        L.ref_sasa.restype = d
        L.ref_sasa.argtypes = [C.c_int, _p, _p, _p, _p]
        L.ref_energy.restype = d
        L.ref_energy.argtypes = [C.c_int, _p, _p, _p, _p, _p, _p]
        L.ref_move_dE.restype = d
        L.ref_move_dE.argtypes = [C.c_int, _p, _p, _p, _p, _p, C.c_int, C.c_int, d, _p, _p, _p]
        L.ref_pair_e.restype = d
        L.ref_pair_e.argtypes = [_p, _p, d, d]
        L.ref_num_threads.restype = C.c_int
        self.L = L
        self.path = path

    def topology(self, resnames, atomnames, res_idx, ss_pairs=(), xyz=None, cutoff=6.0):
        n = len(resnames)
        rn = (C.c_char_p * n)(*[s.encode() for s in resnames])
        an = (C.c_char_p * n)(*[s.encode() for s in atomnames])
        ri = _c(res_idx, np.int32)
        h = self.L.ref_topo_build(n, C.cast(rn, _p), C.cast(an, _p), ri.ctypes.data)
        for i, j in ss_pairs:
            self.L.ref_topo_add_disulfide(h, int(i), int(j))
        if xyz is not None:
            x = _c(xyz, np.float64).reshape(-1, 3)
            self.L.ref_topo_concerted_sidechain(h, n, x.ctypes.data, cutoff)
        return RefTopoHandle(self.L, h)

    def nl(self, xyz):
        xyz = _c(xyz, np.float64).reshape(-1, 3)
        n = xyz.shape[0]
        counts = np.zeros(n, np.int64)
        cap = 256 * n + 16
        cols = np.zeros(cap, np.int32)
        m = self.L.ref_nl(n, xyz.ctypes.data, counts.ctypes.data, cols.ctypes.data, cap)
        if m < 0:
            cap = -m
            cols = np.zeros(cap, np.int32)
            m = self.L.ref_nl(n, xyz.ctypes.data, counts.ctypes.data, cols.ctypes.data, cap)
        ptr = np.zeros(n + 1, np.int64)
        ptr[1:] = np.cumsum(counts)
        return ptr, cols[:m].copy()

    def born_radii(self, xyz, q, radius, eps):
        xyz = _c(xyz, np.float64).reshape(-1, 3)
        q, radius, eps = (_c(v, np.float64) for v in (q, radius, eps))
        a = np.zeros(xyz.shape[0])
        self.L.ref_born_radii(xyz.shape[0], xyz.ctypes.data, q.ctypes.data, radius.ctypes.data, eps.ctypes.data,
                              a.ctypes.data)
        return a

    def energy(self, xyz, q, radius, eps, topo=None):
        xyz = _c(xyz, np.float64).reshape(-1, 3)
        q, radius, eps = (_c(v, np.float64) for v in (q, radius, eps))
        terms = np.zeros(5)
        self.L.ref_energy(xyz.shape[0], xyz.ctypes.data, q.ctypes.data, radius.ctypes.data, eps.ctypes.data,
                          topo.h if topo is not None else None, terms.ctypes.data)
        return terms

    def move_dE(self, xyz, q, radius, eps, topo, kind, bond, delta):
        xyz = _c(xyz, np.float64).reshape(-1, 3)
        n = xyz.shape[0]
        q, radius, eps = (_c(v, np.float64) for v in (q, radius, eps))
        terms = np.zeros(4)
        new_xyz = np.zeros((n, 3))
        new_a = np.zeros(n)
        dE = self.L.ref_move_dE(n, xyz.ctypes.data, q.ctypes.data, radius.ctypes.data, eps.ctypes.data, topo.h,
                                int(kind), int(bond), float(delta), terms.ctypes.data, new_xyz.ctypes.data,
                                new_a.ctypes.data)
        return dE, terms, new_xyz, new_a


class RefTopoHandle:
    def __init__(self, L, h):
        self.L, self.h = L, h

    def __del__(self):
        try:
            self.L.ref_topo_free(self.h)
        except Exception:
            pass

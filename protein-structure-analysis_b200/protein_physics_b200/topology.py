"""Covalent bond topology: exclusions, rotatable bonds, j-sides, dihedral records.

Host-side input to the energy path, with the surface of the reference's
``protein_physics.BondTopology`` (physics_engine.cpp:1129-1746, bound at
:3726-3841): ``build(resnames, atomnames, res_idx)``, ``add_disulfide``,
``identify_concerted_sidechain_pairs``, ``bonded``, ``is_excluded``,
``j_side`` and the same read-only attributes and flat exports
(``rb_atom_i``, ``dih_term_offsets`` ...).  The residue bond graphs and
rotatable-bond specs are the reference's tables, stored as data in
``data/residue_tables.json`` in their original order; adjacency order
therefore matches the reference's, which fixes the dihedral-record atoms.

``flatten(topo)`` turns this class *or* the reference's own BondTopology
into the CSR arrays the device engine consumes, so either can drive it.
"""
from __future__ import annotations

import enum
import json
import math
import os
from dataclasses import dataclass

import numpy as np

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
with open(os.path.join(_DATA, "residue_tables.json")) as _f:
    _TABLES = json.load(_f)
BOND_TEMPLATES: dict = _TABLES["bond_templates"]
ROT_SPECS: dict = _TABLES["rot_specs"]

# physics_engine.cpp:1565 — N_ref for the lever-arm scale sqrt(N_ref / N_down).
LEVER_NREF = 10.0
# physics_engine.cpp:1652 — cap on concerted sidechain pairs.
MAX_CONCERTED_SC_PAIRS = 4000
# Terminal / protonation patches bonded whenever both atoms exist (:1466-1478).
_PATCHES = (("N", "H1"), ("N", "H2"), ("N", "H3"), ("C", "OXT"), ("NE2", "HE2"))


class BondKind(enum.IntEnum):
    """Rotatable-bond label (physics_engine.cpp:448-478)."""
    BACKBONE_PHI = 0
    BACKBONE_PSI = 1
    SIDECHAIN = 2
    FIXED = 3


@dataclass(frozen=True)
class RotBond:
    """One rotatable bond i -> j; the j-side rotates (physics_engine.cpp:501-508)."""
    i: int
    j: int
    kind: BondKind


@dataclass
class DihRecord:
    a: int
    b: int
    c: int
    d: int
    terms: list  # [(V2, n, gamma)]


def dihedral_terms(kind: BondKind, atomname_j: str) -> list:
    """Fourier terms keyed by bond kind and the j atom's element
    (get_dih_terms, physics_engine.cpp:513-533)."""
    if kind == BondKind.BACKBONE_PHI:
        return [(0.40, 3, math.pi), (0.29, 2, math.pi)]
    if kind == BondKind.BACKBONE_PSI:
        return [(0.40, 3, 0.0), (0.29, 2, math.pi)]
    e = atomname_j[0] if atomname_j else "C"
    if e == "O":
        return [(1.18, 2, math.pi), (0.14, 3, 0.0)]
    if e == "S":
        return [(0.60, 3, 0.0)]
    if e == "N":
        return [(0.50, 3, 0.0), (0.16, 2, 0.0)]
    return [(0.56, 3, 0.0)]


def _adj_csr(n, adj):
    ptr = np.zeros(n + 1, dtype=np.int64)
    for i, row in enumerate(adj):
        ptr[i + 1] = ptr[i] + len(row)
    idx = np.fromiter((j for row in adj for j in row), dtype=np.int32, count=int(ptr[-1]))
    return ptr, idx


def _j_sides(n, adj, bonds_ij):
    """j_side for every (i, j): DFS from j that never enters i
    (physics_engine.cpp:1731-1745), visiting in the reference's stack order."""
    from . import _lib  # native DFS; the pure-Python walk is O(N * bonds)
    ptr, idx = _adj_csr(n, adj)
    return _lib.topo_sides(n, ptr, idx, bonds_ij)


def _j_sides_compact(n, adj, bonds_ij):
    from . import _lib
    ptr, idx = _adj_csr(n, adj)
    return _lib.topo_sides_compact(n, ptr, idx, bonds_ij)


class BondTopology:
    """Drop-in for the reference ``BondTopology`` (same methods/attributes)."""

    def __init__(self):
        self.N = 0
        self.adj: list[list[int]] = []
        self.bonds: list[tuple[int, int]] = []
        self.rot_bonds: list[RotBond] = []
        self._sides_dfs = None
        self._sides = None  # compact (lo, hi, count, ex_ptr, ex_idx)
        self.excl: list[list[int]] = []
        self.dihedrals: list[DihRecord] = []
        self.rot_bond_scale: list[float] = []
        self.concerted_pairs: list[tuple[int, int]] = []
        self.concerted_sidechain_pairs: list[tuple[int, int]] = []
        self.disulfide_pairs: list[tuple[int, int]] = []
        self.atomnames: list[str] = []
        # Bumped by every method that changes the topology; ``flatten`` keys
        # its cached arrays on it.  The reference exposes these attributes
        # read-only (physics_engine.cpp:3732-3740), so the methods below are
        # the only way its state changes.
        self._version = 0
        self._flat = None

    # ---- build (physics_engine.cpp:1341-1597) --------------------------------
    def build(self, resnames, atomnames, res_idx):
        n = len(resnames)
        if len(atomnames) != n or len(res_idx) != n:
            raise ValueError("resnames, atomnames and res_idx must have the same length")
        self._version += 1
        self.N = n
        self.adj = [[] for _ in range(n)]
        self.bonds = []
        self.rot_bonds = []
        self.atomnames = list(atomnames)
        if n == 0:
            return
        lookup = {}
        for k in range(n):  # later duplicates overwrite, as std::map operator[]
            lookup[(int(res_idx[k]), atomnames[k])] = k
        unique_res, res_of = [], {}
        for k in range(n):
            r = int(res_idx[k])
            if r not in res_of:
                unique_res.append(r)
                rn = resnames[k]
                res_of[r] = "HID" if rn == "HIS" else rn

        adj, bonds = self.adj, self.bonds

        def add_bond(i, j):
            if i == j:
                return
            if i > j:
                i, j = j, i
            adj[i].append(j)
            adj[j].append(i)
            bonds.append((i, j))

        for r in unique_res:  # intra-residue template bonds
            for a, b in BOND_TEMPLATES.get(res_of[r], ()):
                ia, ib = lookup.get((r, a)), lookup.get((r, b))
                if ia is not None and ib is not None:
                    add_bond(ia, ib)
        for r1, r2 in zip(unique_res, unique_res[1:]):  # peptide bonds
            if r2 != r1 + 1:
                continue
            ic, inn = lookup.get((r1, "C")), lookup.get((r2, "N"))
            if ic is not None and inn is not None:
                add_bond(ic, inn)
        for r in unique_res:  # terminal / protonation patches
            for a, b in _PATCHES:
                ia, ib = lookup.get((r, a)), lookup.get((r, b))
                if ia is not None and ib is not None:
                    add_bond(ia, ib)
        for r in unique_res:  # rotatable bonds
            for a, b, kind in ROT_SPECS.get(res_of[r], ()):
                ia, ib = lookup.get((r, a)), lookup.get((r, b))
                if ia is not None and ib is not None:
                    self.rot_bonds.append(RotBond(ia, ib, BondKind[kind]))

        # 1-2 and 1-3 exclusions, each row sorted and unique (:1515-1531).
        excl = [set() for _ in range(n)]
        for bi, bj in bonds:
            excl[bi].add(bj)
        for j2 in range(n):
            nb = adj[j2]
            for i in nb:
                for k in nb:
                    if k != i:
                        lo, hi = (i, k) if i < k else (k, i)
                        excl[lo].add(hi)
        self.excl = [sorted(s) for s in excl]

        # One dihedral record per rotatable bond (:1542-1552).
        self.dihedrals = []
        for rb in self.rot_bonds:
            a_idx = next((x for x in adj[rb.i] if x != rb.j), -1)
            d_idx = next((x for x in adj[rb.j] if x != rb.i), -1)
            if a_idx < 0 or d_idx < 0:
                continue
            self.dihedrals.append(DihRecord(a_idx, rb.i, rb.j, d_idx,
                                            dihedral_terms(rb.kind, atomnames[rb.j])))

        # j-sides in compact form (the DFS-ordered lists are produced on
        # demand by the rot_bond_sides attribute).
        self._sides_dfs = None
        self._sides = _j_sides_compact(n, adj, [(rb.i, rb.j) for rb in self.rot_bonds])
        self.rot_bond_scale = [min(1.0, max(0.05, math.sqrt(LEVER_NREF / max(1.0, float(c)))))
                               for c in self._sides[2]]

        # Crankshaft pairs: phi and psi sharing a CA (:1580-1596).  The
        # reference walks an unordered_map, so its order is hash-defined;
        # here the pairs are listed by ascending phi index.
        phi_at_ca, psi_at_ca = {}, {}
        for k, rb in enumerate(self.rot_bonds):
            if rb.kind == BondKind.BACKBONE_PHI:
                phi_at_ca[rb.j] = k
            elif rb.kind == BondKind.BACKBONE_PSI:
                psi_at_ca[rb.i] = k
        self.concerted_pairs = sorted((pk, psi_at_ca[ca]) for ca, pk in phi_at_ca.items() if ca in psi_at_ca)

    @property
    def rot_bond_sides(self):
        """j_side of every rotatable bond, in the reference's DFS order."""
        if self._sides_dfs is None:
            self._sides_dfs = (_j_sides(self.N, self.adj, [(rb.i, rb.j) for rb in self.rot_bonds])
                               if self.rot_bonds else [])
        return self._sides_dfs

    def side_set(self, k):
        """Atoms of rotatable bond k's j-side as a Python set."""
        lo, hi, _, ex_ptr, ex_idx = self._sides
        out = set(range(int(lo[k]), int(hi[k])))
        out.update(ex_idx[ex_ptr[k]:ex_ptr[k + 1]].tolist())
        return out

    # ---- disulfides (:1303-1313) --------------------------------------------
    def add_disulfide(self, atom_i, atom_j):
        i, j = int(atom_i), int(atom_j)
        if i < 0 or j < 0 or i >= self.N or j >= self.N or i == j:
            return
        if i > j:
            i, j = j, i
        self._version += 1
        self.disulfide_pairs.append((i, j))
        row = self.excl[i]
        if j not in row:
            row.append(j)
            row.sort()

    # ---- concerted sidechain pairs (:1640-1673) ------------------------------
    def identify_concerted_sidechain_pairs(self, init_coords, cutoff=6.0):
        xyz = _coords(init_coords)
        self._version += 1
        self.concerted_sidechain_pairs = []
        cut2 = cutoff * cutoff
        sc = [k for k, rb in enumerate(self.rot_bonds) if rb.kind == BondKind.SIDECHAIN]
        sides = {k: self.side_set(k) for k in sc}
        out = self.concerted_sidechain_pairs
        for ia, a in enumerate(sc):
            if len(out) >= MAX_CONCERTED_SC_PAIRS:
                break
            pa = xyz[self.rot_bonds[a].j]
            for b in sc[ia + 1:]:
                if len(out) >= MAX_CONCERTED_SC_PAIRS:
                    break
                pb = xyz[self.rot_bonds[b].j]
                dx, dy, dz = pa[0] - pb[0], pa[1] - pb[1], pa[2] - pb[2]
                if dx * dx + dy * dy + dz * dz > cut2:
                    continue
                if sides[a].isdisjoint(sides[b]):
                    out.append((a, b))

    # ---- queries --------------------------------------------------------------
    def bonded(self, i, j):
        if i < 0 or i >= self.N:
            return False
        return j in self.adj[i]

    def is_excluded(self, i, j):
        if i < 0 or j < 0 or i >= self.N or j >= self.N:
            return False
        if i > j:
            i, j = j, i
        row = self.excl[i]
        k = int(np.searchsorted(row, j))
        return k < len(row) and row[k] == j

    def j_side(self, bond_i, bond_j):
        if bond_i < 0 or bond_i >= self.N or bond_j < 0 or bond_j >= self.N:
            return []
        return _j_sides(self.N, self.adj, [(bond_i, bond_j)])[0]

    # ---- flat exports (:3746-3841) ---------------------------------------------
    @property
    def rb_atom_i(self):
        return [rb.i for rb in self.rot_bonds]

    @property
    def rb_atom_j(self):
        return [rb.j for rb in self.rot_bonds]

    @property
    def rb_kind(self):
        return [int(rb.kind) for rb in self.rot_bonds]

    @property
    def dih_a(self):
        return [d.a for d in self.dihedrals]

    @property
    def dih_b(self):
        return [d.b for d in self.dihedrals]

    @property
    def dih_c(self):
        return [d.c for d in self.dihedrals]

    @property
    def dih_d(self):
        return [d.d for d in self.dihedrals]

    @property
    def dih_term_offsets(self):
        off = [0]
        for d in self.dihedrals:
            off.append(off[-1] + len(d.terms))
        return off

    @property
    def dih_term_v2(self):
        return [t[0] for d in self.dihedrals for t in d.terms]

    @property
    def dih_term_n(self):
        return [t[1] for d in self.dihedrals for t in d.terms]

    @property
    def dih_term_gamma(self):
        return [t[2] for d in self.dihedrals for t in d.terms]

    num_dihedrals = property(lambda self: len(self.dihedrals))
    num_atoms = property(lambda self: self.N)
    num_bonds = property(lambda self: len(self.bonds))
    num_rot_bonds = property(lambda self: len(self.rot_bonds))
    num_concerted_pairs = property(lambda self: len(self.concerted_pairs))
    num_disulfide_pairs = property(lambda self: len(self.disulfide_pairs))


def _coords(particles_or_xyz):
    if isinstance(particles_or_xyz, np.ndarray):
        return np.asarray(particles_or_xyz, dtype=np.float64).reshape(-1, 3)
    return np.array([(p.x, p.y, p.z) for p in particles_or_xyz], dtype=np.float64).reshape(-1, 3)


@dataclass
class FlatTopology:
    """CSR form of a topology, the engine's input (int32 atom indices)."""
    n: int
    excl_ptr: np.ndarray      # int64 [n+1]
    excl_cols: np.ndarray     # int32, j > i sorted per row
    rb_i: np.ndarray          # int32 [nrb]
    rb_j: np.ndarray          # int32 [nrb]
    rb_kind: np.ndarray       # int32 [nrb]
    rb_scale: np.ndarray      # float64 [nrb]
    side_ptr: np.ndarray      # int64 [nrb+1] explicit j-side atoms, sorted
    side_idx: np.ndarray      # int32
    side_lo: np.ndarray       # int32 [nrb] plus the atom range [lo, hi)
    side_hi: np.ndarray       # int32 [nrb]
    side_count: np.ndarray    # int64 [nrb] j-side sizes
    dih_abcd: np.ndarray      # int32 [ndih, 4]
    term_off: np.ndarray      # int32 [ndih+1]
    term_v2: np.ndarray       # float64
    term_n: np.ndarray        # int32
    term_gamma: np.ndarray    # float64
    ss: np.ndarray            # int32 [nss, 2]
    crank: np.ndarray         # int32 [ncp, 2] (phi rot-bond, psi rot-bond)
    conc_sc: np.ndarray       # int32 [ncsp, 2]

    @property
    def nrb(self):
        return int(self.rb_i.shape[0])

    @property
    def ndih(self):
        return int(self.dih_abcd.shape[0])


def _csr(rows, dtype=np.int32, sort=False):
    ptr = np.zeros(len(rows) + 1, dtype=np.int64)
    for k, r in enumerate(rows):
        ptr[k + 1] = ptr[k] + len(r)
    flat = np.empty(int(ptr[-1]), dtype=dtype)
    for k, r in enumerate(rows):
        v = np.asarray(r, dtype=dtype)
        flat[ptr[k]:ptr[k + 1]] = np.sort(v) if sort else v
    return ptr, flat


def _compact_from_lists(sides):
    """Compact form of explicit j-side lists (longest consecutive run + rest)."""
    nb = len(sides)
    lo = np.zeros(nb, np.int32)
    hi = np.zeros(nb, np.int32)
    cnt = np.zeros(nb, np.int64)
    rows = []
    for k, sd in enumerate(sides):
        v = np.sort(np.asarray(sd, dtype=np.int64))
        cnt[k] = v.size
        if v.size >= 2:
            brk = np.flatnonzero(np.diff(v) != 1)
            starts = np.concatenate(([0], brk + 1))
            ends = np.concatenate((brk + 1, [v.size]))
            r = int(np.argmax(ends - starts))
            if ends[r] - starts[r] >= 2:
                lo[k], hi[k] = v[starts[r]], v[starts[r]] + (ends[r] - starts[r])
                v = np.concatenate((v[:starts[r]], v[ends[r]:]))
        rows.append(v)
    ptr, idx = _csr(rows)
    return lo, hi, cnt, ptr, idx


def flatten(topo) -> FlatTopology:
    """CSR arrays from this module's BondTopology or the reference's.

    For this module's BondTopology the result is cached until one of its
    mutating methods runs; the reference's objects are flattened each call.
    The returned arrays are shared between calls and must not be written."""
    ver = getattr(topo, "_version", None)
    if ver is not None:
        hit = getattr(topo, "_flat", None)
        if hit is not None and hit[0] == ver:
            return hit[1]
        flat = _flatten(topo)
        for a in vars(flat).values():
            if isinstance(a, np.ndarray):
                a.flags.writeable = False
        topo._flat = (ver, flat)
        return flat
    return _flatten(topo)


def _flatten(topo) -> FlatTopology:
    n = int(topo.num_atoms)
    excl_ptr, excl_cols = _csr(list(topo.excl))
    comp = getattr(topo, "_sides", None)
    if comp is None:  # the reference's BondTopology: explicit DFS lists
        comp = _compact_from_lists(list(topo.rot_bond_sides))
    side_lo, side_hi, side_count, side_ptr, side_idx = comp
    ndih = int(topo.num_dihedrals)
    dih = np.stack([np.asarray(topo.dih_a, np.int32), np.asarray(topo.dih_b, np.int32),
                    np.asarray(topo.dih_c, np.int32), np.asarray(topo.dih_d, np.int32)],
                   axis=1) if ndih else np.zeros((0, 4), np.int32)
    ss = np.asarray(list(topo.disulfide_pairs), dtype=np.int32).reshape(-1, 2)
    crank = np.asarray(list(topo.concerted_pairs), dtype=np.int32).reshape(-1, 2)
    csp = np.asarray(list(topo.concerted_sidechain_pairs), dtype=np.int32).reshape(-1, 2)
    return FlatTopology(
        n=n, excl_ptr=excl_ptr, excl_cols=excl_cols,
        rb_i=np.asarray(topo.rb_atom_i, np.int32), rb_j=np.asarray(topo.rb_atom_j, np.int32),
        rb_kind=np.asarray(topo.rb_kind, np.int32),
        rb_scale=np.asarray(list(topo.rot_bond_scale), np.float64),
        side_ptr=np.asarray(side_ptr, np.int64), side_idx=np.asarray(side_idx, np.int32),
        side_lo=np.asarray(side_lo, np.int32), side_hi=np.asarray(side_hi, np.int32),
        side_count=np.asarray(side_count, np.int64), dih_abcd=np.ascontiguousarray(dih, np.int32),
        term_off=np.asarray(topo.dih_term_offsets, np.int32),
        term_v2=np.asarray(topo.dih_term_v2, np.float64),
        term_n=np.asarray(topo.dih_term_n, np.int32),
        term_gamma=np.asarray(topo.dih_term_gamma, np.float64),
        ss=ss, crank=crank, conc_sc=csp)

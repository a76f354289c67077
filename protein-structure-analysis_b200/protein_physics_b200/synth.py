"""Seeded synthetic all-atom chains (the benchmark inputs).

Chains are built by NeRF (natural extension reference frame) from the
internal-coordinate templates in data/residue_ic.json: backbone bond
lengths/angles, per-residue sidechain and hydrogen geometry, with phi, psi,
omega and the chi angles chosen by the caller.  Atom names follow the
reference's residue bond templates, so BondTopology.build gives the
reference exclusions / rotatable bonds.  Charges, R* and epsilon come from
data/ff_params.json (the reference's amber_params ff14SB lookup).

This module needs numpy and scipy only (no package-relative imports), so
a benchmark can load it by path to build inputs for another engine.

Workloads (residue counts and shapes of the reference's benchmark
configurations, all seeded):
  * ``chain(n_res, seed)``      — phi ~ N(-60, 15), psi ~ N(-45, 15) deg,
                                  chi from the wells {60, 180, 300} +- U(10)
  * ``compact_chain(...)``      — a coil chain collapsed in torsion space
                                  (L-BFGS over phi / psi of a soft-sphere bead
                                  model on a radius-of-gyration restraint)
  * ``coil_chain(...)``         — helix/coil phi-psi mixture
"""
from __future__ import annotations

import json
import math
import os
from dataclasses import dataclass

import numpy as np

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
with open(os.path.join(_DATA, "residue_ic.json")) as _f:
    _IC = json.load(_f)
with open(os.path.join(_DATA, "ff_params.json")) as _f:
    _FF = json.load(_f)
with open(os.path.join(_DATA, "residue_tables.json")) as _f:
    _BOND_TEMPLATES = json.load(_f)["bond_templates"]

RESIDUES = ["ALA", "ARG", "ASN", "ASP", "CYS", "GLN", "GLU", "GLY", "HID", "ILE",
            "LEU", "LYS", "MET", "PHE", "PRO", "SER", "THR", "TRP", "TYR", "VAL"]
ROTAMER_WELLS = (60.0, 180.0, 300.0)


@dataclass
class Chain:
    """A synthetic chain: particle arrays plus the topology inputs."""
    xyz: np.ndarray        # [n, 3] float64, Å
    charge: np.ndarray     # [n]
    radius: np.ndarray     # [n] R* (Å)
    epsilon: np.ndarray    # [n] kcal/mol
    resnames: list
    atomnames: list
    res_idx: list
    sequence: list

    @property
    def n(self):
        return int(self.xyz.shape[0])


def _place(a, b, c, bond, ang_deg, dih_deg):
    """Atom d with |cd| = bond, angle bcd = ang, dihedral abcd = dih (NeRF).
    Scalar arithmetic: this runs once per atom of every trial placement."""
    ang, dih = math.radians(ang_deg), math.radians(dih_deg)
    ax, ay, az = float(a[0]), float(a[1]), float(a[2])
    bx, by, bz = float(b[0]), float(b[1]), float(b[2])
    cx, cy, cz = float(c[0]), float(c[1]), float(c[2])
    ux, uy, uz = cx - bx, cy - by, cz - bz
    l = math.sqrt(ux * ux + uy * uy + uz * uz)
    ux, uy, uz = ux / l, uy / l, uz / l
    vx, vy, vz = bx - ax, by - ay, bz - az
    nx, ny, nz = vy * uz - vz * uy, vz * ux - vx * uz, vx * uy - vy * ux
    l = math.sqrt(nx * nx + ny * ny + nz * nz)
    nx, ny, nz = nx / l, ny / l, nz / l
    mx, my, mz = ny * uz - nz * uy, nz * ux - nx * uz, nx * uy - ny * ux
    d0 = -bond * math.cos(ang)
    d1 = bond * math.sin(ang) * math.cos(dih)
    d2 = bond * math.sin(ang) * math.sin(dih)
    return np.array([cx + d0 * ux + d1 * mx + d2 * nx, cy + d0 * uy + d1 * my + d2 * ny,
                     cz + d0 * uz + d1 * mz + d2 * nz])


def n_chi(resname):
    return len(_IC["residues"][resname]["chi_template"])


def _place_residue(res, N, CA, C, phi, psi, chis):
    """Positions of every template atom of one residue from its backbone."""
    T = _IC["residues"][res]
    pos = {"N": N, "CA": CA, "C": C}
    tors = {"phi": phi, "psi": psi}
    chi_t = T["chi_template"]
    for k, key in enumerate(sorted(chi_t)):
        tors[key] = float(chis[k]) if chis is not None and k < len(chis) else float(chi_t[key])
    for name, p1, p2, p3, bond, ang_deg, var, off in T["atoms"]:
        d = off + (tors[var] if var else 0.0)
        pos[name] = _place(pos[p3], pos[p2], pos[p1], bond, ang_deg, d)
    order = ["N", "CA", "C"] + [a[0] for a in T["atoms"]]
    return order, np.array([pos[nm] for nm in order])


def build(sequence, phi, psi, omega=None, chis=None):
    """NeRF build.  sequence: residue names; phi/psi/omega: degrees per
    residue; chis: per residue list of chi angles (degrees).  Returns a Chain."""
    n_res = len(sequence)
    bb = _IC["backbone"]
    omega = np.full(n_res, 180.0) if omega is None else np.asarray(omega, float)
    blocks, names, resn, ridx = [], [], [], []
    prev = None  # (N, CA, C) of the previous residue
    for r, res in enumerate(sequence):
        T = _IC["residues"][res]
        ph = float(phi[r]) if res != "PRO" else float(T["phi_template"])
        if prev is None:
            N = np.zeros(3)
            CA = np.array([bb["b_n_ca"], 0.0, 0.0])
            ang = math.radians(bb["a_n_ca_c"])
            C = CA + bb["b_ca_c"] * np.array([-math.cos(ang), math.sin(ang), 0.0])
        else:
            pN, pCA, pC = prev
            N = _place(pN, pCA, pC, bb["b_c_n"], bb["a_ca_c_n"], float(psi[r - 1]))
            CA = _place(pCA, pC, N, bb["b_n_ca"], bb["a_c_n_ca"], float(omega[r - 1]))
            C = _place(pC, N, CA, bb["b_ca_c"], bb["a_n_ca_c"], ph)
        order, P = _place_residue(res, N, CA, C, ph, float(psi[r]), chis[r] if chis is not None else None)
        blocks.append(P)
        names += order
        resn += [res] * len(order)
        ridx += [r] * len(order)
        prev = (N, CA, C)
    xyz = np.concatenate(blocks).astype(np.float64)
    q = np.empty(len(names))
    rad = np.empty(len(names))
    eps = np.empty(len(names))
    for k, (res, name) in enumerate(zip(resn, names)):
        q[k], rad[k], eps[k] = _FF["%s:%s" % (res, name)]
    ch = Chain(xyz, q, rad, eps, resn, names, ridx, list(sequence))
    ch.phi = np.array([float(phi[r]) if sequence[r] != "PRO" else float(_IC["residues"]["PRO"]["phi_template"])
                       for r in range(n_res)])
    ch.psi = np.asarray(psi, float).copy()
    ch.chis = [list(c) for c in chis] if chis is not None else None
    return ch


def _clash_pairs(ch, xyz, heavy_cut=2.2, any_cut=1.3):
    """Non-bonded close pairs (atoms >= 2 residues apart, or in the same or
    adjacent residue but not within three bonds along the residue graph is
    approximated by the residue gap test only)."""
    from scipy.spatial import cKDTree
    ridx = np.asarray(ch.res_idx)
    pairs = cKDTree(xyz).query_pairs(heavy_cut, output_type="ndarray")
    if len(pairs) == 0:
        return pairs
    i, j = pairs[:, 0], pairs[:, 1]
    far = np.abs(ridx[i] - ridx[j]) >= 2
    d = np.linalg.norm(xyz[i] - xyz[j], axis=1)
    hv = np.array([not a.startswith("H") for a in ch.atomnames])
    bad = far & ((hv[i] & hv[j]) | (d < any_cut))
    return pairs[bad]


def repack(ch, rng, passes=4):
    """Seeded greedy rotamer repacking: for residues in a clash, try every
    chi-well combination of the first three chis (others kept) and keep the
    one with the fewest clashes."""
    if ch.chis is None:
        return ch
    xyz = ch.xyz.copy()
    ridx = np.asarray(ch.res_idx)
    first = np.searchsorted(ridx, np.arange(len(ch.sequence) + 1))
    chis = [list(c) for c in ch.chis]
    for _ in range(passes):
        bad = _clash_pairs(ch, xyz)
        if len(bad) == 0:
            break
        residues = sorted(set(ridx[bad[:, 0]].tolist()) | set(ridx[bad[:, 1]].tolist()))
        for r in residues:
            res = ch.sequence[r]
            m = n_chi(res)
            if m == 0:
                continue
            a0, a1 = first[r], first[r + 1]
            N, CA, C = xyz[a0], xyz[a0 + 1], xyz[a0 + 2]
            best, best_cost = None, None
            k = min(m, 3)
            for combo in np.ndindex(*([3] * k)):
                trial = list(chis[r])
                for q in range(k):
                    trial[q] = ROTAMER_WELLS[combo[q]] + rng.uniform(-10.0, 10.0)
                _, P = _place_residue(res, N, CA, C, float(ch.phi[r]), float(ch.psi[r]), trial)
                x2 = xyz.copy()
                x2[a0:a1] = P
                sel = _clash_pairs(ch, x2)
                cost = int(np.sum((ridx[sel[:, 0]] == r) | (ridx[sel[:, 1]] == r))) if len(sel) else 0
                if best_cost is None or cost < best_cost:
                    best, best_cost, best_P = trial, cost, P
                if cost == 0:
                    break
            chis[r] = best
            xyz[a0:a1] = best_P
    out = Chain(xyz, ch.charge, ch.radius, ch.epsilon, ch.resnames, ch.atomnames, ch.res_idx, ch.sequence)
    out.phi, out.psi, out.chis = ch.phi, ch.psi, chis
    return out


def random_sequence(n_res, rng):
    return [RESIDUES[k] for k in rng.integers(0, len(RESIDUES), size=n_res)]


def _draw_chis(res, rng):
    m = n_chi(res)
    return list(rng.choice(ROTAMER_WELLS, size=m) + rng.uniform(-10.0, 10.0, size=m))


_BB_ATOMS = ("N", "CA", "C", "O", "H", "HA", "CB", "CD")  # placed from phi/psi only (CD: PRO)
_INTRA = {}


def _intra_pairs(res, order):
    """(i, j) index pairs of one residue's atoms >= 4 bonds apart (may clash)."""
    if res in _INTRA:
        return _INTRA[res]
    adj = {}
    for a, b in _BOND_TEMPLATES[res]:
        adj.setdefault(a, []).append(b)
        adj.setdefault(b, []).append(a)
    idx = {nm: k for k, nm in enumerate(order)}
    pairs = []
    for a in order:
        dist = {a: 0}
        q = [a]
        while q:
            x = q.pop(0)
            for y in adj.get(x, []):
                if y not in dist:
                    dist[y] = dist[x] + 1
                    q.append(y)
        for b in order:
            if idx[b] > idx[a] and dist.get(b, 99) >= 4:
                pairs.append((idx[a], idx[b]))
    _INTRA[res] = np.array(pairs, dtype=int).reshape(-1, 2)
    return _INTRA[res]


# Sidechain packing scores overlaps against the force field's own contact
# distance R*_i + R*_j: a pair closer than PACK_FRAC of it (C-C 2.85 Å, H-H
# 2.2 Å, O to an aliphatic H 2.4 Å) counts by its depth.  Real contacts sit
# above that (C-C >= 3.4 Å); the energy model's r^-12 term makes anything
# below it cost tens to thousands of kcal/mol.
PACK_FRAC = 0.75


def _radius(res, name):
    return float(_FF["%s:%s" % (res, name)][1])


def _intra_cost(res, order, P, heavy_cut, any_cut):
    pr = _intra_pairs(res, order)
    if len(pr) == 0:
        return 0.0
    d = np.linalg.norm(P[pr[:, 0]] - P[pr[:, 1]], axis=1)
    rad = np.array([_radius(res, nm) for nm in order])
    over = PACK_FRAC * (rad[pr[:, 0]] + rad[pr[:, 1]]) - d
    return float(np.sum(over[over > 0]))


class _Grid:
    """Uniform spatial hash for clash queries (cell = query radius); the
    points of the last residues can be taken out again (backtracking)."""

    def __init__(self, cell):
        self.cell = cell
        self.cells = {}
        self.by_res = {}  # residue -> [(cell key, x, y, z, heavy)]

    def add(self, P, hv, r, rad=None):
        ent = []
        for k in range(P.shape[0]):
            x, y, z = float(P[k][0]), float(P[k][1]), float(P[k][2])
            key = (math.floor(x / self.cell), math.floor(y / self.cell), math.floor(z / self.cell))
            item = (x, y, z, bool(hv[k]), r, float(rad[k]) if rad is not None else 0.0)
            self.cells.setdefault(key, []).append(item)
            ent.append((key, item))
        self.by_res.setdefault(r, []).extend(ent)

    def remove(self, r):
        for key, item in self.by_res.pop(r, ()):
            lst = self.cells[key]
            lst.remove(item)

    def cost(self, P, hv, r, heavy_cut, any_cut, min_gap=2, rad=None):
        """Clashes of points P (residue r) with the stored points of
        residues >= min_gap away: a count by the heavy / any cutoffs, or,
        with radii, the summed depth below PACK_FRAC (R*_i + R*_j)."""
        c = 0.0 if rad is not None else 0
        a2, h2 = any_cut * any_cut, heavy_cut * heavy_cut
        for k in range(P.shape[0]):
            x, y, z = float(P[k][0]), float(P[k][1]), float(P[k][2])
            kx, ky, kz = math.floor(x / self.cell), math.floor(y / self.cell), math.floor(z / self.cell)
            hk = bool(hv[k])
            rk = float(rad[k]) if rad is not None else 0.0
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        for (px, py, pz, ph, pr, prad) in self.cells.get((kx + dx, ky + dy, kz + dz), ()):
                            if abs(pr - r) < min_gap:
                                continue
                            d2 = (x - px) ** 2 + (y - py) ** 2 + (z - pz) ** 2
                            if rad is not None:
                                lim = PACK_FRAC * (rk + prad)
                                if d2 < lim * lim:
                                    c += lim - math.sqrt(d2)
                            elif d2 < a2 or (d2 < h2 and hk and ph):
                                c += 1
        return c


def grow(sequence, draw_phipsi, rng, tries=12, heavy_cut=2.2, any_cut=1.3, back=3, budget_per_res=30, max_back=1000000):
    """Two-phase seeded build.

    1. Backbone (N CA C O H HA CB) residue by residue: (phi, psi of the
       previous residue) are redrawn up to `tries` times while a new atom
       clashes with backbone atoms >= 2 residues away (heavy-heavy closer
       than heavy_cut, any pair closer than any_cut); when every draw
       clashes the last `back` residues are regrown (bounded budget).
    2. Sidechains, in a seeded random residue order: the drawn chis are kept
       when clash-free, otherwise every well combination of the first three
       chis is tried and the least clashing kept.
    draw_phipsi(r) -> (phi, psi) in degrees."""
    n_res = len(sequence)
    bb = _IC["backbone"]
    phi = np.zeros(n_res)
    psi = np.zeros(n_res)
    frames = [None] * n_res
    bbpos = [None] * n_res
    budget = budget_per_res * n_res + 100
    fails = np.zeros(n_res, int)

    def backbone_atoms(r, N, CA, C, ph, ps):
        order, P = _place_residue(sequence[r], N, CA, C, ph, ps, None)
        keep = [k for k, nm in enumerate(order) if nm in _BB_ATOMS and not (nm == "CD" and sequence[r] != "PRO")]
        return (P[keep], np.array([not order[k].startswith("H") for k in keep]),
                np.array([_radius(sequence[r], order[k]) for k in keep]))

    grid = _Grid(max(heavy_cut, any_cut, 2.0 * PACK_FRAC * max(v[1] for v in _FF.values())))
    grid_upto = -1
    r = 0
    while r < n_res:
        while grid_upto > max(r - 2, -1):  # backtracked: take the regrown residues out
            grid.remove(grid_upto)
            grid_upto -= 1
        while grid_upto < r - 2:
            grid_upto += 1
            grid.add(bbpos[grid_upto][0], bbpos[grid_upto][1], grid_upto, rad=bbpos[grid_upto][2])
        best = None
        for t in range(tries):
            ph, ps = draw_phipsi(r)
            if sequence[r] == "PRO":
                ph = float(_IC["residues"]["PRO"]["phi_template"])
            ps_prev = psi[r - 1] if r > 0 else 0.0
            if r > 0 and t >= tries // 2:
                ps_prev = draw_phipsi(r - 1)[1]
                if sequence[r] == "PRO":  # pre-proline residues sit in the PPII / beta basin
                    ps_prev = float(rng.normal(145.0, 15.0))
            if r == 0:
                N = np.zeros(3)
                CA = np.array([bb["b_n_ca"], 0.0, 0.0])
                ang = math.radians(bb["a_n_ca_c"])
                C = CA + bb["b_ca_c"] * np.array([-math.cos(ang), math.sin(ang), 0.0])
            else:
                pN, pCA, pC = frames[r - 1]
                N = _place(pN, pCA, pC, bb["b_c_n"], bb["a_ca_c_n"], ps_prev)
                CA = _place(pCA, pC, N, bb["b_n_ca"], bb["a_c_n_ca"], 180.0)
                C = _place(pC, N, CA, bb["b_ca_c"], bb["a_n_ca_c"], ph)
            P, hv, rad = backbone_atoms(r, N, CA, C, ph, ps)
            cost = grid.cost(P, hv, r, heavy_cut, any_cut, rad=rad) if r >= 2 else 0
            if r >= 3 and ps_prev != psi[r - 1]:  # the redrawn psi moves residue r-1's O too: check it again
                pN, pCA, pC = frames[r - 1]
                Pp, hvp, radp = backbone_atoms(r - 1, pN, pCA, pC, phi[r - 1], ps_prev)
                cost += grid.cost(Pp, hvp, r - 1, heavy_cut, any_cut, rad=radp)
            if best is None or cost < best[0]:
                best = (cost, ph, ps, ps_prev, P, hv, rad, (N, CA, C))
            if cost == 0:
                break
        cost, ph, ps, ps_prev, P, hv, rad, frame = best
        budget -= 1
        if cost > 0 and budget > 0 and r >= 2:
            fails[r] += 1
            r -= min(r - 1, back * min(int(fails[r]), max_back))
            continue
        if r > 0 and ps_prev != psi[r - 1]:
            psi[r - 1] = ps_prev
            pN, pCA, pC = frames[r - 1]
            bbpos[r - 1] = backbone_atoms(r - 1, pN, pCA, pC, phi[r - 1], ps_prev)
        phi[r], psi[r] = ph, ps
        bbpos[r], frames[r] = (P, hv, rad), frame
        r += 1
    return pack_sidechains(sequence, phi, psi, frames, bbpos, rng, heavy_cut, any_cut)


def pack_sidechains(sequence, phi, psi, frames, bbpos, rng, heavy_cut=2.2, any_cut=1.3):
    """Greedy seeded sidechain placement on a fixed backbone: in a random
    residue order, keep the drawn chis when clash-free, else try every well
    combination of the first three chis and keep the least clashing.  A
    clash is an overlap below PACK_FRAC of the force field's contact
    distance, weighed by its depth."""
    n_res = len(sequence)
    chis = [_draw_chis(res, rng) for res in sequence]
    # the contact test reaches PACK_FRAC x the largest R* pair
    grid = _Grid(max(heavy_cut, any_cut, 2.0 * PACK_FRAC * max(v[1] for v in _FF.values())))
    for rr in range(n_res):
        P0, hv0 = bbpos[rr][0], bbpos[rr][1]
        grid.add(P0, hv0, rr, rad=bbpos[rr][2] if len(bbpos[rr]) > 2 else np.full(len(P0), 1.7))
    for rr in rng.permutation(n_res):
        res = sequence[rr]
        m = n_chi(res)
        N, CA, C = frames[rr]
        order, P = _place_residue(res, N, CA, C, phi[rr], psi[rr], chis[rr])
        sc = [k for k, nm in enumerate(order) if nm not in _BB_ATOMS or (nm == "CD" and res != "PRO")]
        if not sc:
            continue
        hv = np.array([not order[k].startswith("H") for k in sc])
        rad = np.array([_radius(res, order[k]) for k in sc])
        cost = grid.cost(P[sc], hv, rr, heavy_cut, any_cut, min_gap=1, rad=rad) + \
            _intra_cost(res, order, P, heavy_cut, any_cut)
        if cost and m:
            best = (cost, chis[rr], P)
            for combo in np.ndindex(*([3] * min(m, 3))):
                trial = list(chis[rr])
                for q, w in enumerate(combo):
                    trial[q] = ROTAMER_WELLS[w] + rng.uniform(-10.0, 10.0)
                _, P2 = _place_residue(res, N, CA, C, phi[rr], psi[rr], trial)
                c2 = (grid.cost(P2[sc], hv, rr, heavy_cut, any_cut, min_gap=1, rad=rad)
                      + _intra_cost(res, order, P2, heavy_cut, any_cut))
                if c2 < best[0]:
                    best = (c2, trial, P2)
                if c2 == 0:
                    break
            chis[rr], P = best[1], best[2]
        grid.add(P[sc], hv, rr, rad=rad)
    return build(sequence, phi, psi, chis=chis)


def _chis(sequence, rng):
    return [_draw_chis(res, rng) for res in sequence]


def chain(n_res, seed, phi_mu=-60.0, psi_mu=-45.0, sd=15.0):
    """phi ~ N(phi_mu, sd), psi ~ N(psi_mu, sd), chi from rotamer wells,
    conditioned on no steric clash (seeded rejection, see grow)."""
    rng = np.random.default_rng(seed)
    seq = random_sequence(n_res, rng)
    return grow(seq, lambda r: (rng.normal(phi_mu, sd), rng.normal(psi_mu, sd)), rng)


def coil_chain(n_res, seed, helix_frac=0.5):
    """Helix/coil mixture: helical segments phi/psi ~ N(-60,-45; 10), coil
    segments from the beta / PPII basins."""
    rng = np.random.default_rng(seed)
    seq = random_sequence(n_res, rng)
    kind = np.empty(n_res, int)
    r = 0
    while r < n_res:
        seg = int(rng.integers(4, 16))
        kind[r:r + seg] = 0 if rng.random() < helix_frac else 1
        r += seg

    def draw(k):
        if kind[k] == 0:
            return rng.normal(-60, 10), rng.normal(-45, 10)
        if rng.random() < 0.5:
            return rng.normal(-120, 15), rng.normal(130, 15)
        return rng.normal(-70, 15), rng.normal(145, 15)

    return grow(seq, draw, rng)


def radius_of_gyration(xyz):
    c = xyz - xyz.mean(axis=0)
    return float(np.sqrt((c * c).sum(axis=1).mean()))


def _frames(ch):
    """(N, CA, C) per residue and the backbone-phase atoms of a built chain."""
    ridx = np.asarray(ch.res_idx)
    first = np.searchsorted(ridx, np.arange(len(ch.sequence) + 1))
    frames, bbpos = [], []
    for r, res in enumerate(ch.sequence):
        a0, a1 = first[r], first[r + 1]
        names = ch.atomnames[a0:a1]
        frames.append((ch.xyz[a0], ch.xyz[a0 + 1], ch.xyz[a0 + 2]))
        keep = [k for k, nm in enumerate(names) if nm in _BB_ATOMS and not (nm == "CD" and res != "PRO")]
        bbpos.append((ch.xyz[a0:a1][keep], np.array([not names[k].startswith("H") for k in keep]),
                      np.array([_radius(res, names[k]) for k in keep])))
    return frames, bbpos


def _wrap(deg):
    """An angle difference in degrees, wrapped to [-180, 180)."""
    return (deg + 180.0) % 360.0 - 180.0


def _torsion(a, b, c, d):
    b1, b2, b3 = b - a, c - b, d - c
    n1, n2 = np.cross(b1, b2), np.cross(b2, b3)
    return math.degrees(math.atan2(np.linalg.norm(b2) * np.dot(b1, n2), np.dot(n1, n2)))


# Heavy sidechain atoms per residue: size of the sidechain bead of the
# collapse model.
_N_SIDECHAIN = {"GLY": 0, "ALA": 1, "SER": 2, "CYS": 2, "VAL": 3, "THR": 3, "PRO": 3, "ILE": 4, "LEU": 4, "ASP": 4,
                "ASN": 4, "MET": 4, "GLU": 5, "GLN": 5, "LYS": 5, "HID": 6, "PHE": 7, "ARG": 7, "TYR": 8, "TRP": 10}


class _BeadChain:
    """Collapse model of a built chain: per residue N, CA, a sidechain bead,
    C and the carbonyl O (in that order, so every torsion moves a suffix of
    the points), each a soft sphere; the backbone phi / psi are the degrees
    of freedom (omega and the bond geometry stay as built).  The O atoms
    keep neighbouring backbone turns at hydrogen-bond distance or more
    (without them a collapse packs carbonyls into each other)."""

    PER_RES = 5

    def __init__(self, ch, radius_scale):
        n_res = len(ch.sequence)
        ridx = np.asarray(ch.res_idx)
        first = np.searchsorted(ridx, np.arange(n_res + 1))
        N, CA, C = ch.xyz[first[:-1]], ch.xyz[first[:-1] + 1], ch.xyz[first[:-1] + 2]
        names = np.asarray(ch.atomnames)
        O = np.empty_like(N)
        for r in range(n_res):
            k = np.flatnonzero(names[first[r]:first[r + 1]] == "O")
            O[r] = ch.xyz[first[r] + k[0]] if len(k) else C[r]
        nsc = np.array([_N_SIDECHAIN[r] for r in ch.sequence])
        # bead on the ideal C-beta direction, further out for larger sidechains
        b, c = CA - N, C - CA
        d = -0.58273431 * np.cross(b, c) + 0.56802827 * b - 0.54067466 * c
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        B = CA + np.minimum(1.53 + 0.45 * np.maximum(nsc - 1, 0), 4.0)[:, None] * d
        P = self.PER_RES
        self.X0 = np.stack([N, CA, B, C, O], 1).reshape(-1, 3)
        self.rad = radius_scale * np.stack([np.full(n_res, 1.6), np.full(n_res, 1.9),
                                            np.where(nsc > 0, 1.9 + 0.35 * np.sqrt(nsc), 0.0),
                                            np.full(n_res, 1.7), np.full(n_res, 1.5)], 1).reshape(-1)
        self.res = np.repeat(np.arange(n_res), P)
        self.bead = np.tile(np.arange(P) == 2, n_res)
        self.carbonyl = np.tile(np.arange(P) == 4, n_res)
        self.real = np.flatnonzero(self.rad > 0)
        tors = []
        for r in range(n_res):
            if r > 0 and ch.sequence[r] != "PRO":
                tors.append((P * r, P * r + 1, P * r + 2))  # phi about N-CA: moves the bead, C, O and beyond
            if r < n_res - 1:
                tors.append((P * r + 1, P * r + 3, P * r + 4))  # psi about CA-C: moves O and the next residues
        self.tors = np.array(tors, dtype=np.int64).reshape(-1, 3)
        self.owner = np.searchsorted(self.tors[:, 2], np.arange(self.X0.shape[0]), side="right") - 1
        # residues before a proline: psi held in the PPII / beta basin (the
        # proline's ring sits against the residue before it for other psi;
        # the bead model does not carry the ring)
        psi_k = {int(t[0]) // P: k for k, t in enumerate(self.tors) if t[2] % P == 4}
        self.prepro = [(psi_k[r], P * r, P * r + 1, P * r + 3, P * (r + 1)) for r in range(n_res - 1)
                       if ch.sequence[r + 1] == "PRO" and r in psi_k]
        self.prepro_sign = np.ones(len(self.prepro))
        if self.prepro:  # d psi / d theta of each such torsion (+1 or -1), from a small turn
            th = np.zeros(len(self.tors))
            for q, (k, a, b, c, d) in enumerate(self.prepro):
                th[k] = 1e-3
            X1 = self.coords(th)
            for q, (k, a, b, c, d) in enumerate(self.prepro):
                dpsi = _wrap(_torsion(X1[a], X1[b], X1[c], X1[d]) - _torsion(self.X0[a], self.X0[b], self.X0[c],
                                                                             self.X0[d]))
                self.prepro_sign[q] = 1.0 if dpsi > 0 else -1.0

    PREPRO_PSI, PREPRO_HALF = 140.0, 45.0  # degrees: the allowed psi band before a proline

    def prepro_terms(self, X, k_pp):
        """(energy, [(torsion, dE/dtheta)]) of the flat-bottom psi restraint
        k_pp (degrees outside the band)^2 on the residues before a proline."""
        E, out = 0.0, []
        for q, (k, a, b, c, d) in enumerate(self.prepro):
            off = _wrap(_torsion(X[a], X[b], X[c], X[d]) - self.PREPRO_PSI)
            viol = abs(off) - self.PREPRO_HALF
            if viol > 0:
                E += k_pp * viol * viol
                out.append((k, 2.0 * k_pp * viol * math.copysign(1.0, off) * self.prepro_sign[q] * 180.0 / math.pi))
        return E, out

    def coords(self, theta):
        """Points after turning torsion k by theta[k] (radians), axes as built:
        x -> T_1 o ... o T_k(p) (x), k(p) the last torsion moving point p."""
        X0, t = self.X0, self.tors
        u = X0[t[:, 1]] - X0[t[:, 0]]
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        A = X0[t[:, 0]]
        c, s = np.cos(theta), np.sin(theta)
        ux, uy, uz = u[:, 0], u[:, 1], u[:, 2]
        k1 = 1.0 - c
        R = np.empty((len(theta), 3, 3))
        R[:, 0, 0], R[:, 0, 1], R[:, 0, 2] = c + ux * ux * k1, ux * uy * k1 - uz * s, ux * uz * k1 + uy * s
        R[:, 1, 0], R[:, 1, 1], R[:, 1, 2] = uy * ux * k1 + uz * s, c + uy * uy * k1, uy * uz * k1 - ux * s
        R[:, 2, 0], R[:, 2, 1], R[:, 2, 2] = uz * ux * k1 - uy * s, uz * uy * k1 + ux * s, c + uz * uz * k1
        tk = A - np.einsum("kij,kj->ki", R, A)
        Ms = np.empty_like(R)
        ts = np.empty_like(A)
        M, tt = np.eye(3), np.zeros(3)
        for k in range(len(theta)):  # cumulative composition, outermost torsion first
            tt = M @ tk[k] + tt
            M = M @ R[k]
            Ms[k], ts[k] = M, tt
        X = X0.copy()
        sel = self.owner >= 0
        w = self.owner[sel]
        X[sel] = np.einsum("pij,pj->pi", Ms[w], X0[sel]) + ts[w]
        return X

    def energy(self, X, groups, rg_target, k_rg, k_rep):
        """k_rg sum_g (Rg_g - target)^2 over the point groups + k_rep sum
        (r_i + r_j - d)^2 over overlapping pairs two or more residues apart
        (bead pairs of neighbouring residues too); returns (E, dE/dX)."""
        from scipy.spatial import cKDTree
        g = np.zeros_like(X)
        E = 0.0
        for idx in groups:
            d = X[idx] - X[idx].mean(0)
            rg = math.sqrt((d * d).sum(1).mean())
            E += k_rg * (rg - rg_target) ** 2
            g[idx] += 2.0 * k_rg * (rg - rg_target) * d / (len(idx) * rg)
        P = X[self.real]
        pr = cKDTree(P).query_pairs(2.0 * self.rad.max(), output_type="ndarray")
        i, j = self.real[pr[:, 0]], self.real[pr[:, 1]]
        dr = np.abs(self.res[i] - self.res[j])
        keep = (dr >= 2) | ((dr == 1) & ((self.bead[i] & self.bead[j]) | (self.carbonyl[i] & self.carbonyl[j])))
        i, j = i[keep], j[keep]
        v = X[i] - X[j]
        dist = np.sqrt((v * v).sum(1))
        d0 = self.rad[i] + self.rad[j]
        m = dist < d0
        i, j, v, dist, d0 = i[m], j[m], v[m], dist[m], d0[m]
        E += k_rep * float(((d0 - dist) ** 2).sum())
        f = (-2.0 * k_rep * (d0 - dist) / np.maximum(dist, 1e-9))[:, None] * v
        np.add.at(g, i, f)
        np.add.at(g, j, -f)
        return E, g

    def torsion_grad(self, X, g):
        """dE/dtheta_k = u_k . sum over the moved suffix of (x - a_k) x g."""
        xg = np.cross(X, g)
        Sxg = np.concatenate([np.cumsum(xg[::-1], 0)[::-1], np.zeros((1, 3))])
        Sg = np.concatenate([np.cumsum(g[::-1], 0)[::-1], np.zeros((1, 3))])
        t = self.tors
        u = X[t[:, 1]] - X[t[:, 0]]
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        return (u * (Sxg[t[:, 2]] - np.cross(X[t[:, 0]], Sg[t[:, 2]]))).sum(1)


def collapse(ch: Chain, seed, rg_target, iters=6000, k_rg=5.0, k_rep=10.0, radius_scale=0.85, domains=None):
    """Seeded backbone collapse: L-BFGS over every backbone phi / psi of a
    soft-sphere bead model (N, CA, C, O and one sidechain bead per residue) on
    k_rg (Rg - rg_target)^2 plus the overlap penalty, then a rebuild from
    the resulting phi / psi and a seeded sidechain packing.  The restraint
    target sits below the Rg wanted: the overlap penalty holds the chain
    out at about the density of packed beads.  With domains = [(r0, r1),
    ...] the Rg term is one per residue range (multi-domain chains)."""
    from scipy.optimize import minimize
    rng = np.random.default_rng(seed)
    model = _BeadChain(ch, radius_scale)
    P = _BeadChain.PER_RES
    if domains:
        groups = [np.intersect1d(model.real, np.arange(P * r0, P * r1)) for r0, r1 in domains]
    else:
        groups = [model.real]

    def f(theta):
        X = model.coords(theta)
        E, g = model.energy(X, groups, rg_target, k_rg, k_rep)
        gt = model.torsion_grad(X, g)
        Ep, gp = model.prepro_terms(X, 0.05)
        for k, v in gp:
            gt[k] += v
        return E + Ep, gt

    res = minimize(f, np.zeros(len(model.tors)), jac=True, method="L-BFGS-B",
                   options={"maxiter": int(iters), "maxfun": 2 * int(iters)})
    X = model.coords(res.x).reshape(-1, P, 3)
    N, CA, C = X[:, 0], X[:, 1], X[:, 3]
    n_res = len(ch.sequence)
    phi, psi = ch.phi.copy(), ch.psi.copy()
    for r in range(n_res):
        if r > 0 and ch.sequence[r] != "PRO":
            phi[r] = _torsion(C[r - 1], N[r], CA[r], C[r])
        if r + 1 < n_res:
            psi[r] = _torsion(N[r], CA[r], C[r], N[r + 1])
    bb_only = build(ch.sequence, phi, psi, chis=ch.chis)
    frames, bbpos = _frames(bb_only)
    return pack_sidechains(ch.sequence, phi, psi, frames, bbpos, rng)


def compact_chain(n_res, seed, rg_target=None, iters=6000):
    """A coil chain collapsed by the bead model (collapse).  The default
    restraint target 0.7 * 2.2 * n_res^0.38 Å ends near the Rg of a packed
    globular protein of that length (300 residues: ~18 Å all-atom); the
    device relaxation of workloads.py then clears the remaining clashes."""
    ch = coil_chain(n_res, seed)
    if rg_target is None:
        rg_target = 0.7 * 2.2 * n_res ** 0.38
    return collapse(ch, seed + 7919, rg_target, iters=iters)


def multidomain_chain(n_domains, domain_res, linker_res, seed, iters=None):
    """n_domains compact domains of domain_res residues joined by coil
    linkers of linker_res residues: one coil chain collapsed with one Rg
    restraint per domain."""
    n_res = n_domains * domain_res + (n_domains - 1) * linker_res
    ch = coil_chain(n_res, seed)
    doms = [(d * (domain_res + linker_res), d * (domain_res + linker_res) + domain_res) for d in range(n_domains)]
    return collapse(ch, seed + 7919, 0.7 * 2.2 * domain_res ** 0.38, iters=iters or 6000, domains=doms)

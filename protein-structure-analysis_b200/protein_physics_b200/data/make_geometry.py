"""Regenerates residue_ic.json: internal-coordinate templates for the
synthetic chain builder (protein_physics_b200.synth).

    python make_geometry.py /path/to/reference

No ff14SB ideal-geometry table is available offline, so the templates are
measured on the all-atom structure the reference ships, data/1XQ8.pdb
(17 residue types, with hydrogens).  Every residue atom other than N, CA, C
is placed by NeRF from three atoms of the same residue: its parent P1 in a
BFS tree rooted at N (tree over the reference's residue bond graph,
residue_tables.json), P2 = parent of P1, P3 = parent of P2, where the
parent of CA is N and the "parent" of N is C (so atoms hung on CA or N are
placed against the N-CA-C frame).  Each atom stores its bond length, bond
angle and a dihedral written as (torsion variable, offset): atoms whose
(P2 -> P1) axis is a rotatable sidechain bond follow that chi; O follows psi;
the amide H (and PRO's CD) follow phi; everything else is a fixed
dihedral.  CYS, TRP and ARG do not occur in 1XQ8: their templates are built
here from standard textbook geometry (tetrahedral / trigonal angles, C-S
1.81 A, S-H 1.34 A, aromatic C-C 1.39 A, C-N 1.33-1.46 A) and are marked
approximate.
"""
import json
import math
import os
import sys
from collections import OrderedDict, deque

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def dihedral(a, b, c, d):
    """IUPAC torsion angle a-b-c-d in degrees (the convention NeRF uses)."""
    b1, b2, b3 = b - a, c - b, d - c
    n1, n2 = np.cross(b1, b2), np.cross(b2, b3)
    return math.degrees(math.atan2(np.linalg.norm(b2) * np.dot(b1, n2), np.dot(n1, n2)))


def angle(a, b, c):
    u, v = a - b, c - b
    return math.degrees(math.acos(np.clip(np.dot(u, v) / np.linalg.norm(u) / np.linalg.norm(v), -1, 1)))


def read_pdb(path):
    res = OrderedDict()
    for line in open(path):
        if line.startswith("ENDMDL"):
            break
        if not line.startswith("ATOM"):
            continue
        key = (line[21], int(line[22:26]))
        r = res.setdefault(key, {"name": line[17:20].strip(), "atoms": OrderedDict()})
        r["atoms"][line[12:16].strip()] = np.array([float(line[30:38]), float(line[38:46]), float(line[46:54])])
    return list(res.values())


def tree(bonds):
    """BFS parents from N over the residue graph (N, CA, C placed first)."""
    adj = {}
    for a, b in bonds:
        adj.setdefault(a, []).append(b)
        adj.setdefault(b, []).append(a)
    parent = {"N": "C", "CA": "N", "C": "CA"}
    order = ["N", "CA", "C"]
    seen = set(order)
    dq = deque(order)
    while dq:
        x = dq.popleft()
        for y in adj.get(x, []):
            if y not in seen:
                seen.add(y)
                parent[y] = x
                order.append(y)
                dq.append(y)
    return order, parent


def rot_axes(rot_specs, resname):
    out = {}
    for i, j, kind in rot_specs.get(resname, []):
        if kind == "SIDECHAIN":
            out[(i, j)] = "chi%d" % (len(out) + 1)
    return out


def template_from_instance(resname, atoms, prev_c, next_n, bonds, rot_specs):
    order, parent = tree(bonds)
    axes = rot_axes(rot_specs, resname)
    P = dict(atoms)
    P["C-"] = prev_c
    phi_t = dihedral(prev_c, P["N"], P["CA"], P["C"])
    psi_t = dihedral(P["N"], P["CA"], P["C"], next_n)
    entries, raw = [], []
    for x in order[3:]:
        if x not in P:
            continue
        p1 = parent[x]
        p2 = parent[p1]
        p3 = parent[p2] if p2 != "C" else "N"
        if p1 == "N":  # atoms on N: the N-CA-C frame
            p2, p3 = "CA", "C"
        if p1 == "CA":
            p2, p3 = "N", "C"
        raw.append((x, p1, p2, p3, dihedral(P[x], P[p1], P[p2], P[p3])))
    # a chi is the dihedral of the first heavy atom hung on its axis
    primary = {}
    for x, p1, p2, p3, d in raw:
        var = axes.get((p2, p1))
        if var and (var not in primary) and not x.startswith("H"):
            primary[var] = d
    for x, p1, p2, p3, d in raw:
        var = axes.get((p2, p1))
        if var and var not in primary:
            primary[var] = d
    for x, p1, p2, p3, d in raw:
        var, off = None, d
        if (p2, p1) in axes:
            var = axes[(p2, p1)]
            off = d - primary[var]
        elif (p1, p2, p3) == ("C", "CA", "N"):
            var, off = "psi", d - psi_t
        elif (p1, p2, p3) == ("N", "CA", "C"):
            var, off = "phi", d - phi_t
        entries.append([x, p1, p2, p3, float(np.linalg.norm(P[x] - P[p1])), angle(P[x], P[p1], P[p2]), var,
                        (off + 180.0) % 360.0 - 180.0])
    chi = {v: primary[v] for v in primary}
    return {"atoms": entries, "chi_template": chi, "phi_template": phi_t}


# --- hand-written approximate templates (standard geometry) ------------------
def _approx_cys():
    return {"approximate": True, "phi_template": -65.0, "chi_template": {"chi1": -60.0, "chi2": 180.0},
            "atoms": [
                ["H", "N", "CA", "C", 1.01, 119.0, "phi", 180.0],
                ["HA", "CA", "N", "C", 1.09, 109.5, None, -118.0],
                ["CB", "CA", "N", "C", 1.53, 110.5, None, 122.5],
                ["O", "C", "CA", "N", 1.23, 120.5, "psi", 180.0],
                ["HB2", "CB", "CA", "N", 1.09, 109.5, "chi1", 120.0],
                ["HB3", "CB", "CA", "N", 1.09, 109.5, "chi1", -120.0],
                ["SG", "CB", "CA", "N", 1.81, 114.0, "chi1", 0.0],
                ["HG", "SG", "CB", "CA", 1.34, 96.0, "chi2", 0.0]]}


def _approx_arg():
    a = {"approximate": True, "phi_template": -65.0,
         "chi_template": {"chi1": -60.0, "chi2": 180.0, "chi3": 180.0, "chi4": 180.0},
         "atoms": [
             ["H", "N", "CA", "C", 1.01, 119.0, "phi", 180.0],
             ["HA", "CA", "N", "C", 1.09, 109.5, None, -118.0],
             ["CB", "CA", "N", "C", 1.53, 110.5, None, 122.5],
             ["O", "C", "CA", "N", 1.23, 120.5, "psi", 180.0],
             ["HB2", "CB", "CA", "N", 1.09, 109.5, "chi1", 120.0],
             ["HB3", "CB", "CA", "N", 1.09, 109.5, "chi1", -120.0],
             ["CG", "CB", "CA", "N", 1.53, 114.0, "chi1", 0.0],
             ["HG2", "CG", "CB", "CA", 1.09, 109.5, "chi2", 120.0],
             ["HG3", "CG", "CB", "CA", 1.09, 109.5, "chi2", -120.0],
             ["CD", "CG", "CB", "CA", 1.53, 111.5, "chi2", 0.0],
             ["HD2", "CD", "CG", "CB", 1.09, 109.5, "chi3", 120.0],
             ["HD3", "CD", "CG", "CB", 1.09, 109.5, "chi3", -120.0],
             ["NE", "CD", "CG", "CB", 1.46, 112.0, "chi3", 0.0],
             ["HE", "NE", "CD", "CG", 1.01, 118.0, "chi4", 180.0],
             ["CZ", "NE", "CD", "CG", 1.33, 124.5, "chi4", 0.0],
             ["NH1", "CZ", "NE", "CD", 1.33, 120.0, None, 0.0],
             ["HH11", "NH1", "CZ", "NE", 1.01, 120.0, None, 0.0],
             ["HH12", "NH1", "CZ", "NE", 1.01, 120.0, None, 180.0],
             ["NH2", "CZ", "NE", "CD", 1.33, 120.0, None, 180.0],
             ["HH21", "NH2", "CZ", "NE", 1.01, 120.0, None, 0.0],
             ["HH22", "NH2", "CZ", "NE", 1.01, 120.0, None, 180.0]]}
    return a


def _approx_trp():
    # Indole: a regular pentagon (CG CD1 NE1 CE2 CD2, 108 deg) fused on
    # CE2-CD2 with a regular hexagon (CE2 CZ2 CH2 CZ3 CE3 CD2, 120 deg), all
    # planar; ring hydrogens bisect the exterior angles.
    return {"approximate": True, "phi_template": -65.0, "chi_template": {"chi1": -60.0, "chi2": 90.0},
            "atoms": [
                ["H", "N", "CA", "C", 1.01, 119.0, "phi", 180.0],
                ["HA", "CA", "N", "C", 1.09, 109.5, None, -118.0],
                ["CB", "CA", "N", "C", 1.53, 110.5, None, 122.5],
                ["O", "C", "CA", "N", 1.23, 120.5, "psi", 180.0],
                ["HB2", "CB", "CA", "N", 1.09, 109.5, "chi1", 120.0],
                ["HB3", "CB", "CA", "N", 1.09, 109.5, "chi1", -120.0],
                ["CG", "CB", "CA", "N", 1.50, 114.0, "chi1", 0.0],
                ["CD1", "CG", "CB", "CA", 1.37, 126.0, "chi2", 0.0],
                ["CD2", "CG", "CB", "CA", 1.43, 126.0, "chi2", 180.0],
                ["HD1", "CD1", "CG", "CB", 1.08, 126.0, None, 0.0],
                ["NE1", "CD1", "CG", "CB", 1.38, 108.0, None, 180.0],
                ["HE1", "NE1", "CD1", "CG", 1.01, 126.0, None, 180.0],
                ["CE2", "CD2", "CG", "CB", 1.41, 108.0, None, 180.0],
                ["CE3", "CD2", "CG", "CB", 1.40, 132.0, None, 0.0],
                ["HE3", "CE3", "CD2", "CG", 1.08, 120.0, None, 0.0],
                ["CZ2", "CE2", "CD2", "CG", 1.40, 120.0, None, 180.0],
                ["HZ2", "CZ2", "CE2", "CD2", 1.08, 120.0, None, 180.0],
                ["CZ3", "CE3", "CD2", "CG", 1.39, 120.0, None, 180.0],
                ["HZ3", "CZ3", "CE3", "CD2", 1.08, 120.0, None, 180.0],
                ["CH2", "CZ3", "CE3", "CD2", 1.40, 120.0, None, 0.0],
                ["HH2", "CH2", "CZ3", "CE3", 1.08, 120.0, None, 180.0]]}


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("ALMA_REFERENCE", "")
    if not ref or not os.path.isdir(ref):
        sys.exit("usage: %s REFERENCE_TREE (or set ALMA_REFERENCE): the reference checkout" % sys.argv[0])
    tables = json.load(open(os.path.join(HERE, "residue_tables.json")))
    bt, rs = tables["bond_templates"], tables["rot_specs"]
    residues = read_pdb(os.path.join(ref, "data", "1XQ8.pdb"))
    out, backbone = {}, {"b_n_ca": [], "b_ca_c": [], "b_c_n": [], "a_c_n_ca": [], "a_n_ca_c": [],
                         "a_ca_c_n": []}
    for k in range(1, len(residues) - 1):
        r, prev, nxt = residues[k], residues[k - 1], residues[k + 1]
        A = r["atoms"]
        if not all(x in A for x in ("N", "CA", "C")) or "C" not in prev["atoms"] or "N" not in nxt["atoms"]:
            continue
        backbone["b_n_ca"].append(np.linalg.norm(A["CA"] - A["N"]))
        backbone["b_ca_c"].append(np.linalg.norm(A["C"] - A["CA"]))
        backbone["b_c_n"].append(np.linalg.norm(nxt["atoms"]["N"] - A["C"]))
        backbone["a_c_n_ca"].append(angle(prev["atoms"]["C"], A["N"], A["CA"]))
        backbone["a_n_ca_c"].append(angle(A["N"], A["CA"], A["C"]))
        backbone["a_ca_c_n"].append(angle(A["CA"], A["C"], nxt["atoms"]["N"]))
        name = "HID" if r["name"] == "HIS" else r["name"]
        if name in out or name not in bt:
            continue
        names = {x for pair in bt[name] for x in pair}
        if not names.issubset(A.keys()):
            continue
        out[name] = template_from_instance(name, A, prev["atoms"]["C"], nxt["atoms"]["N"], bt[name], rs)
    out["CYS"] = _approx_cys()
    out["ARG"] = _approx_arg()
    out["TRP"] = _approx_trp()
    bb = {k: float(np.mean(v)) for k, v in backbone.items()}
    json.dump({"backbone": bb, "residues": out}, open(os.path.join(HERE, "residue_ic.json"), "w"), indent=0)
    print("templates:", sorted(out), "backbone:", {k: round(v, 3) for k, v in bb.items()})


if __name__ == "__main__":
    main()

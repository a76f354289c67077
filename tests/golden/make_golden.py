"""Generates the golden vectors in tests/golden/ from the reference itself.

    python tests/golden/make_golden.py [/path/to/reference]
    python tests/golden/make_golden.py --workloads [wl_c2 wl_c4 wl_c5]

Needs the reference tree (ALMA sources + data) and its compiled engine
(oracle/_ref, `make -C oracle ref`).  Every number stored here is produced
by the reference's own code: the neighbor list, Born radii, energies and
move ΔE come from oracle/_ref (the reference physics_engine.cpp compiled
from source), topology attributes from its BondTopology, atom parameters
from its python/amber_params.py.  Inputs:

  bridge     the 3-particle case of tests/bridge_test.py (no topology)
  xq8        data/1XQ8.pdb, all-atom with hydrogens (2017 atoms)
  insulin    data/SM_P01308.pdb, heavy atoms, 3 disulfides, H charges
             folded onto heavy atoms (amber_params.missing_hydrogen_charge)
  synth64    the seeded synthetic 64-residue chain (protein_physics_b200.synth)
  wl_c2/4/5  the benchmark chains in workloads/ (300-residue compact chain,
             1,000-residue globule, 4 x 1,000-residue multi-domain chain);
             inputs stay in workloads/, the golden keeps their SHA-256

PDB reading mirrors the reference parser's rules (python/gui_main.py:281-605):
first model only, water and nucleotide residues dropped, non-finite
coordinates dropped, ATOM residues numbered in encounter order and HETATM
residues from 100000, SG-SG < 2.5 Å registered as disulfides, concerted
sidechain pairs identified with the default 6 Å cutoff.  BioPython is not
available, so the file is read by fixed columns (first altloc kept).
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "protein-structure-analysis_b200"))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def read_pdb(path, ap):
    water = {"HOH", "WAT", "H2O", "TIP", "TIP3", "SOL"}
    nucleo = {"DA", "DC", "DG", "DT", "DI", "A", "C", "G", "U", "I"}
    recs = []
    seen_model = False
    for line in open(path):
        if line.startswith("MODEL"):
            if seen_model:
                break
            seen_model = True
        if line.startswith("ENDMDL"):
            break
        if not (line.startswith("ATOM") or line.startswith("HETATM")):
            continue
        if line[16] not in (" ", "A", "1"):
            continue
        het = line.startswith("HETATM")
        res = line[17:20].strip()
        if (het and res in water) or res in nucleo:
            continue
        try:
            xyz = (float(line[30:38]), float(line[38:46]), float(line[46:54]))
        except ValueError:
            continue
        if not np.all(np.isfinite(xyz)):
            continue
        recs.append(dict(het=het, name=line[12:16].strip(), res=res, key=(line[21], int(line[22:26]), line[26]),
                         xyz=xyz))
    rmap, resn, atn, ridx = {}, [], [], []
    for r in recs:
        if r["key"] not in rmap:
            rmap[r["key"]] = len(rmap) if not r["het"] else 100000 + len(rmap)
        resn.append(r["res"])
        atn.append(r["name"])
        ridx.append(rmap[r["key"]])
    q, rad, eps = np.zeros(len(recs)), np.zeros(len(recs)), np.zeros(len(recs))
    for k, r in enumerate(recs):
        q[k], rad[k], eps[k] = ap.get_atom_params(r["res"], r["name"])
    names_of = {}
    for ri, an in zip(ridx, atn):
        names_of.setdefault(ri, set()).add(an)
    for k in range(len(recs)):
        extra = ap.missing_hydrogen_charge(resn[k], atn[k], names_of[ridx[k]])
        if extra:
            q[k] += extra
    xyz = np.array([r["xyz"] for r in recs], dtype=np.float64)
    sg = [k for k, r in enumerate(recs) if not r["het"] and r["res"] == "CYS" and r["name"] == "SG"]
    ss = []
    for a in range(len(sg)):
        for b in range(a + 1, len(sg)):
            d = xyz[sg[a]] - xyz[sg[b]]
            if float(d @ d) < 6.25:
                ss.append((sg[a], sg[b]))
    return dict(xyz=xyz, q=q, r=rad, eps=eps, resnames=resn, atomnames=atn, res_idx=ridx, ss=ss)


def topo_record(pp, sysd):
    T = pp.BondTopology()
    T.build(sysd["resnames"], sysd["atomnames"], sysd["res_idx"])
    for i, j in sysd["ss"]:
        T.add_disulfide(int(i), int(j))
    parts = [pp.Particle(*map(float, x), 0.0) for x in sysd["xyz"]]
    T.identify_concerted_sidechain_pairs(parts)
    excl_rows = [list(e) for e in T.excl]
    excl_cnt = np.array([len(e) for e in excl_rows], np.int64)
    excl_flat = np.array([j for e in excl_rows for j in e], np.int32)
    if len(sysd["xyz"]) < 20000:
        sides = [list(s) for s in T.rot_bond_sides]
        side_cnt = np.array([len(s) for s in sides], np.int64)
        side_flat = np.array([j for s in sides for j in s], np.int32)
    else:  # ~10^8 side entries: counts only (the DFS lists would not fit in Python lists)
        side_cnt = np.array([T.j_side(rb.i, rb.j).__len__() for rb in T.rot_bonds], np.int64)
        side_flat = None
    return T, dict(
        excl_cnt=excl_cnt, excl_sha=sha(excl_flat),
        rb=np.array([(rb.i, rb.j, int(rb.kind)) for rb in T.rot_bonds], np.int32).reshape(-1, 3),
        side_cnt=side_cnt, side_sha=sha(side_flat) if side_flat is not None else "",
        rot_bond_scale=np.array(list(T.rot_bond_scale)),
        dih=np.stack([T.dih_a, T.dih_b, T.dih_c, T.dih_d], 1).astype(np.int32) if T.num_dihedrals else
        np.zeros((0, 4), np.int32),
        dih_term_offsets=np.array(T.dih_term_offsets, np.int32), dih_term_v2=np.array(T.dih_term_v2),
        dih_term_n=np.array(T.dih_term_n, np.int32), dih_term_gamma=np.array(T.dih_term_gamma),
        crank=np.array(sorted(tuple(c) for c in T.concerted_pairs), np.int32).reshape(-1, 2),
        conc_sc=np.array([tuple(c) for c in T.concerted_sidechain_pairs], np.int32).reshape(-1, 2),
        ss=np.array(list(T.disulfide_pairs), np.int32).reshape(-1, 2))


def golden_system(name, sysd, R, pp, rng, n_torsion=24, n_crank=8, full_nl=False, inputs=True, fixture=None,
                  n_policy=0):
    from oracle import RefEngine  # noqa: F401
    out = {}
    T, trec = topo_record(pp, sysd)
    out.update({"topo_" + k: v for k, v in trec.items()})
    x, q, r, e = sysd["xyz"], sysd["q"], sysd["r"], sysd["eps"]
    ptr, cols = R.nl(x)
    out["nl_row_cnt"] = np.diff(ptr).astype(np.int32)
    out["nl_sha"] = sha(cols.astype(np.int32))
    if full_nl:
        out["nl_cols"] = cols.astype(np.int32)
    out["born"] = R.born_radii(x, q, r, e)
    rt = R.topology(sysd["resnames"], sysd["atomnames"], sysd["res_idx"], sysd["ss"], x)
    out["energy_topo"] = R.energy(x, q, r, e, rt)
    out["energy_notopo"] = R.energy(x, q, r, e, None)
    moves = []
    nrb = trec["rb"].shape[0]
    ncp = trec["crank"].shape[0]
    # crank pairs in the reference's own order (its unordered_map walk)
    ref_crank = [tuple(c) for c in T.concerted_pairs]
    for _ in range(n_torsion):
        k = int(rng.integers(0, nrb))
        d = float(rng.uniform(-0.5236, 0.5236))
        dE, terms, _, _ = R.move_dE(x, q, r, e, rt, 0, k, d)
        moves.append((0, k, d, dE, *terms))
    # moves of the size the samplers propose (generate_ensemble's first
    # max_angle, 0.12 rad, x the lever scale, x2.5 for sidechain bonds)
    for _ in range(n_policy):
        k = int(rng.integers(0, nrb))
        lim = 0.12 * float(trec["rot_bond_scale"][k]) * (2.5 if int(trec["rb"][k, 2]) == 2 else 1.0)
        d = float(rng.uniform(-lim, lim))
        dE, terms, _, _ = R.move_dE(x, q, r, e, rt, 0, k, d)
        moves.append((0, k, d, dE, *terms))
    for _ in range(n_crank if ncp else 0):
        kref = int(rng.integers(0, ncp))
        d = float(rng.uniform(-0.2, 0.2))
        dE, terms, _, _ = R.move_dE(x, q, r, e, rt, 1, kref, d)
        # store the pair itself (phi, psi rot-bond indices), not the index
        phi_k, psi_k = ref_crank[kref]
        moves.append((1, phi_k * 100000 + psi_k, d, dE, *terms))
    out["moves"] = np.array(moves, dtype=np.float64).reshape(-1, 8)
    out["ss_in"] = np.array(sysd["ss"], np.int32).reshape(-1, 2)
    if not inputs:
        out["fixture"] = np.array(fixture)
        out["xyz_sha"] = np.array(sha(np.asarray(x, np.float64)))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, "atoms", x.shape[0], "pairs", int(out["nl_row_cnt"].sum()), "E", out["energy_topo"][4])
        return
    out["xyz"], out["q"], out["r"], out["eps"] = x, q, r, e
    meta = dict(resnames=list(sysd["resnames"]), atomnames=list(sysd["atomnames"]),
                res_idx=[int(v) for v in sysd["res_idx"]])
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    with open(os.path.join(HERE, name + ".names.json"), "w") as f:
        json.dump(meta, f)
    print(name, "atoms", x.shape[0], "pairs", len(cols), "E", out["energy_topo"][4])


WORKLOAD_FIXTURES = {"wl_c2": "c2_chain_300res.npz", "wl_c4": "c4_globule_1000res.npz",
                     "wl_c5": "c5_multidomain_4x1000res.npz"}


def workload_goldens(R, pp, names=None):
    """Goldens of the benchmark chains (workloads/*.npz, written by
    workloads/make_workloads.py): the same reference outputs as for the
    other systems, without a copy of the inputs (the tests read them from
    the fixture) and with 16 torsion moves of up to 30 degrees, 16 of the
    samplers' own size and 8 crankshaft replays."""
    rng = np.random.default_rng(20261204)
    for name, fname in WORKLOAD_FIXTURES.items():
        if names and name not in names:
            continue
        path = os.path.join(ROOT, "workloads", fname)
        if not os.path.exists(path):
            print("skip", name, "(no", fname + ")")
            continue
        d = np.load(path, allow_pickle=False)
        sysd = dict(xyz=d["xyz"].astype(np.float64), q=d["charge"], r=d["radius"], eps=d["epsilon"],
                    resnames=[str(v) for v in d["resnames"]], atomnames=[str(v) for v in d["atomnames"]],
                    res_idx=[int(v) for v in d["res_idx"]], ss=[])
        golden_system(name, sysd, R, pp, rng, n_torsion=16, n_crank=8, inputs=False, fixture=fname, n_policy=16)


def main():
    if len(sys.argv) > 1 and sys.argv[1] == "--workloads":
        from oracle import RefEngine, ref_so_path
        sys.path.insert(0, os.path.dirname(ref_so_path()))
        import protein_physics as pp
        workload_goldens(RefEngine(), pp, sys.argv[2:])
        return
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("ALMA_REFERENCE", "")
    if not ref or not os.path.isdir(ref):
        sys.exit("usage: %s REFERENCE_TREE (or set ALMA_REFERENCE): the reference checkout" % sys.argv[0])
    sys.path.insert(0, os.path.join(ref, "python"))
    import amber_params as ap
    from oracle import RefEngine, ref_so_path
    sys.path.insert(0, os.path.dirname(ref_so_path()))
    import protein_physics as pp
    R = RefEngine()
    rng = np.random.default_rng(20261203)
    # bridge_test.py: three particles, defaults R*=1.9, eps=0.1, no topology
    P = [pp.Particle(0.0, 0.0, 0.0, 1.0), pp.Particle(5.0, 0.0, 0.0, -1.0), pp.Particle(10.0, 0.0, 0.0, 0.5)]
    e3 = pp.PhysicsEngine().calculate_potential(P)
    with open(os.path.join(HERE, "bridge.json"), "w") as f:
        json.dump({"xyz": [[0, 0, 0], [5, 0, 0], [10, 0, 0]], "q": [1.0, -1.0, 0.5], "radius": 1.9, "epsilon": 0.1,
                   "energy": e3}, f)
    print("bridge", repr(e3))
    golden_system("xq8", read_pdb(os.path.join(ref, "data", "1XQ8.pdb"), ap), R, pp, rng)
    golden_system("insulin", read_pdb(os.path.join(ref, "data", "SM_P01308.pdb"), ap), R, pp, rng)
    from protein_physics_b200 import synth
    ch = synth.chain(64, 1)
    sysd = dict(xyz=ch.xyz, q=ch.charge, r=ch.radius, eps=ch.epsilon, resnames=ch.resnames, atomnames=ch.atomnames,
                res_idx=ch.res_idx, ss=[])
    golden_system("synth64", sysd, R, pp, rng, full_nl=True)


if __name__ == "__main__":
    main()

"""Generates the compact-chain inputs of the benchmark configurations.

    python workloads/make_workloads.py [--only c2,c4] [--cache DIR] [--out DIR]

c2: a 300-residue chain (seed 2) collapsed to an all-atom radius of
    gyration near 17 Å: coil chain -> bead-model collapse on the host
    (synth.compact_chain) -> device relaxation with the full energy plus
    an Rg restraint toward 17 Å (descent, then 2,000 Metropolis moves at
    300 K; protein_physics_b200.workloads.relax).
c4: a 1,000-residue globule (seed 4), the same steps with the restraint at
    17 Å x (1000 / 300)^0.38 (the same compaction relative to the Rg of a
    folded protein of that length, 2.2 N^0.38 Å).
c5: four 1,000-residue domains joined by 10-residue coil linkers (seed 11),
    one Rg restraint per domain at the c4 target.

Writes <out>/c2_chain_300res.npz, c4_globule_1000res.npz and
c5_multidomain_4x1000res.npz (plain
arrays: coordinates, parameters, names; numpy alone reads them) and prints
one JSON line per chain with what the relaxation did.  The host collapse
is cached in --cache (the slow part on a laptop-class CPU); the device
relaxation needs one GPU.
"""
import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "protein-structure-analysis_b200"))

SPECS = {
    "c2": dict(n_res=300, seed=2, rg=17.0, file="c2_chain_300res.npz"),
    "c4": dict(n_res=1000, seed=4, rg=17.0 * (1000 / 300) ** 0.38, file="c4_globule_1000res.npz"),
    "c5": dict(n_res=4030, seed=11, rg=17.0 * (1000 / 300) ** 0.38, file="c5_multidomain_4x1000res.npz",
               domains=[(d * 1010, d * 1010 + 1000) for d in range(4)]),
}


def collapsed(name, cache):
    from protein_physics_b200 import synth, workloads
    spec = SPECS[name]
    path = os.path.join(cache, "%s_collapsed.npz" % name) if cache else None
    if path and os.path.exists(path):
        return workloads.load_chain(path)
    if "domains" in spec:
        ch = synth.multidomain_chain(4, 1000, 10, spec["seed"])
    else:
        ch = synth.compact_chain(spec["n_res"], spec["seed"])
    if path:
        os.makedirs(cache, exist_ok=True)
        workloads.save_chain(path, ch)
    return ch


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default="c2,c4")
    ap.add_argument("--cache", default="")
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--host-only", action="store_true", help="run the host collapse into --cache and stop")
    ap.add_argument("--k-rg", type=float, default=200.0)
    a = ap.parse_args()
    for name in a.only.split(","):
        t0 = time.time()
        ch = collapsed(name, a.cache)
        t1 = time.time()
        if a.host_only:
            print(json.dumps({"chain": name, "atoms": ch.n, "host_collapse_s": round(t1 - t0, 1)}))
            continue
        from protein_physics_b200 import synth, workloads
        spec = SPECS[name]
        out, info = workloads.relax(ch, spec["rg"], k_rg=a.k_rg, seed=spec["seed"], domains=spec.get("domains"))
        info.update(chain=name, atoms=out.n, rg_all_atom=synth.radius_of_gyration(out.xyz),
                    clashes=int(len(synth._clash_pairs(out, out.xyz))), host_collapse_s=round(t1 - t0, 1),
                    relax_s=round(time.time() - t1, 1), k_rg=a.k_rg, rg_target=spec["rg"])
        workloads.save_chain(os.path.join(a.out, spec["file"]), out, rg_target=spec["rg"], seed=spec["seed"])
        print(json.dumps(info))


if __name__ == "__main__":
    main()

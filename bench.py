"""Benchmark: Metropolis proposals/s of the B200 engine (and of the reference).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload single|batched|globule|replica]

Workload "single" (default): one synthetic 300-residue compact chain
(~4,700 atoms, all-atom with hydrogens, seeded), torsion moves restricted to
bonds whose j-side holds <= 25 % of the atoms, 300 K (0.5962 kcal/mol), the
reference's adaptive step (cur_max, lever scale, 2.5x sidechain), neighbor
list 12 Å + 2 Å skin rebuilt on drift, FP32 pair terms with FP64 ΔE and
Metropolis test.  One step = 1,000 proposals followed by a full energy
recomputation (Born radii + energy).
Workload "batched": 256 chains, 50-600 residues each (per-chain seeds),
temperatures geometric over 280-400 K, one step = 100 proposals per chain.
Workload "globule": a 1,000-residue chain: energy+force evals/s, 500
torsion-space descent steps, then MALA proposals/s.
Workload "replica": 16 replicas of a 4 x 1,000-residue chain, MALA:torsion
1:3, replica exchange every 100 sweeps.

value  = proposals/s of the whole job on the device (CUDA events, inputs
         resident), max over ranks;
e2e    = the same metric through the public API (PhysicsEngine.
         generate_ensemble with host particle lists: host->device copy, list
         build, MC, device->host copy of the final coordinates every step).
Multi-GPU: every rank runs its own independent chain(s) (replicas; no
data-path collective); value sums the proposals of all ranks.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "protein-structure-analysis_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

KB = 0.0019872  # kcal/mol/K
FP32_PEAK_NOMINAL = 148 * 128 * 2 * 1.965e9  # ops/s: SMs x FP32 lanes x FMA x max SM clock
OPS_PAIR, OPS_HCT, OPS_SASA = 47.0, 21.0, 11.0  # algorithmic ops per unit (FP32 + MUFU)


def rank_info():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


class ClockSampler:
    """nvidia-smi clocks / throttle reasons every 200 ms during the timed region."""

    def __init__(self, gpu):
        self.gpu, self.rows, self.proc = gpu, [], None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=5)

    def summary(self):
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if r[3 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def _coil_chain(n_res, seed):
    sys.path.insert(0, os.path.join(ROOT, "protein-structure-analysis_b200"))
    from protein_physics_b200 import synth
    return synth.coil_chain(n_res, seed)


def host_threads():
    """Host threads available to this process (what the reference's OpenMP
    engine uses: OMP_NUM_THREADS when set, else the CPUs this process may run
    on)."""
    env = os.environ.get("OMP_NUM_THREADS", "")
    if env.strip().isdigit() and int(env) > 0:
        return int(env)
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def make_workload(kind, rank, n_chains=256):
    from protein_physics_b200 import synth
    from protein_physics_b200.dist import rank_seed
    from protein_physics_b200.topology import BondTopology, flatten
    if kind == "single":
        chains = [synth.compact_chain(300, seed=rank_seed(2, rank))]
        temps = [300.0 * KB]
    else:
        import multiprocessing as mp
        import numpy as np
        rng = np.random.default_rng(rank_seed(3, rank))
        sizes = rng.integers(50, 601, size=256)[:n_chains]
        jobs = [(int(n), rank_seed(k, rank)) for k, n in enumerate(sizes)]
        # chain generation is host Python: spread it over the host cores
        with mp.get_context("spawn").Pool(min(32, os.cpu_count() or 1)) as pool:
            chains = pool.starmap(_coil_chain, jobs, chunksize=1)
        temps = list(280.0 * (400.0 / 280.0) ** (np.arange(256) / 255.0) * KB)[:n_chains]
    systems, movesets, topos = [], [], []
    for ch in chains:
        T = BondTopology()
        T.build(ch.resnames, ch.atomnames, ch.res_idx)
        F = flatten(T)
        systems.append((ch.xyz, ch.charge, ch.radius, ch.epsilon, F))
        movesets.append([k for k in range(F.nrb) if F.side_count[k] <= 0.25 * F.n])
        topos.append(T)
    return chains, systems, movesets, temps, topos


def run_ours(args, rank, world, local):
    import numpy as np
    import torch
    from protein_physics_b200 import _lib
    from protein_physics_b200.device import DeviceBatch
    from protein_physics_b200.mc import MCRunner
    torch.cuda.set_device(local)
    if world > 1:
        from protein_physics_b200.dist import init
        init("nccl", timeout_s=120)
    chains, systems, movesets, temps, topos = make_workload(args.workload, rank)
    per_step = 1000 if args.workload == "single" else 100
    batch = DeviceBatch(systems, precision="mixed")
    from protein_physics_b200.mc import autotune
    if args.config:
        tuned = tuple(int(v) for v in args.config.split(","))
    else:
        tuned = autotune(batch, temps, seed=777, policy=2, moveset=movesets,
                         proposals=1000 if args.workload == "single" else 30)
    tuned = (tuple(tuned) + (1,))[:3]
    runner = MCRunner(batch, temps, seed=12345 + rank, policy=2, cur_max0=0.12, moveset=movesets,
                      cluster_size=tuned[0], threads=tuned[1], spec_teams=tuned[2])
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()

    def step():
        runner.run(per_step)
        runner.reset_energy()  # full energy recomputation every per_step proposals

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    ctr0 = batch.move_counters().astype(np.float64)
    st0 = runner.state()
    launches0 = _lib.lib().alma_launch_count()
    rebuild0 = runner.rebuilds
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(local)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    t_wall0 = time.perf_counter()
    with sampler:
        ev0.record(stream)
        for _ in range(args.steps):
            flush.fill_(1.0)  # L2 flush between steps (256 MiB write)
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    t_wall = time.perf_counter() - t_wall0
    ms = ev0.elapsed_time(ev1)
    st1 = runner.state()
    ctr1 = batch.move_counters().astype(np.float64)
    launches = _lib.lib().alma_launch_count() - launches0 + args.steps  # + the flush fills
    proposals = float(np.sum(st1["step"] - st0["step"]))
    accepted = float(np.sum(st1["n_accepted"] - st0["n_accepted"]))
    # mc kernel time alone (roofline): time one extra chunk without rebuilds
    dctr = (ctr1 - ctr0).sum(axis=0)
    ops = dctr[0] * OPS_PAIR + dctr[1] * OPS_HCT + dctr[2] * OPS_SASA
    from protein_physics_b200.dist import reduce_timing
    ms_max, prop_total = reduce_timing(ms, proposals, device="cuda")
    # isolated MC-kernel timing for the roofline: chunk without host rebuild logic
    ke0, ke1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0 = batch.move_counters().astype(np.float64).sum(axis=0)
    lim = int(runner.state()["step"].max()) + 200
    ke0.record(stream)
    runner.launch(lim)
    ke1.record(stream)
    torch.cuda.synchronize()
    k_ms = ke0.elapsed_time(ke1)
    c1 = batch.move_counters().astype(np.float64).sum(axis=0)
    k_ops = (c1 - c0)[0] * OPS_PAIR + (c1 - c0)[1] * OPS_HCT + (c1 - c0)[2] * OPS_SASA
    achieved = k_ops / (k_ms * 1e-3)
    # e2e through the public API: generate_ensemble from host particle lists
    from protein_physics_b200 import Particle, PhysicsEngine
    eng = PhysicsEngine(precision="mixed", seed=99 + rank)
    e2e_val = None
    h2d = d2h = 0
    e2e_single = None
    if args.workload == "single":
        ch = chains[0]
        P0 = [Particle(*x, q, r, e) for x, q, r, e in zip(ch.xyz, ch.charge, ch.radius, ch.epsilon)]
        n_e2e = max(1, args.steps // 2)

        def e2e_rate(ncand):
            P = P0
            eng.generate_ensemble(P, topos[0], ncand, 50)  # warm
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(n_e2e):
                P = eng.generate_ensemble(P, topos[0], ncand, per_step)[0]
            e1.record(stream)
            torch.cuda.synchronize()
            return n_e2e * ncand * per_step / (e0.elapsed_time(e1) * 1e-3) * world

        # the call the reference arm times: as many candidates as the host has
        # threads (its OpenMP spans candidates), per_step proposals each
        ncand = host_threads()
        e2e_val = e2e_rate(ncand)
        e2e_single = e2e_rate(1)
        h2d = ncand * ch.n * 8 * 3 + ch.n * 8 * 3  # coordinates per candidate + charge, radius, epsilon
        d2h = ncand * ch.n * 8 * 3
    clocks = sampler.summary()
    de_err = de_error_vs_fp64(systems[0], movesets[0], runner.state()["cur_max"][0]) if rank == 0 else None
    out = None
    if rank == 0:
        value = prop_total / (ms_max * 1e-3)
        cpu = cpu_baseline(chains[0], topos[0], temps[0], args) if world == 1 else None
        plain = plain_gpu_baseline(chains[0], temps[0]) if (world == 1 and args.workload == "single") else None
        ef = energy_force_rate(systems[0], topos[0])
        out = {
            "metric": "Metropolis proposals/s", "value": value, "unit": "proposals/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 pair terms, f64 dE",
            "data": "synthetic (seeded NeRF chains, ff14SB parameters from the reference tables)",
            "config": {"workload": ("single chain, 300 residues compact, %d atoms, torsion moves with j-side <= 25%%"
                                    " of atoms, T=300 K, 1000 proposals + full energy per step" % chains[0].n)
                       if args.workload == "single" else
                       "256 chains x 50-600 residues (%d atoms), T 280-400 K, 100 proposals/chain per step"
                       % sum(c.n for c in chains),
                       "atoms": sum(c.n for c in chains),
                       "rg_A": round(__import__("protein_physics_b200.synth", fromlist=["x"]).radius_of_gyration(
                           chains[0].xyz), 1),
                       "accept_rate": accepted / max(1.0, proposals), "nl_rebuilds": runner.rebuilds - rebuild0,
                       "l2": "flushed between steps (256 MiB write)", "parallelism": "replicas" if world > 1 else "1 GPU"},
            "clocks": clocks,
            "gpu_launches": int(launches),
            "dE_error_vs_fp64": de_err,
            "tuned": {"cluster_size": tuned[0], "threads_per_system": tuned[1], "spec_teams": tuned[2]},
            "wall_s": t_wall,
            "e2e": {"value": e2e_val, "unit": "proposals/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "candidates": host_threads() if args.workload == "single" else None,
                    "single_candidate": e2e_single,
                    "api": "PhysicsEngine.generate_ensemble(host particles, topology, n_candidates, 1000), "
                           "n_candidates = the host threads, the call the reference arm times; single_candidate: "
                           "the same with 1 candidate",
                    "workload": "the reference's own move policy (25 % crankshaft, every rotatable bond), as the "
                                "reference arm runs it: heavier moves and more list rebuilds than the timed value"},
            "roofline": {"bound": "fp32", "kernel": ("mc_spec_kernel<float,%d,%d> x %d teams" % (tuned[1], tuned[0], tuned[2])
                                                    if tuned[2] > 1 else "mc_kernel<float,%d,%d>" % (tuned[1], tuned[0])),
                         "achieved": achieved / 1e12,
                         "peak": FP32_PEAK_NOMINAL / 1e12, "unit": "TOP/s (FP32+MUFU ops)",
                         "frac": achieved / FP32_PEAK_NOMINAL,
                         "peak_source": "nominal 148 SM x 128 FP32 lanes x 2 x 1965 MHz (no measured FP32 peak "
                                        "in MEASURED_PEAKS.json; the kernel is neither HBM- nor tensor-bound)",
                         "work_per_launch": {"pair_terms": float((c1 - c0)[0]), "hct": float((c1 - c0)[1]),
                                             "sasa_visits": float((c1 - c0)[2]), "proposals": 200},
                         "kernel_ms": k_ms, "traffic": None},
            "cpu_baseline": cpu,
            "plain_gpu_path": plain,
            "energy_force": ef,
        }
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return out


def de_error_vs_fp64(system, moveset, cur_max, n=256):
    """|ΔE(mixed) - ΔE(fp64)| over n seeded torsion proposals on the bench
    chain (same state, same moves; the device FP64 path matches the
    reference to 1e-7 kcal/mol)."""
    import numpy as np
    from protein_physics_b200.device import DeviceBatch
    rng = np.random.default_rng(4242)
    bm = DeviceBatch([system], precision="mixed")
    bf = DeviceBatch([system], precision="fp64")
    for b in (bm, bf):
        b.build_nl()
        b.born_radii()
    errs, mags = [], []
    F = system[4]
    for _ in range(n):
        k = int(moveset[rng.integers(0, len(moveset))])
        base = cur_max * (1.0 if F.rb_kind[k] in (0, 1) else 2.5) * F.rb_scale[k]
        d = float(rng.uniform(-base, base))
        em, _ = bm.move_dE([0], [k], [[d, 0.0]])
        ef, _ = bf.move_dE([0], [k], [[d, 0.0]])
        em, ef = float(em[0]), float(ef[0])
        errs.append(abs(em - ef))
        mags.append(abs(ef))
    errs = np.array(errs)
    return {"max": float(errs.max()), "p99": float(np.percentile(errs, 99)), "median": float(np.median(errs)),
            "n_moves": n, "median_abs_dE": float(np.median(mags)), "unit": "kcal/mol"}


def cpu_baseline(ch, topo, T, args, budget_s=12.0):
    """The reference engine (oracle/_ref, compiled from the reference sources)
    timed on the host: generate_ensemble on the same chain, one candidate."""
    import glob
    hits = glob.glob(os.path.join(ROOT, "oracle", "_ref", "protein_physics*.so"))
    if not hits:
        return {"value": None, "unit": "proposals/s", "cores": 0, "kind": "reference",
                "sample": "unavailable: oracle/_ref not built"}
    sys.path.insert(0, os.path.dirname(hits[0]))
    import protein_physics as pp
    R = pp.BondTopology()
    R.build(ch.resnames, ch.atomnames, ch.res_idx)
    P = [pp.Particle(*map(float, x), float(q), float(r), float(e)) for x, q, r, e in
         zip(ch.xyz, ch.charge, ch.radius, ch.epsilon)]
    eng = pp.PhysicsEngine()
    t0 = time.perf_counter()
    eng.generate_ensemble(P, R, 1, 5, T, 0.12)
    dt5 = max(1e-3, time.perf_counter() - t0)
    n = max(10, int(budget_s / dt5 * 5))
    t0 = time.perf_counter()
    eng.generate_ensemble(P, R, 1, n, T, 0.12)
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": "proposals/s", "cores": 1, "kind": "reference",
            "sample": f"reference generate_ensemble(chain of {ch.n} atoms, 1 candidate, {n} proposals) in "
                      f"{dt:.1f} s; one chain runs on one thread (OpenMP spans candidates)"}


def plain_gpu_baseline(ch, T, budget_s=8.0):
    """The reference's own plain GPU path (src/physics_engine_cuda.cu built
    unmodified for sm_100a into oracle/_ref): generate_ensemble on the same
    chain, one candidate, on this GPU."""
    import glob
    hits = glob.glob(os.path.join(ROOT, "oracle", "_ref", "protein_physics_cuda*.so"))
    cpu = glob.glob(os.path.join(ROOT, "oracle", "_ref", "protein_physics.*so"))
    if not hits or not cpu:
        return {"value": None, "unit": "proposals/s", "unavailable": "oracle/_ref/protein_physics_cuda not built"}
    sys.path.insert(0, os.path.dirname(hits[0]))
    import protein_physics as pp
    import protein_physics_cuda as pc
    R = pp.BondTopology()
    R.build(ch.resnames, ch.atomnames, ch.res_idx)
    P = [pc.Particle(*map(float, x), float(q), float(r), float(e)) for x, q, r, e in
         zip(ch.xyz, ch.charge, ch.radius, ch.epsilon)]
    eng = pc.PhysicsEngine()
    t0 = time.perf_counter()
    eng.generate_ensemble(P, R, 1, 5, T, 0.12)
    dt5 = max(1e-3, time.perf_counter() - t0)
    n = max(10, int(budget_s / dt5 * 5))
    t0 = time.perf_counter()
    eng.generate_ensemble(P, R, 1, n, T, 0.12)
    dt = time.perf_counter() - t0
    # its full-energy path (the reference has no forces): calculate_potential
    eng.calculate_potential(P, R)
    t0 = time.perf_counter()
    ne = 0
    while time.perf_counter() - t0 < 2.0 or ne < 3:
        eng.calculate_potential(P, R)
        ne += 1
    de = time.perf_counter() - t0
    return {"value": n / dt, "unit": "proposals/s", "proposals": n, "seconds": dt,
            "what": "reference protein_physics_cuda.generate_ensemble(chain, 1 candidate) on this B200 "
                    "(physics_engine_cuda.cu built unmodified for sm_100a; host SASA and two H2D/D2H round "
                    "trips per proposal)",
            "energy": {"value": ne / de, "unit": "energy evals/s", "evals": ne, "seconds": de,
                       "what": "reference protein_physics_cuda calculate_potential(particles, topology) on the "
                               "same chain (energy only: the reference has no gradient)"}}


def energy_force_rate(system, topo, steps=20):
    """Full energy + analytic gradient evaluations per second on one system:
    neighbor-list build, Born radii, energy terms and alma_forces per eval
    (device events, inputs resident)."""
    import torch
    from protein_physics_b200.device import DeviceBatch
    b = DeviceBatch([system], precision="mixed")
    grad = torch.zeros((b.natoms, 4), dtype=torch.float64, device="cuda")
    terms = torch.zeros((1, 5), dtype=torch.float64, device="cuda")

    def ev():
        b.nl_ready = False
        b.build_nl(check=False)
        b.energy_terms(recompute_born=True, out=terms)
        b.forces(out=grad)

    b.build_nl()
    for _ in range(3):
        ev()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        ev()
    e1.record()
    f0.record()
    for _ in range(steps):
        b.forces(out=grad)
    f1.record()
    g0.record()
    for _ in range(steps):
        b.nl_ready = False
        b.build_nl(check=False)
        b.energy_terms(recompute_born=True, out=terms)
    g1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    # the same evaluation replayed as one captured CUDA graph
    b.evaluate(graph=True)
    torch.cuda.synchronize()
    h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h0.record()
    for _ in range(steps):
        b.evaluate(graph=True)
    h1.record()
    torch.cuda.synchronize()
    ms_graph = h0.elapsed_time(h1) / steps
    # the same energy through the public API, host particles in and a float out
    from protein_physics_b200 import Particle, PhysicsEngine
    xyz, q, r, eps, flat = system
    P = [Particle(*map(float, x), float(qq), float(rr), float(ee)) for x, qq, rr, ee in zip(xyz, q, r, eps)]
    eng = PhysicsEngine(precision="mixed")
    eng.calculate_potential(P, topo)
    t0 = time.perf_counter()
    ne = 0
    while time.perf_counter() - t0 < 1.0 or ne < 3:
        eng.calculate_potential(P, topo)
        ne += 1
    api = ne / (time.perf_counter() - t0)
    return {"value": 1e3 / ms, "unit": "energy+force evals/s", "atoms": b.natoms, "ms_per_eval": ms,
            "forces_ms": f0.elapsed_time(f1) / steps, "energy_only_ms": g0.elapsed_time(g1) / steps,
            "graph": {"value": 1e3 / ms_graph, "ms_per_eval": ms_graph,
                      "what": "DeviceBatch.evaluate(graph=True): the same list + energy + gradient replayed as "
                              "one CUDA graph, with its per-call overflow check (one status read)"},
            "calculate_potential_per_s": api,
            "what": "neighbor list + Born radii + energy terms + analytic dE/dx (alma_forces), mixed precision"}


def run_reference(args, rank, world):
    """--impl reference: the reference CPU engine on all host threads."""
    if rank != 0:
        return None
    import glob
    hits = glob.glob(os.path.join(ROOT, "oracle", "_ref", "protein_physics*.so"))
    if not hits:
        return {"impl": "reference", "unavailable": "reference engine not built (oracle/_ref)"}
    sys.path.insert(0, os.path.dirname(hits[0]))
    import protein_physics as pp
    chains, systems, movesets, temps, topos = make_workload(args.workload, 0)
    ch = chains[0]
    R = pp.BondTopology()
    R.build(ch.resnames, ch.atomnames, ch.res_idx)
    P = [pp.Particle(*map(float, x), float(q), float(r), float(e)) for x, q, r, e in
         zip(ch.xyz, ch.charge, ch.radius, ch.epsilon)]
    eng = pp.PhysicsEngine()
    ncand = eng.num_threads()
    t0 = time.perf_counter()
    eng.generate_ensemble(P, R, ncand, 3, temps[0], 0.12)
    per = max(1e-3, time.perf_counter() - t0) / 3
    n = max(5, int(20.0 / max(1, args.steps + args.warmup) / per))
    for _ in range(args.warmup):
        eng.generate_ensemble(P, R, ncand, n, temps[0], 0.12)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        eng.generate_ensemble(P, R, ncand, n, temps[0], 0.12)
    dt = time.perf_counter() - t0
    value = args.steps * n * ncand / dt
    return {"impl": "reference", "metric": "Metropolis proposals/s", "value": value, "unit": "proposals/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (same seeded chain)",
            "config": {"workload": f"reference generate_ensemble on the {ch.n}-atom chain, {ncand} candidates x "
                                   f"{n} proposals per step (one chain per OpenMP thread)"},
            "cpu_baseline": {"value": value, "unit": "proposals/s", "cores": ncand, "kind": "reference",
                             "sample": f"{args.steps} x {ncand} chains x {n} proposals"},
            "e2e": {"value": value, "unit": "proposals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def _line(metric, value, unit, args, ms_per_step, config, clocks, launches, **extra):
    out = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f32 pair terms, f64 dE / accumulation", "data": "synthetic (seeded NeRF chains)",
           "config": config, "clocks": clocks, "gpu_launches": int(launches)}
    out.update(extra)
    return out


def run_globule(args):
    """Differentiation workload: one 1,000-residue collapsed chain (~16k
    atoms).  Reports energy+force evals/s, 500 descent steps, then the timed
    MALA torsion proposals (step 0.5 deg, 300 K): one bench step = 10 MALA
    proposals (each: all-bond move, list, Born, energy, forces, torsion
    gradient, Metropolis-Hastings)."""
    import numpy as np
    import torch
    from protein_physics_b200 import _lib, synth
    from protein_physics_b200.device import DeviceBatch
    from protein_physics_b200.topology import BondTopology, flatten
    from protein_physics_b200.torsion import MALARunner, TorsionSpace, minimize
    ch = synth.compact_chain(1000, seed=4)
    T = BondTopology()
    T.build(ch.resnames, ch.atomnames, ch.res_idx)
    system = (ch.xyz, ch.charge, ch.radius, ch.epsilon, flatten(T))
    ef = energy_force_rate(system, T)
    b = DeviceBatch([system], precision="mixed")
    ts = TorsionSpace(b)
    torch.cuda.synchronize()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record()
    hist, eta = minimize(b, steps=500, ts=ts)
    g1.record()
    torch.cuda.synchronize()
    gd_ms = g0.elapsed_time(g1)
    E = hist[:, 0].cpu().numpy()
    fd = force_fd_check(b, system)
    R = MALARunner(b, 300.0 * KB, seed=2024, step=np.radians(0.5), ts=ts)
    per = 10
    R.run(300)  # step-scale adaptation (window 20) settles before the timed proposals
    for _ in range(args.warmup):
        R.run(per)
    st0 = R.state()
    l0 = _lib.lib().alma_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(0)
    torch.cuda.synchronize()
    R.run(per, graph=True)  # capture the proposal graph
    st0 = R.state()
    with sampler:
        e0.record()
        for _ in range(args.steps):
            R.run(per, graph=True)
        e1.record()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    st1 = R.state()
    ee0, ee1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ee0.record()
    R.run(per)  # the same proposals launched one by one from the host, for comparison
    ee1.record()
    torch.cuda.synchronize()
    eager_rate = per / (ee0.elapsed_time(ee1) * 1e-3)
    n = int(st1["n_proposed"][0] - st0["n_proposed"][0])
    acc = int(st1["n_accepted"][0] - st0["n_accepted"][0])
    return _line("MALA torsion proposals/s", n / (ms * 1e-3), "proposals/s", args, ms / args.steps,
                 {"workload": "1,000-residue collapsed chain, %d atoms, Rg %.1f A; 500 descent steps, then MALA "
                              "(all %d rotatable bonds per proposal, step 0.5 deg, truncated drift), 300 K, "
                              "10 proposals per step" % (ch.n, synth.radius_of_gyration(ch.xyz), ts.nrb),
                  "atoms": ch.n, "mala_accept_rate": acc / max(1, n), "mala_step_scale": float(st1["scale"][0]),
                  "launch": "one CUDA graph per proposal (%.0f proposals/s when launched from the host)" % eager_rate,
                  "l2": "inputs > L2 (16k atoms x lists)"},
                 sampler.summary(), _lib.lib().alma_launch_count() - l0,
                 energy_force=ef, force_check=fd,
                 descent={"steps": 500, "ms": gd_ms, "steps_per_s": 500 / (gd_ms * 1e-3), "E_start": float(E[0]),
                          "E_end": float(E[-1]), "unit": "kcal/mol"})


def force_fd_check(b, system, n_atoms=64, h=1e-4, seed=64):
    """Analytic forces (mixed and FP64) vs central finite differences of the
    FP64 device energy (h = 1e-4 Å, list fixed) on n_atoms random atoms of
    the batch's current coordinates; atoms with a pair within 1e-3 Å of the
    12 Å cutoff (where the reference energy jumps) are not drawn."""
    import numpy as np
    import torch
    from protein_physics_b200.device import DeviceBatch
    x0 = b.coords(0).copy()
    _, q, r, e, F = system
    b64 = DeviceBatch([(x0, q, r, e, F)], precision="fp64")
    b64.build_nl()
    b64.energy_terms()
    g64 = b64.forces()[:b64.natoms, :3].cpu().numpy()
    bm = DeviceBatch([(x0, q, r, e, F)], precision="mixed")
    bm.build_nl()
    bm.energy_terms()
    gm = bm.forces()[:bm.natoms, :3].cpu().numpy()
    rp, cols, _ = b64.nl_host(0, half=True)
    I = np.repeat(np.arange(x0.shape[0]), np.diff(rp))
    dist = np.sqrt(((x0[I] - x0[cols]) ** 2).sum(1))
    near = np.zeros(x0.shape[0], bool)
    bad = np.abs(dist - 12.0) < 1e-3 + 2 * h
    near[I[bad]] = True
    near[cols[bad]] = True
    atoms = np.random.default_rng(seed).choice(np.flatnonzero(~near), size=n_atoms, replace=False)
    xd = b64.xyz

    def E(i, c, d):
        xd[i, c] += d
        b64.nl_ready = True
        v = float(b64.energy_terms()[0, 4])
        xd[i, c] -= d
        return v

    worst = {"fp64": 0.0, "mixed": 0.0}
    for i in atoms:
        fdv = np.array([(E(int(i), c, h) - E(int(i), c, -h)) / (2 * h) for c in range(3)])
        scale = max(np.abs(fdv).max(), 1.0)
        worst["fp64"] = max(worst["fp64"], float(np.abs(g64[i] - fdv).max() / scale))
        worst["mixed"] = max(worst["mixed"], float(np.abs(gm[i] - fdv).max() / scale))
    return {"atoms": int(n_atoms), "h_A": h, "max_rel_err_fp64": worst["fp64"], "max_rel_err_mixed": worst["mixed"],
            "what": "max over atoms of max|F - FD| / max(|FD|, 1 kcal/mol/A); FD of the FP64 energy, list fixed"}


def run_replica(args):
    """Combined workload: 16 temperature replicas (300-450 K geometric) of a
    4-domain chain (4 x 1,000 residues + 10-residue linkers); MALA and plain
    torsion proposals 1:3, replica exchange every 100 sweeps.  One bench
    step = one exchange interval (100 proposals per replica)."""
    import torch
    from protein_physics_b200 import _lib, synth
    from protein_physics_b200.replica import ReplicaExchange, geometric_ladder
    from protein_physics_b200.topology import BondTopology, flatten
    ch = synth.multidomain_chain(4, 1000, 10, seed=11)
    T = BondTopology()
    T.build(ch.resnames, ch.atomnames, ch.res_idx)
    F = flatten(T)
    moveset = [k for k in range(F.nrb) if F.side_count[k] <= 0.25 * F.n]
    RE = ReplicaExchange((ch.xyz, ch.charge, ch.radius, ch.epsilon, F), geometric_ladder(300, 450, 16), seed=9,
                         moveset=moveset, minimize_steps=500, mala_warmup=400)
    for _ in range(args.warmup):
        RE.interval(100)
    torch.cuda.synchronize()
    p0 = RE.proposals
    l0 = _lib.lib().alma_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(0)
    with sampler:
        e0.record()
        for _ in range(args.steps):
            RE.interval(100)
        e1.record()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    st = RE.stats()
    return _line("Metropolis proposals/s (replica exchange)", (RE.proposals - p0) / (ms * 1e-3), "proposals/s", args,
                 ms / args.steps,
                 {"workload": "16 replicas x %d-atom 4-domain chain (%d atoms), T 300-450 K geometric, "
                              "MALA:torsion 1:3, exchange every 100 sweeps" % (ch.n, 16 * ch.n),
                  "atoms": 16 * ch.n, "l2": "inputs > L2"},
                 sampler.summary(), _lib.lib().alma_launch_count() - l0, exchange=st)


def run_profile_case(args):
    """Small cases for ncu.  "mc": the single-chain workload, 100 warm-up
    proposals, then exactly one mc launch of up to 200 proposals (it stops
    at the first drift flag); --config CL,NT[,K] picks the launch shape.
    "forces": the same chain, one energy evaluation and one alma_forces
    call (4 gradient kernels).  "energy": the first 48 chains of the batched
    workload (about 0.24M atoms, rows well above L2), one neighbor-list
    build, one full energy evaluation and one gradient (alma_forces)."""
    import torch
    from protein_physics_b200.device import DeviceBatch
    from protein_physics_b200.mc import MCRunner
    if args.profile == "energy":
        chains, systems, _, _, _ = make_workload("batched", 0, n_chains=48)
        batch = DeviceBatch(systems, precision="mixed")
        batch.build_nl()
        terms = batch.energy_terms()
        batch.forces()
        torch.cuda.synchronize()
        print(json.dumps({"profile_case": "energy", "systems": len(chains), "atoms": batch.natoms,
                          "half_entries": int(batch.half_len.sum()), "full_entries": int(batch.full_len.sum()),
                          "total_energy": float(terms[:, 4].sum())}))
        return
    chains, systems, movesets, temps, topos = make_workload("single", 0)
    batch = DeviceBatch(systems, precision="mixed")
    if args.profile == "forces":
        batch.energy_terms()
        g = batch.forces()
        torch.cuda.synchronize()
        print(json.dumps({"profile_case": "forces", "atoms": chains[0].n, "grad_norm": float(g.norm())}))
        return
    cl, nt, k = (tuple(int(v) for v in args.config.split(",")) + (1,))[:3] if args.config else \
        (args.cluster, args.threads, 1)
    runner = MCRunner(batch, temps, seed=12345, policy=2, moveset=movesets, cluster_size=cl, threads=nt,
                      spec_teams=k)
    runner.run(100)
    lim = int(runner.state()["step"].max()) + 200
    runner.launch(lim)
    torch.cuda.synchronize()
    st = runner.state()
    print(json.dumps({"profile_case": "single chain", "atoms": chains[0].n, "steps_done": int(st["step"][0]),
                      "cluster": cl, "threads": nt, "spec_teams": k}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--profile", nargs="?", const="mc", default=None, choices=["mc", "forces", "energy"],
                    help="a small case for ncu: one mc launch (mc), one gradient evaluation (forces) "
                         "or one batched list build + energy evaluation (energy)")
    ap.add_argument("--config", default="", help="CL,NT[,K]: cluster size, CTA size and speculative teams "
                                                 "instead of the autotuner")
    ap.add_argument("--cluster", type=int, default=16)
    ap.add_argument("--threads", type=int, default=512)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="single", choices=["single", "batched", "globule", "replica"])
    args = ap.parse_args()
    rank, world, local = rank_info()
    if args.profile:
        run_profile_case(args)
        return
    if args.impl == "reference":
        out = run_reference(args, rank, world)
    elif args.workload == "globule":
        out = run_globule(args) if rank == 0 else None
    elif args.workload == "replica":
        out = run_replica(args) if rank == 0 else None
    else:
        out = run_ours(args, rank, world, local)
    if rank == 0 and out is not None:
        print(json.dumps(out))


if __name__ == "__main__":
    main()

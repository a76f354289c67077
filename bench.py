"""Benchmark: Metropolis proposals/s of the B200 engine (and of the reference).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload batched|single|globule|replica]

Workload "batched" (default): 256 independent chains, 50-600 residues each
(seeded, helix/coil phi/psi, ~1.36 M atoms), temperatures geometric over
280-400 K, the reference generate_ensemble proposal policy (every rotatable
bond, 25 % crankshaft, adaptive cur_max, 2.5x sidechain steps), FP32 pair
terms with FP64 ΔE and Metropolis test; one step = 100 proposals per chain.
The line also carries the single-chain drop-in ("single_chain": the
300-residue compact chain below, with the reference's plain GPU path and
CPU engine beside it).
Workload "single": the 300-residue compact chain (4,962 atoms, Rg ~17 Å,
workloads/c2_chain_300res.npz), torsion moves of bonds whose j-side holds
<= 25 % of the atoms, 300 K; one step = 1,000 proposals + a full energy.
Workload "globule": the 1,000-residue globule (workloads/c4_globule_1000res.npz):
energy+force evals/s, 500 descent steps, then MALA proposals/s.
Workload "replica": 16 replicas of the 4 x 1,000-residue chain
(workloads/c5_multidomain_4x1000res.npz), MALA:torsion 1:3, replica
exchange every 100 sweeps.

value  = proposals/s of the whole job on the device (CUDA events, inputs
         resident), max over ranks;
e2e    = the same metric through the public API with host buffers every
         step (batched: BatchedEnsemble.run, coordinates in and out;
         single: PhysicsEngine.generate_ensemble with particle lists).
--impl reference runs the reference engine (oracle/_ref, compiled from the
reference sources) on the host cores on the same inputs and prints the
same config; it loads nothing of this package (the chain generator
synth.py is loaded by path: numpy and scipy only).
Multi-GPU: every rank runs its own independent chains (replicas; no
data-path collective); value sums the proposals of all ranks.
"""
import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "protein-structure-analysis_b200")
WORKLOADS = os.path.join(ROOT, "workloads")

KB = 0.0019872  # kcal/mol/K
FP32_PEAK_NOMINAL = 148 * 128 * 2 * 1.965e9  # ops/s: SMs x FP32 lanes x FMA x max SM clock
OPS_PAIR, OPS_HCT, OPS_SASA = 47.0, 21.0, 11.0  # algorithmic ops per unit (FP32 + MUFU)
C3_CHAINS, C3_PER_STEP, C2_PER_STEP = 256, 100, 1000
L2_NOTE = "inputs larger than L2 (lists of 1.36 M atoms) and a 256 MiB L2 flush between GPU steps"
# DRAM bytes (read + write) per proposal of the MC kernel, from one ncu capture
# of a smaller case of the same workload, scaled by the proposals of a launch:
# profiles/mc_kernel_batched_48_chains.md (168.8 MB / 266 proposals)
DRAM_BYTES_PER_PROPOSAL = {"batched": 168.8e6 / 266}


def rank_info():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def seed_of(base, rank):
    """Seed of rank `rank`'s inputs (disjoint streams per rank)."""
    return int(base) + 1000 * int(rank)


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


# ---- inputs (numpy only: both arms build them the same way) --------------------------
def load_synth():
    """The chain generator, loaded by path (numpy + scipy; no package import)."""
    if "alma_synth" in sys.modules:
        return sys.modules["alma_synth"]
    spec = importlib.util.spec_from_file_location(
        "alma_synth", os.path.join(PKG, "protein_physics_b200", "synth.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["alma_synth"] = mod
    spec.loader.exec_module(mod)
    return mod


def _chain_dict(ch):
    return dict(xyz=ch.xyz, charge=ch.charge, radius=ch.radius, epsilon=ch.epsilon, resnames=list(ch.resnames),
                atomnames=list(ch.atomnames), res_idx=[int(v) for v in ch.res_idx])


def _coil_chain_job(n_res, seed):
    return _chain_dict(load_synth().coil_chain(n_res, seed))


def fixture(fname):
    """A chain written by workloads/make_workloads.py (plain arrays)."""
    import numpy as np
    d = np.load(os.path.join(WORKLOADS, fname), allow_pickle=False)
    return dict(xyz=d["xyz"].astype(np.float64), charge=d["charge"], radius=d["radius"], epsilon=d["epsilon"],
                resnames=[str(v) for v in d["resnames"]], atomnames=[str(v) for v in d["atomnames"]],
                res_idx=[int(v) for v in d["res_idx"]])


def rg_of(xyz):
    import numpy as np
    c = xyz - xyz.mean(0)
    return float(np.sqrt((c * c).sum(1).mean()))


def c3_inputs(rank, n_chains=C3_CHAINS, world=1):
    """The batched workload: chain sizes U{50..600} residues and per-chain
    seeds, helix/coil chains (synth.coil_chain), temperatures geometric over
    280-400 K (kcal/mol)."""
    import multiprocessing as mp
    import numpy as np
    rng = np.random.default_rng(seed_of(3, rank))
    sizes = rng.integers(50, 601, size=C3_CHAINS)[:n_chains]
    jobs = [(int(n), seed_of(k, rank)) for k, n in enumerate(sizes)]
    procs = max(1, min(32, (os.cpu_count() or 1) // max(1, world)))  # host Python: the cores, shared by the ranks
    with mp.get_context("spawn").Pool(procs) as pool:
        chains = pool.starmap(_coil_chain_job, jobs, chunksize=1)
    temps = list(280.0 * (400.0 / 280.0) ** (np.arange(C3_CHAINS) / (C3_CHAINS - 1)) * KB)[:n_chains]
    return chains, temps


def config_of(kind, chains):
    """The workload description both arms print (the same dict)."""
    atoms = int(sum(len(c["xyz"]) for c in chains))
    if kind == "batched":
        return {"workload": "batched MC: %d independent chains of 50-600 residues (seeded helix/coil, all-atom), "
                            "T 280-400 K geometric, the reference generate_ensemble proposal policy, "
                            "%d proposals per chain per step" % (len(chains), C3_PER_STEP),
                "chains": len(chains), "atoms": atoms, "proposals_per_chain_per_step": C3_PER_STEP,
                "moves": "every rotatable bond, 25 % crankshaft, cur_max adapted per 200 proposals",
                "l2": L2_NOTE, "parallelism": "replicas"}
    return {"workload": "single chain: 300-residue compact chain (%d atoms, Rg %.1f A), torsion moves of bonds "
                        "whose j-side holds <= 25 %% of the atoms, 300 K, %d proposals + a full energy per step"
                        % (atoms, rg_of(chains[0]["xyz"]), C2_PER_STEP),
            "chains": 1, "atoms": atoms, "rg_A": round(rg_of(chains[0]["xyz"]), 2),
            "l2": "a 256 MiB L2 flush between steps", "parallelism": "replicas"}


# ---- our arm --------------------------------------------------------------------------
def _our_systems(chains):
    sys.path.insert(0, PKG)
    from protein_physics_b200.topology import BondTopology, flatten
    systems, topos = [], []
    for c in chains:
        T = BondTopology()
        T.build(c["resnames"], c["atomnames"], c["res_idx"])
        systems.append((c["xyz"], c["charge"], c["radius"], c["epsilon"], flatten(T)))
        topos.append(T)
    return systems, topos


def _moveset(F):
    return [k for k in range(F.nrb) if F.side_count[k] <= 0.25 * F.n]


def _timed_mc(runner, batch, args, per_step, full_energy, world, local, flush):
    """W untimed steps, then K timed steps between events on the launching
    stream (L2 flushed between steps); returns the measurements."""
    import numpy as np
    import torch
    from protein_physics_b200 import _lib
    stream = torch.cuda.current_stream()

    def step():
        runner.run(per_step)
        if full_energy:
            runner.reset_energy()  # the full energy recomputation of every step

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    st0 = runner.state()
    launches0 = _lib.lib().alma_launch_count()
    rebuild0 = runner.rebuilds
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(local)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with sampler:
        ev0.record(stream)
        for _ in range(args.steps):
            flush.fill_(1.0)
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    st1 = runner.state()
    return dict(ms=ms, proposals=float(np.sum(st1["step"] - st0["step"])),
                accepted=float(np.sum(st1["n_accepted"] - st0["n_accepted"])),
                launches=_lib.lib().alma_launch_count() - launches0 + args.steps,  # + the flush fills
                rebuilds=runner.rebuilds - rebuild0, clocks=sampler.summary())


def _kernel_roofline(runner, batch, tuned, proposals_per_launch, workload=None):
    """One extra MC launch alone (no host rebuild step), timed with events
    on its stream; algorithmic ops from the kernel's own work counters."""
    import numpy as np
    import torch
    stream = torch.cuda.current_stream()
    ke0, ke1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    st0 = runner.state()
    c0 = batch.move_counters().astype(np.float64).sum(axis=0)
    lim = int(st0["step"].max()) + proposals_per_launch
    ke0.record(stream)
    runner.launch(lim)
    ke1.record(stream)
    torch.cuda.synchronize()
    k_ms = ke0.elapsed_time(ke1)
    c1 = batch.move_counters().astype(np.float64).sum(axis=0)
    st1 = runner.state()
    d = c1 - c0
    ops = d[0] * OPS_PAIR + d[1] * OPS_HCT + d[2] * OPS_SASA
    achieved = ops / (k_ms * 1e-3)
    name = ("mc_spec_kernel<float,%d,%d> x %d teams" % (tuned[1], tuned[0], tuned[2]) if tuned[2] > 1 else
            "mc_kernel<float,%d,%d>" % (tuned[1] or 512, tuned[0]))
    nprop = float(np.sum(st1["step"] - st0["step"]))
    per = DRAM_BYTES_PER_PROPOSAL.get(workload)
    traffic = per * nprop if per else None
    return {"bound": "fp32", "kernel": name, "achieved": achieved / 1e12, "peak": FP32_PEAK_NOMINAL / 1e12,
            "unit": "TOP/s (FP32+MUFU ops)", "frac": achieved / FP32_PEAK_NOMINAL,
            "peak_source": "nominal 148 SM x 128 FP32 lanes x 2 x 1965 MHz (no measured FP32 peak in "
                           "MEASURED_PEAKS.json; the kernel is neither HBM- nor tensor-bound)",
            "work_per_launch": {"pair_terms": float(d[0]), "hct": float(d[1]), "sasa_visits": float(d[2]),
                                "moved_atoms": float(d[3]), "proposals": nprop},
            "kernel_ms": k_ms, "traffic": traffic,
            "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum per proposal of a 48-chain capture "
                               "(profiles/mc_kernel_batched_48_chains.md) x this launch's proposals; "
                               "%.1f GB/s achieved" % (traffic / (k_ms * 1e-3) / 1e9)) if traffic else None}


def run_ours(args, rank, world, local):
    import numpy as np
    import torch
    sys.path.insert(0, PKG)
    from protein_physics_b200.device import DeviceBatch
    from protein_physics_b200.mc import BatchedEnsemble, MCRunner, autotune
    torch.cuda.set_device(local)
    if world > 1:
        from protein_physics_b200.dist import init
        init("nccl", timeout_s=120)
    if args.workload == "batched":
        chains, temps = c3_inputs(rank, world=world)
        policy, per_step, full_energy = 0, C3_PER_STEP, False
    else:
        chains, temps = [fixture("c2_chain_300res.npz")], [300.0 * KB]
        policy, per_step, full_energy = 2, C2_PER_STEP, True
    config = config_of(args.workload, chains)
    systems, topos = _our_systems(chains)
    movesets = None if policy == 0 else [_moveset(s[4]) for s in systems]
    batch = DeviceBatch(systems, precision="mixed")
    if args.config:
        tuned = tuple(int(v) for v in args.config.split(","))
    else:
        tuned = autotune(batch, temps, seed=777, policy=policy, moveset=movesets,
                         proposals=1000 if policy == 2 else 30)
    tuned = (tuple(tuned) + (1,))[:3]
    runner = MCRunner(batch, temps, seed=12345 + rank, policy=policy, cur_max0=0.12, moveset=movesets,
                      cluster_size=tuned[0], threads=tuned[1], spec_teams=tuned[2])
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    t = _timed_mc(runner, batch, args, per_step, full_energy, world, local, flush)
    from protein_physics_b200.dist import reduce_timing
    ms_max, prop_total = reduce_timing(t["ms"], t["proposals"], device="cuda")
    roof = _kernel_roofline(runner, batch, tuned, 200 if policy == 2 else 50, args.workload)
    # e2e through the public API, host buffers in and out every step
    if args.workload == "batched":
        e2e = e2e_batched(systems, temps, tuned, args, world)
    else:
        e2e = e2e_single(chains[0], topos[0], args, world)
    out = None
    if rank == 0:
        stats = {"accept_rate": t["accepted"] / max(1.0, t["proposals"]), "nl_rebuilds": t["rebuilds"],
                 "rg_A_mean": float(np.mean([rg_of(c["xyz"]) for c in chains])),
                 "full_row_mean": float(batch.full_len[:batch.natoms].double().mean()),
                 "half_row_mean": float(batch.half_len[:batch.natoms].double().mean())}
        out = {
            "metric": "Metropolis proposals/s", "value": prop_total / (ms_max * 1e-3), "unit": "proposals/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 pair terms, f64 dE",
            "data": "synthetic (seeded NeRF chains, ff14SB parameters from the reference tables)",
            "config": config, "workload_stats": stats, "clocks": t["clocks"], "gpu_launches": int(t["launches"]),
            "tuned": {"cluster_size": tuned[0], "threads_per_system": tuned[1], "spec_teams": tuned[2]},
            "e2e": e2e, "roofline": roof,
        }
        if world == 1:
            out["cpu_baseline"] = cpu_baseline(args.workload, chains, temps)
            if args.workload == "batched":
                out["single_chain"] = single_chain_section(args)
            else:
                out.update(single_extras(chains[0], topos[0], systems[0], movesets[0], runner))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return out


def e2e_batched(systems, temps, tuned, args, world):
    """BatchedEnsemble.run(100, xyz=host coordinates) per step: host->device
    copy of every chain's coordinates, the device MC, device->host copy of
    the final coordinates."""
    import torch
    from protein_physics_b200.mc import BatchedEnsemble
    ens = BatchedEnsemble(systems, temps, seed=4242, shape=tuned)
    X = ens.run(5).copy()
    n = max(3, args.steps // 2)
    p0 = ens.state()["step"].sum()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(n):
        X = ens.run(C3_PER_STEP, xyz=X)
    dt = time.perf_counter() - t0
    props = float(ens.state()["step"].sum() - p0)
    nbytes = int(X.nbytes)
    return {"value": props / dt * world, "unit": "proposals/s", "h2d_bytes_per_step": nbytes,
            "d2h_bytes_per_step": nbytes, "steps": n,
            "api": "BatchedEnsemble(systems, temperatures).run(100, xyz=host coordinates of all chains): "
                   "host->device copy, fresh lists and energies, the MC, device->host copy (wall clock)"}


def e2e_single(ch, topo, args, world):
    """PhysicsEngine.generate_ensemble(host particle lists, n candidates,
    1,000 proposals) with n = the host threads (the call the reference arm
    times for one chain), and with one candidate."""
    import torch
    from protein_physics_b200 import Particle, PhysicsEngine
    eng = PhysicsEngine(precision="mixed", seed=99)
    P0 = [Particle(*x, q, r, e) for x, q, r, e in zip(ch["xyz"], ch["charge"], ch["radius"], ch["epsilon"])]
    n_e2e = max(1, args.steps // 2)
    stream = torch.cuda.current_stream()

    def rate(ncand):
        P = P0
        eng.generate_ensemble(P, topo, ncand, 50)  # warm
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(n_e2e):
            P = eng.generate_ensemble(P, topo, ncand, C2_PER_STEP)[0]
        e1.record(stream)
        torch.cuda.synchronize()
        return n_e2e * ncand * C2_PER_STEP / (e0.elapsed_time(e1) * 1e-3) * world

    pp = _ref_module()  # one candidate per thread of the reference engine, as its arm runs
    ref_threads = pp.PhysicsEngine().num_threads() if pp is not None else None
    ncand = ref_threads or host_threads()
    n = len(P0)
    return {"value": rate(ncand), "unit": "proposals/s", "h2d_bytes_per_step": ncand * n * 24 + n * 24,
            "d2h_bytes_per_step": ncand * n * 24, "candidates": ncand, "reference_threads": ref_threads,
            "host_threads": host_threads(), "single_candidate": rate(1),
            "api": "PhysicsEngine.generate_ensemble(host particles, topology, n_candidates, 1000), n_candidates = "
                   "the host threads; single_candidate: the same with 1 candidate",
            "workload": "the reference's own move policy (every rotatable bond, 25 % crankshaft), as the reference "
                        "times it"}


def single_extras(ch, topo, system, moveset, runner):
    """Beside the single-chain number: the reference's plain GPU path, FP64
    proposals/s, the ΔE error against FP64 and energy+force evals/s."""
    return {"plain_gpu_path": plain_gpu_baseline(ch, 300.0 * KB),
            "fp64": fp64_rate(system, moveset),
            "dE_error_vs_fp64": de_error_vs_fp64(system, moveset, runner.state()["cur_max"][0]),
            "energy_force": energy_force_rate(system, topo)}


def single_chain_section(args):
    """The single-chain drop-in on the 300-residue compact chain: device
    rate, its kernel roofline, e2e through generate_ensemble, and the
    comparators (reference plain GPU path and CPU engine, FP64 rate)."""
    import torch
    from protein_physics_b200.device import DeviceBatch
    from protein_physics_b200.mc import MCRunner, autotune

    class A:
        steps, warmup = max(3, args.steps // 2), 3
    ch = fixture("c2_chain_300res.npz")
    systems, topos = _our_systems([ch])
    ms = [_moveset(systems[0][4])]
    temps = [300.0 * KB]
    batch = DeviceBatch(systems, precision="mixed")
    tuned = (tuple(autotune(batch, temps, seed=777, policy=2, moveset=ms, proposals=1000)) + (1,))[:3]
    runner = MCRunner(batch, temps, seed=12345, policy=2, cur_max0=0.12, moveset=ms, cluster_size=tuned[0],
                      threads=tuned[1], spec_teams=tuned[2])
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    t = _timed_mc(runner, batch, A, C2_PER_STEP, True, 1, torch.cuda.current_device(), flush)
    out = {"value": t["proposals"] / (t["ms"] * 1e-3), "unit": "proposals/s", "steps": A.steps,
           "config": config_of("single", [ch]),
           "workload_stats": {"accept_rate": t["accepted"] / max(1.0, t["proposals"]), "nl_rebuilds": t["rebuilds"],
                              "full_row_mean": float(batch.full_len[:batch.natoms].double().mean()),
                              "half_row_mean": float(batch.half_len[:batch.natoms].double().mean())},
           "tuned": {"cluster_size": tuned[0], "threads_per_system": tuned[1], "spec_teams": tuned[2]},
           "clocks": t["clocks"], "roofline": _kernel_roofline(runner, batch, tuned, 200),
           "e2e": e2e_single(ch, topos[0], A, 1),
           "cpu_baseline": cpu_baseline("single", [ch], temps)}
    out.update(single_extras(ch, topos[0], systems[0], ms[0], runner))
    return out


def fp64_rate(system, moveset, steps=3):
    """Proposals/s of the same single-chain workload with FP64 pair terms
    (the reference's own precision), same launch shape rules."""
    import torch
    from protein_physics_b200.device import DeviceBatch
    from protein_physics_b200.mc import MCRunner
    b = DeviceBatch([system], precision="fp64")
    R = MCRunner(b, [300.0 * KB], seed=54321, policy=2, moveset=[moveset])
    R.run(C2_PER_STEP)
    torch.cuda.synchronize()
    st0 = R.state()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        R.run(C2_PER_STEP)
        R.reset_energy()
    e1.record()
    torch.cuda.synchronize()
    n = float((R.state()["step"] - st0["step"]).sum())
    return {"value": n / (e0.elapsed_time(e1) * 1e-3), "unit": "proposals/s", "precision": "fp64 pair terms",
            "steps": steps, "spec_teams": int(R.cfg.spec_teams), "cluster_size": int(R.cfg.cluster_size)}


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


# ---- the reference engine (oracle/_ref) -------------------------------------------------
def _ref_module():
    import glob
    hits = glob.glob(os.path.join(ROOT, "oracle", "_ref", "protein_physics.*so"))
    if not hits:
        return None
    sys.path.insert(0, os.path.dirname(hits[0]))
    import protein_physics as pp
    return pp


def _ref_inputs(pp, c):
    R = pp.BondTopology()
    R.build(c["resnames"], c["atomnames"], c["res_idx"])
    P = [pp.Particle(*map(float, x), float(q), float(r), float(e)) for x, q, r, e in
         zip(c["xyz"], c["charge"], c["radius"], c["epsilon"])]
    return P, R


def stratified(chains, k, offset=0.5):
    """k chain indices spread evenly over the size order."""
    import numpy as np
    order = np.argsort([len(c["xyz"]) for c in chains], kind="stable")
    return [int(order[min(len(order) - 1, int((s + offset) / k * len(order)))]) for s in range(k)]


def ref_batched_rate(pp, chains, temps, picks, n_props, ncand):
    """The reference on the batched workload: for each picked chain,
    generate_ensemble(chain, ncand candidates, n_props proposals, its own
    temperature) — one OpenMP thread per candidate — timed as a whole."""
    eng = pp.PhysicsEngine()
    inputs = [_ref_inputs(pp, chains[k]) for k in picks]
    t0 = time.perf_counter()
    for (P, R), k in zip(inputs, picks):
        eng.generate_ensemble(P, R, ncand, n_props, temps[k], 0.12)
    return len(picks) * ncand * n_props, time.perf_counter() - t0


def cpu_baseline(kind, chains, temps, budget_s=12.0):
    """The reference engine (oracle/_ref) on the host cores, a bounded sample
    of the same workload."""
    pp = _ref_module()
    if pp is None:
        return {"value": None, "unit": "proposals/s", "cores": 0, "kind": "reference",
                "sample": "unavailable: oracle/_ref not built"}
    eng = pp.PhysicsEngine()
    if kind == "batched":
        ncand = eng.num_threads()
        picks = stratified(chains, 8)
        props, dt = ref_batched_rate(pp, chains, temps, picks[:1], 5, ncand)
        n = max(5, int(budget_s / max(dt, 1e-3) * 5 / len(picks)))
        props, dt = ref_batched_rate(pp, chains, temps, picks, n, ncand)
        return {"value": props / dt, "unit": "proposals/s", "cores": ncand, "kind": "reference",
                "sample": "reference generate_ensemble on 8 chains spread over the size range, %d candidates x %d "
                          "proposals each, %d proposals in %.1f s" % (ncand, n, props, dt)}
    P, R = _ref_inputs(pp, chains[0])
    t0 = time.perf_counter()
    eng.generate_ensemble(P, R, 1, 5, temps[0], 0.12)
    dt5 = max(1e-3, time.perf_counter() - t0)
    n = max(10, int(budget_s / dt5 * 5))
    t0 = time.perf_counter()
    eng.generate_ensemble(P, R, 1, n, temps[0], 0.12)
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": "proposals/s", "cores": 1, "kind": "reference",
            "sample": f"reference generate_ensemble(chain of {len(P)} atoms, 1 candidate, {n} proposals) in "
                      f"{dt:.1f} s; one chain runs on one thread (OpenMP spans candidates)"}


def run_reference(args, rank, world):
    """--impl reference: the reference CPU engine (oracle/_ref) on all host
    threads, on the same inputs, printing the same config."""
    if rank != 0:
        return None
    pp = _ref_module()
    if pp is None:
        return {"impl": "reference", "unavailable": "reference engine not built (oracle/_ref)"}
    eng = pp.PhysicsEngine()
    ncand = eng.num_threads()
    if args.workload == "batched":
        chains, temps = c3_inputs(0)
        picks_w = stratified(chains, max(1, args.warmup), offset=0.25)
        picks = stratified(chains, args.steps)
        _, dt = ref_batched_rate(pp, chains, temps, picks_w[:1], 5, ncand)
        n = max(5, int(20.0 / max(1, args.steps + args.warmup) / max(dt, 1e-3) * 5))
        ref_batched_rate(pp, chains, temps, picks_w, n, ncand)
        props, dt = ref_batched_rate(pp, chains, temps, picks, n, ncand)
        sample = ("one chain per step, %d chains spread over the size range (of %d), generate_ensemble with %d "
                  "candidates x %d proposals each at the chain's temperature" % (args.steps, len(chains), ncand, n))
    elif args.workload == "single":
        chains, temps = [fixture("c2_chain_300res.npz")], [300.0 * KB]
        P, R = _ref_inputs(pp, chains[0])
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
        props = args.steps * n * ncand
        sample = "%d x generate_ensemble(%d candidates x %d proposals), every rotatable bond (the reference " \
                 "cannot restrict its moves)" % (args.steps, ncand, n)
    else:
        return {"impl": "reference", "unavailable": "the reference has no %s workload (no gradient, no MALA)"
                % args.workload}
    value = props / dt
    return {"impl": "reference", "metric": "Metropolis proposals/s", "value": value, "unit": "proposals/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded NeRF chains, ff14SB parameters from the reference tables)",
            "config": config_of(args.workload, chains),
            "cpu_baseline": {"value": value, "unit": "proposals/s", "cores": ncand, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "proposals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def plain_gpu_baseline(ch, T, budget_s=8.0):
    """The reference's own plain GPU path (src/physics_engine_cuda.cu built
    unmodified for sm_100a into oracle/_ref): generate_ensemble on the same
    chain, one candidate, on this GPU."""
    import glob
    hits = glob.glob(os.path.join(ROOT, "oracle", "_ref", "protein_physics_cuda*.so"))
    pp = _ref_module()
    if not hits or pp is None:
        return {"value": None, "unit": "proposals/s", "unavailable": "oracle/_ref/protein_physics_cuda not built"}
    sys.path.insert(0, os.path.dirname(hits[0]))
    import protein_physics_cuda as pc
    R = pp.BondTopology()
    R.build(ch["resnames"], ch["atomnames"], ch["res_idx"])
    P = [pc.Particle(*map(float, x), float(q), float(r), float(e)) for x, q, r, e in
         zip(ch["xyz"], ch["charge"], ch["radius"], ch["epsilon"])]
    eng = pc.PhysicsEngine()
    t0 = time.perf_counter()
    eng.generate_ensemble(P, R, 1, 5, T, 0.12)
    dt5 = max(1e-3, time.perf_counter() - t0)
    n = max(10, int(budget_s / dt5 * 5))
    t0 = time.perf_counter()
    eng.generate_ensemble(P, R, 1, n, T, 0.12)
    dt = time.perf_counter() - t0
    eng.calculate_potential(P, R)  # its full-energy path (the reference has no forces)
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
    sys.path.insert(0, PKG)
    from protein_physics_b200 import _lib
    from protein_physics_b200.device import DeviceBatch
    from protein_physics_b200.torsion import MALARunner, TorsionSpace, minimize
    ch = fixture("c4_globule_1000res.npz")
    systems, topos = _our_systems([ch])
    system, T = systems[0], topos[0]
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
                 {"workload": "1,000-residue globule, %d atoms, Rg %.1f A; 500 descent steps, then MALA "
                              "(all %d rotatable bonds per proposal, step 0.5 deg, truncated drift), 300 K, "
                              "10 proposals per step" % (len(ch["xyz"]), rg_of(ch["xyz"]), ts.nrb),
                  "atoms": len(ch["xyz"]), "mala_accept_rate": acc / max(1, n), "mala_step_scale": float(st1["scale"][0]),
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
    sys.path.insert(0, PKG)
    from protein_physics_b200 import _lib
    from protein_physics_b200.replica import ReplicaExchange, geometric_ladder
    ch = fixture("c5_multidomain_4x1000res.npz")
    systems, _ = _our_systems([ch])
    RE = ReplicaExchange(systems[0], geometric_ladder(300, 450, 16), seed=9, moveset=_moveset(systems[0][4]),
                         minimize_steps=500, mala_warmup=400)
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
                              "MALA:torsion 1:3, exchange every 100 sweeps" % (len(ch["xyz"]), 16 * len(ch["xyz"])),
                  "atoms": 16 * len(ch["xyz"]), "l2": "inputs > L2"},
                 sampler.summary(), _lib.lib().alma_launch_count() - l0, exchange=st)


def run_profile_case(args):
    """Small cases for ncu.  "mc": the single-chain workload, 100 warm-up
    proposals, then exactly one mc launch of up to 200 proposals (it stops
    at the first drift flag); --config CL,NT[,K] picks the launch shape.
    "mc-batched": the first 48 chains of the batched workload (~0.25 M
    atoms), 20 warm-up proposals per chain, then one mc launch of up to 20
    proposals per chain.  "forces": the single chain, one energy evaluation
    and one alma_forces call (4 gradient kernels).  "energy": the first 48
    chains of the batched workload, one neighbor-list build, one full energy
    evaluation and one gradient (alma_forces).  The measured part sits
    between cudaProfilerStart/Stop (ncu --profile-from-start off)."""
    import torch
    sys.path.insert(0, PKG)
    from protein_physics_b200.device import DeviceBatch
    from protein_physics_b200.mc import MCRunner
    if args.profile in ("energy", "mc-batched"):
        chains, temps = c3_inputs(0, n_chains=48)
        systems, _ = _our_systems(chains)
        batch = DeviceBatch(systems, precision="mixed")
        if args.profile == "mc-batched":
            runner = MCRunner(batch, temps, seed=12345, policy=0, cluster_size=1, threads=args.threads,
                              spec_teams=1)
            runner.run(20)
            lim = int(runner.state()["step"].max()) + 20
            torch.cuda.synchronize()
            torch.cuda.profiler.start()  # ncu --profile-from-start off: only this launch
            runner.launch(lim)
            torch.cuda.synchronize()
            torch.cuda.profiler.stop()
            print(json.dumps({"profile_case": "mc-batched", "systems": len(chains), "atoms": batch.natoms,
                              "proposals": int(runner.state()["step"].sum())}))
            return
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        batch.build_nl()
        terms = batch.energy_terms()
        batch.forces()
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        print(json.dumps({"profile_case": "energy", "systems": len(chains), "atoms": batch.natoms,
                          "half_entries": int(batch.half_len.sum()), "full_entries": int(batch.full_len.sum()),
                          "total_energy": float(terms[:, 4].sum())}))
        return
    ch = fixture("c2_chain_300res.npz")
    systems, _ = _our_systems([ch])
    temps = [300.0 * KB]
    batch = DeviceBatch(systems, precision="mixed")
    if args.profile == "forces":
        batch.energy_terms()
        g = batch.forces()
        torch.cuda.synchronize()
        print(json.dumps({"profile_case": "forces", "atoms": batch.natoms, "grad_norm": float(g.norm())}))
        return
    cl, nt, k = (tuple(int(v) for v in args.config.split(",")) + (1,))[:3] if args.config else \
        (args.cluster, args.threads, 1)
    runner = MCRunner(batch, temps, seed=12345, policy=2, moveset=[_moveset(systems[0][4])], cluster_size=cl,
                      threads=nt, spec_teams=k)
    runner.run(100)
    lim = int(runner.state()["step"].max()) + 200
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    runner.launch(lim)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    st = runner.state()
    print(json.dumps({"profile_case": "single chain", "atoms": batch.natoms, "steps_done": int(st["step"][0]),
                      "cluster": cl, "threads": nt, "spec_teams": k}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--profile", nargs="?", const="mc", default=None,
                    choices=["mc", "mc-batched", "forces", "energy"],
                    help="a small case for ncu: one mc launch (mc: single chain; mc-batched: 48 chains), one "
                         "gradient evaluation (forces) or one batched list build + energy evaluation (energy)")
    ap.add_argument("--config", default="", help="CL,NT[,K]: cluster size, CTA size and speculative teams "
                                                 "instead of the autotuner")
    ap.add_argument("--cluster", type=int, default=16)
    ap.add_argument("--threads", type=int, default=512)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batched", choices=["batched", "single", "globule", "replica"])
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

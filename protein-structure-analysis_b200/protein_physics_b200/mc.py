"""Host driver of the device Monte Carlo (alma_mc_run) and the reference's
MC entry points on top of it.

``MCRunner`` advances every system of a DeviceBatch by a number of
proposals: it launches the persistent per-system kernel, and when a chain
has drifted more than half the skin since its last list build it rebuilds
that chain's neighbor list, Born radii and energy (the reference does the
same at the start of the next step, physics_engine.cpp:2506-2510) and
relaunches.  All other chains keep their lists.

``generate_ensemble`` / ``run_landscape`` reproduce the reference
semantics (physics_engine.cpp:2273-2543 and :2557-2951): value in, value
out; each candidate chain or the landscape chain starts from the initial
state; cur_max starts at max_angle; the landscape energies are full
calculate_potential evaluations of each snapshot.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .device import DeviceBatch, _ptr, _t
from .engine import particle_arrays, particles_from
from .topology import flatten

K_BOLTZMANN = 0.0019872  # kcal mol^-1 K^-1 (temperatures in K -> kcal/mol)
TAIL_MAX_TEAMS = 4  # speculative teams per chain a tail launch may use (auto_shape's maximum)


def mc_config(seed, policy=0, tune_freq=200, max_angle_bounds=(0.004, 0.5), fixed_delta=0.0, moveset=None,
              nsys=1, device_keep=None):
    """AlmaMCConfig with the reference constants (physics_engine.cpp:2304-2307)."""
    cfg = _lib.AlmaMCConfig()
    cfg.seed = int(seed) & ((1 << 64) - 1)
    cfg.policy = int(policy)
    cfg.tune_freq = int(tune_freq)
    cfg.target_lo, cfg.target_hi = 0.28, 0.52
    cfg.scale_up, cfg.scale_down = 1.06, 0.94
    cfg.angle_min, cfg.angle_max = max_angle_bounds
    cfg.sidechain_mult = 2.5
    cfg.crank_prob = 0.25
    cfg.concerted_prob = 0.15
    cfg.fixed_delta = float(fixed_delta)
    cfg.moveset_off = cfg.moveset = None
    cfg.threads_per_system = 0
    cfg.cluster_size = 1
    cfg.sys_order = None
    if moveset is not None:
        off = np.zeros(nsys + 1, np.int32)
        off[1:] = np.cumsum([len(m) for m in moveset])
        flat = np.concatenate([np.asarray(m, np.int32) for m in moveset]) if off[-1] else np.zeros(1, np.int32)
        keep = (_t(off, torch.int32), _t(flat, torch.int32))
        cfg.moveset_off, cfg.moveset = _ptr(keep[0]), _ptr(keep[1])
        if device_keep is not None:
            device_keep.extend(keep)
    return cfg


def auto_shape(nsys, sms=None):
    """(cluster size, speculative teams) MCRunner picks for nsys systems:
    the largest cluster with every system on its own SMs, then up to four
    teams per system while the SMs last (sms: the device's SM count)."""
    if sms is None:
        sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    cl = next((c for c in (16, 8, 4, 2) if nsys * c <= sms), 1)
    k = next(k for k in (4, 2, 1) if k == 1 or k * nsys * cl <= sms)
    return cl, k


class MCRunner:
    """Device MC over every system of `batch`.

    temperatures: kcal/mol, one per system (scalar broadcast).  cur_max0:
    initial max angle (the reference's max_angle).  cluster_size, threads,
    spec_teams: the launch shape (None / 0: chosen from the batch size).
    tail_shape: once some chain has finished and few are left, launch only
    those, on wider clusters and more teams (same chains, fewer idle SMs)."""

    def __init__(self, batch: DeviceBatch, temperatures, seed, policy=0, cur_max0=0.12, tune_freq=200,
                 fixed_delta=0.0, moveset=None, cluster_size=None, threads=0, spec_teams=None, device_rebuild=False,
                 tail_shape=True):
        self.b = batch
        self.L = batch.L
        self._keep = []
        self.cfg = mc_config(seed, policy, tune_freq, fixed_delta=fixed_delta, moveset=moveset, nsys=batch.nsys,
                             device_keep=self._keep)
        auto_cl, auto_k = auto_shape(batch.nsys)
        if cluster_size is None:  # small batches: spread each chain over a cluster of SMs
            cluster_size = auto_cl
        self.cfg.cluster_size = int(cluster_size)
        self.cfg.threads_per_system = int(threads)
        if spec_teams is None:  # up to four speculative teams per system when the SMs are there
            sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
            spec_teams = next(k for k in (4, 2, 1) if k == 1 or k * batch.nsys * int(cluster_size) <= sms)
        self.cfg.spec_teams = int(spec_teams)
        # device_rebuild: a drifted chain rebuilds its list, radii and energy
        # inside the persistent kernel (one-team launches) instead of
        # stopping for the host.  Off by default: one team has a small share
        # of the GPU for the list's 27-cell scan, and on the bench workloads
        # the whole-GPU host rebuild of all flagged chains is faster.
        self.rebuild_ws = None
        if device_rebuild and int(spec_teams) == 1:  # only one-team launches rebuild in the kernel
            self.rebuild_ws = torch.empty(self.L.alma_mc_rebuild_bytes(batch.natoms, batch.nsys), dtype=torch.uint8,
                                          device="cuda")
            self.cfg.rebuild_ws = _ptr(self.rebuild_ws)
        # tail_shape: once at most half the SMs' worth of chains still have
        # proposals to make before the step limit, those chains alone are
        # launched, on wider clusters and more teams (auto_shape of their
        # count), instead of one CTA each beside idle SMs.  The chains are
        # the same: every shape draws and decides the same proposals.
        self.tail_shape = bool(tail_shape) and self.rebuild_ws is None and batch.nsys > 1
        self._sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
        teams_max = max(int(spec_teams), TAIL_MAX_TEAMS if self.tail_shape else 1)
        if teams_max > 1:
            # K teams per system: K move scratches plus the round buffers, team 0
            # at the start (the batch's counters and single-move calls use it)
            need = self.L.alma_mc_scratch_bytes(batch.natoms, batch.nsys, teams_max)
            if batch.scratch.numel() < need:
                batch.scratch = torch.zeros(need, dtype=torch.uint8, device="cuda")
        # largest systems take the first CTAs: when a batch has more systems
        # than resident CTAs, the long chains start first and the short ones
        # fill the SMs they free (the tail of the launch shortens)
        order = np.argsort(-np.diff(batch.atom_off_h), kind="stable").astype(np.int32)
        self._order = _t(order, torch.int32)
        self.cfg.sys_order = _ptr(self._order)
        T = np.broadcast_to(np.asarray(temperatures, np.float64), (batch.nsys,)).copy()
        if np.any(T <= 0):
            raise ValueError("temperature must be positive")
        st = np.zeros(batch.nsys, dtype=_lib.STATE_DTYPE)
        st["cur_max"] = cur_max0
        st["temperature"] = T
        self.states = torch.from_numpy(st.view(np.uint8).copy()).to("cuda")
        self.terms = torch.zeros((batch.nsys, 5), dtype=torch.float64, device="cuda")
        self.rebuilds = 0
        self.tail_launches = 0
        batch.build_nl()
        self.reset_energy()

    def reset_energy(self, sys_mask=None):
        """Full Born radii + energy of the (masked) systems -> state.energy."""
        self.b.energy_terms(recompute_born=True, sys_mask=sys_mask, out=self.terms)
        _lib.check(self.L.alma_mc_after_rebuild(_ptr(self.states), _ptr(self.terms),
                                                _ptr(sys_mask) if sys_mask is not None else None,
                                                self.b.nsys, self.b._sp()), "alma_mc_after_rebuild")

    def state(self):
        return self.states.cpu().numpy().view(_lib.STATE_DTYPE).copy()

    def _run(self, cfg, step_limit):
        b = self.b
        return self.L.alma_mc_run(C.byref(b.batch_s), C.byref(b.topo_s), C.byref(b.nl_s), C.byref(b.params), b.prec,
                                  _ptr(b.scratch), C.byref(cfg), _ptr(self.states), int(step_limit), b._sp())

    def launch(self, step_limit, tail=None):
        """One persistent launch; tail = (order, n, cluster, teams) from
        _tail_plan launches only those chains, in that shape."""
        if tail is not None:
            order, n, cl, k = tail
            cfg = _lib.AlmaMCConfig.from_buffer_copy(self.cfg)
            self._tail_order = _t(order, torch.int32)  # alive until the state read after the launch
            cfg.sys_order, cfg.launch_systems = _ptr(self._tail_order), int(n)
            cfg.cluster_size, cfg.spec_teams, cfg.threads_per_system = int(cl), int(k), 512
            rc = self._run(cfg, step_limit)
            if rc == _lib.ALMA_EINVAL and k > 1 and b"resident" in self.L.alma_last_error():
                cfg.spec_teams = 1
                rc = self._run(cfg, step_limit)
            _lib.check(rc, "alma_mc_run")
            self.tail_launches += 1
            return
        rc = self._run(self.cfg, step_limit)
        if rc == _lib.ALMA_EINVAL and self.cfg.spec_teams > 1 and b"resident" in self.L.alma_last_error():
            self.cfg.spec_teams = 1  # the teams would not all fit on the GPU at once: one team
            return self.launch(step_limit)
        _lib.check(rc, "alma_mc_run")

    def _tail_plan(self, st, step_limit):
        """(order, n, cluster, teams) for the chains still short of
        step_limit, or None when the batch's own shape is the one to use:
        while every chain is left (the shape the caller or the autotuner
        chose for the batch) or more than half the SMs' worth."""
        if not self.tail_shape:
            return None
        active = np.nonzero(st["step"] < step_limit)[0]
        n = len(active)
        if n == 0 or n == len(st) or 2 * n > self._sms:
            return None
        cl, k = auto_shape(n, self._sms)
        size = np.diff(self.b.atom_off_h)[active]
        order = active[np.argsort(-size, kind="stable")].astype(np.int32)
        return order, n, cl, k

    def run(self, nsteps):
        """Advances every system by nsteps proposals (host loop over rebuilds)."""
        target = int(self.state()["step"].max()) + int(nsteps) if nsteps > 0 else 0
        return self.run_to(target)

    def _read_state(self):
        """Chain states and the batch status word in one device-to-host
        transfer (pinned buffer, one synchronisation)."""
        n = self.states.numel()
        if getattr(self, "_host", None) is None:
            self._host = torch.empty(n + 4, dtype=torch.uint8, pin_memory=True)
        s = self.b.stream or torch.cuda.current_stream()
        with torch.cuda.stream(s):
            self._host[:n].copy_(self.states, non_blocking=True)
            self._host[n:].copy_(self.b.status.view(torch.uint8), non_blocking=True)
        s.synchronize()
        h = self._host.numpy()
        return h[:n].view(_lib.STATE_DTYPE).copy(), int(h[n:].view(np.int32)[0])

    def run_to(self, step_limit):
        tail = None
        while True:
            self.launch(step_limit, tail)
            st, status = self._read_state()
            if status & _lib.ST_SPEC_ABORT:
                raise RuntimeError("alma_mc_run: a speculative round timed out (teams not co-resident)")
            # Every drifted chain rebuilds now, also one flagged on its last
            # proposal: the reference rebuilds at the start of the chain's
            # next step (physics_engine.cpp:2506-2510), the same list from the
            # same coordinates, but here the list stays valid for energies
            # taken after the run (n_rebuild counts it at once).
            need = st["need_rebuild"] != 0
            if need.any():
                mask = torch.from_numpy(need.astype(np.uint8)).to(self.states.device)
                self.b.build_nl(sys_mask=mask)
                self.reset_energy(sys_mask=mask)
                self.rebuilds += int(need.sum())
                tail = self._tail_plan(st, step_limit)
                continue
            if np.all(st["step"] >= step_limit):
                return st
            tail = self._tail_plan(st, step_limit)


_TUNED = {}


def autotune(batch, temperatures, seed, policy=0, moveset=None, proposals=200, candidates=None):
    """Picks (cluster_size, threads_per_system, spec_teams) for this batch shape by
    timing `proposals` proposals per candidate, after as many untimed ones
    (the step scale and the acceptance rate, on which the speculative teams'
    gain depends, settle first), on a scratch copy of the batch state;
    cached per (systems, atom-count bucket, policy)."""
    import time
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    key = (batch.nsys, int(np.log2(max(1, batch.natoms // max(1, batch.nsys)))), policy, moveset is not None)
    if key in _TUNED:
        return _TUNED[key]
    if candidates is None:
        candidates = [(cl, nt, 1) for cl in (1, 2, 4, 8, 16) for nt in (256, 512) if batch.nsys * cl <= 2 * sms]
        candidates += [(cl, 512, k) for cl in (8, 16) for k in (2, 4, 8) if batch.nsys * cl * k <= sms]
    xyz0, born0 = batch.xyz.clone(), batch.born.clone()
    best, best_rate = None, -1.0
    for cand in candidates:
        cl, nt, k = (tuple(cand) + (1,))[:3]
        try:
            R = MCRunner(batch, temperatures, seed, policy=policy, moveset=moveset, cluster_size=cl, threads=nt,
                         spec_teams=k)
            R.run(max(10, proposals))
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            R.run(proposals)
            torch.cuda.synchronize()
            rate = proposals * batch.nsys / (time.perf_counter() - t0)
        except (RuntimeError, ValueError):
            continue
        finally:
            batch.xyz.copy_(xyz0)
            batch.born.copy_(born0)
            batch.nl_ready = False
            batch.invalidate_sasa()
        if rate > best_rate:
            best, best_rate = (cl, nt, k), rate
    batch.build_nl()
    _TUNED[key] = best
    return best


def _check_inputs(state, topology):
    if len(state) == 0:
        raise ValueError("initial_state empty")
    if topology is None:
        raise ValueError("topology is required")
    flat = flatten(topology)
    if flat.n != len(state):
        raise ValueError(f"topology has {flat.n} atoms, initial_state {len(state)}")
    if flat.nrb == 0:
        raise ValueError("topology has no rotatable bonds")
    return flat


def generate_ensemble(engine, initial_state, topology, n_candidates, steps_per_cand, temperature=0.6,
                      max_angle=0.12):
    """n_candidates independent chains of steps_per_cand proposals from the
    initial state, run as one batch (one CTA per chain)."""
    flat = _check_inputs(initial_state, topology)
    if n_candidates <= 0 or steps_per_cand <= 0:
        raise ValueError("ncand/steps must be positive")
    xyz, q, r, e = particle_arrays(initial_state)
    if not np.all(np.isfinite(xyz)):
        raise ValueError("non-finite coordinates")
    batch = engine._batch(xyz, q, r, e, flat, copies=int(n_candidates))
    # Several candidates, one team each on 8- or 16-CTA clusters: each chain
    # rebuilds its own list inside the persistent kernel when it drifts
    # instead of idling until the last chain of the launch has drifted too
    # (16 candidates of a 4,962-atom chain: 25.7k -> 32.6k proposals/s).
    cl, k = auto_shape(batch.nsys)
    runner = MCRunner(batch, temperature, engine._next_seed(), policy=0, cur_max0=max_angle, cluster_size=cl,
                      spec_teams=k, device_rebuild=batch.nsys > 1 and k == 1 and cl >= 8)
    runner.run(steps_per_cand)
    X = batch.coords()
    return [particles_from(X[batch.atom_off_h[c]:batch.atom_off_h[c + 1]], initial_state)
            for c in range(int(n_candidates))]


def run_landscape(engine, initial_state, topology, n_snapshots, steps_per_snapshot, temperature=0.6,
                  max_angle=0.12):
    """One landscape chain (policy 1: concerted sidechain pairs, crankshaft,
    torsion); a snapshot and its full energy every steps_per_snapshot
    proposals.  Returns (snapshots, energies, final cur_max)."""
    flat = _check_inputs(initial_state, topology)
    if n_snapshots <= 0 or steps_per_snapshot <= 0:
        raise ValueError("n_snapshots/steps_per_snapshot must be positive")
    xyz, q, r, e = particle_arrays(initial_state)
    if not np.all(np.isfinite(xyz)):
        raise ValueError("non-finite coordinates")
    batch = DeviceBatch([(xyz, q, r, e, flat)], precision=engine.precision)
    runner = MCRunner(batch, temperature, engine._next_seed(), policy=1, cur_max0=max_angle)
    snaps, energies = [], []
    for _ in range(int(n_snapshots)):
        runner.run(steps_per_snapshot)
        X = batch.coords(0)
        snaps.append(particles_from(X, initial_state))
        shot = engine._batch(X, q, r, e, flat)  # calculate_potential of the snapshot: fresh list
        energies.append(float(shot.energy_terms()[0, 4].item()))
    cur_max = float(runner.state()["cur_max"][0])
    return snaps, energies, cur_max


class BatchedEnsemble:
    """Many independent chains — each its own atoms, topology and
    temperature — advanced together by the device MC: the batched form of
    generate_ensemble with one candidate per chain (the reference runs
    such chains one call, or one OpenMP thread, at a time).

    systems: [(xyz [n,3], charge, radius, epsilon, topology), ...] with a
    BondTopology (or its flatten()) per chain; temperatures in kcal/mol
    (scalar broadcast); policy 0 is generate_ensemble's proposal policy.
    The device batch, neighbor lists and launch shape are set up once;
    each run() is one host round trip: coordinates in (optional), steps
    proposals per chain, coordinates out."""

    def __init__(self, systems, temperatures, seed=0, precision="mixed", max_angle=0.12, policy=0, moveset=None,
                 shape=None):
        sys_flat = []
        for x, q, r, e, topo in systems:
            flat = topo if hasattr(topo, "excl_ptr") else flatten(topo)
            if flat.nrb == 0:
                raise ValueError("a chain has no rotatable bonds")
            sys_flat.append((np.asarray(x, np.float64).reshape(-1, 3), q, r, e, flat))
        self.batch = DeviceBatch(sys_flat, precision=precision)
        self.temperatures = np.broadcast_to(np.asarray(temperatures, np.float64), (self.batch.nsys,)).copy()
        self.max_angle = float(max_angle)
        self.policy, self.moveset = int(policy), moveset
        if shape is None:
            cl, k = auto_shape(self.batch.nsys)
            shape = (cl, 0, k)
        self.shape = tuple(shape)
        self.runner = MCRunner(self.batch, self.temperatures, seed, policy=self.policy, cur_max0=self.max_angle,
                               moveset=moveset, cluster_size=self.shape[0], threads=self.shape[1],
                               spec_teams=self.shape[2])
        n = self.batch.natoms
        self._host_in = torch.empty((n, 3), dtype=torch.float64, pin_memory=True)
        self._host_out = torch.empty((n, 3), dtype=torch.float64, pin_memory=True)
        self._dev = torch.empty((n, 3), dtype=torch.float64, device="cuda")

    @property
    def atom_offsets(self):
        return self.batch.atom_off_h.copy()

    def restart(self, xyz):
        """New starting coordinates [natoms, 3] (all chains, concatenated):
        a fresh list, radii and energy per chain, cur_max back to max_angle
        (as every generate_ensemble call starts); the random stream goes on."""
        b = self.batch
        src = xyz if isinstance(xyz, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(xyz, np.float64))
        if src.device.type == "cpu" and not src.is_pinned():
            self._host_in.copy_(src.reshape(b.natoms, 3))
            src = self._host_in
        self._dev.copy_(src.reshape(b.natoms, 3), non_blocking=True)
        b.xyz[:b.natoms, :3].copy_(self._dev)
        b.nl_ready = False
        b.invalidate_sasa()
        b.status.zero_()
        st = self.runner.state()
        st["cur_max"] = self.max_angle
        st["acc_win"] = st["tot_win"] = st["need_rebuild"] = 0
        self.runner.states.copy_(torch.from_numpy(st.view(np.uint8).copy()))
        b.build_nl()
        self.runner.reset_energy()

    def run(self, steps, xyz=None):
        """steps proposals per chain (from xyz when given, else from where
        the last run left the chains); returns the final coordinates
        [natoms, 3] as a host array (split with atom_offsets)."""
        if steps <= 0:
            raise ValueError("steps must be positive")
        if xyz is not None:
            self.restart(xyz)
        self.runner.run(int(steps))
        self._host_out.copy_(self.batch.xyz[:self.batch.natoms, :3], non_blocking=True)
        torch.cuda.current_stream().synchronize()
        return self._host_out.numpy()

    def state(self):
        return self.runner.state()

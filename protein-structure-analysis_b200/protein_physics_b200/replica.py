"""Replica-exchange sampling of one chain on one GPU: every replica is a
system of one DeviceBatch, plain torsion moves (the device MC kernel) and
gradient-guided MALA torsion proposals mixed in a fixed ratio, and a
temperature swap between neighbours (alma_replica_exchange) every
`sweeps_per_exchange` sweeps.

The reference runs its tempering ladder as Python threads over
run_landscape_segment and swaps on the host (gui_main.py:1960-2013); here
all replicas advance in the same launches and the swap is one kernel over
fresh energies.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .device import DeviceBatch, _ptr
from .mc import K_BOLTZMANN, MCRunner
from .torsion import MALARunner, TorsionSpace, minimize


def geometric_ladder(t_lo_K, t_hi_K, n):
    """n temperatures (K) spaced geometrically from t_lo to t_hi."""
    if n == 1:
        return np.array([float(t_lo_K)])
    return float(t_lo_K) * (float(t_hi_K) / float(t_lo_K)) ** (np.arange(n) / (n - 1))


class ReplicaExchange:
    """system: (xyz, charge, radius, epsilon, FlatTopology); temps_K: the
    ladder (ascending).  mala_fraction of the proposals of a sweep are MALA
    proposals (1:3 -> 0.25), the rest plain torsion moves (policy 2, moves
    restricted to `moveset` when given)."""

    def __init__(self, system, temps_K, seed, mala_fraction=0.25, mala_step=np.radians(0.5), moveset=None,
                 precision="mixed", minimize_steps=0, mala_warmup=0, cluster_size=None, threads=0):
        temps_K = np.asarray(temps_K, np.float64)
        if np.any(np.diff(temps_K) < 0):
            raise ValueError("temperatures must ascend")
        self.R = len(temps_K)
        self.batch = DeviceBatch([system] * self.R, precision=precision)
        self.ts = TorsionSpace(self.batch)
        if minimize_steps:
            minimize(self.batch, steps=minimize_steps, ts=self.ts)
        T = temps_K * K_BOLTZMANN
        ms = [moveset] * self.R if moveset is not None else None
        self.mc = MCRunner(self.batch, T, seed, policy=2, moveset=ms, cluster_size=cluster_size, threads=threads)
        self.mala = MALARunner(self.batch, T, seed + 1, step=mala_step, ts=self.ts)
        if mala_warmup:  # let the MALA step scale adapt before sampling starts
            self.mala.run(int(mala_warmup))
        self.mala_fraction = float(mala_fraction)
        self.seed = int(seed) & ((1 << 64) - 1)
        self.sys_of_temp = torch.arange(self.R, dtype=torch.int32, device="cuda")
        self.attempts = torch.zeros(self.R, dtype=torch.int64, device="cuda")
        self.accepts = torch.zeros(self.R, dtype=torch.int64, device="cuda")
        self.terms = torch.zeros((self.R, 5), dtype=torch.float64, device="cuda")
        self.round = 0
        self.proposals = 0

    def interval(self, sweeps):
        """sweeps sweeps (one proposal per replica each), then one exchange
        round.  Returns the proposals made (all replicas)."""
        b = self.batch
        n_mala = int(round(sweeps * self.mala_fraction))
        n_tors = int(sweeps) - n_mala
        if n_mala:
            self.mala.refresh()
            for _ in range(n_mala):
                self.mala.step()
        if n_tors:
            b.build_nl()
            self.mc.reset_energy()
            self.mc.run(n_tors)
        b.nl_ready = False
        b.energy_terms(recompute_born=True, out=self.terms)
        _lib.check(b.L.alma_replica_exchange(self.R, _ptr(self.terms), _ptr(self.mc.states),
                                             _ptr(self.mala.states), _ptr(self.sys_of_temp), self.seed,
                                             self.round, _ptr(self.attempts), _ptr(self.accepts), b._sp()),
                   "alma_replica_exchange")
        self.round += 1
        self.proposals += self.R * int(sweeps)
        return self.R * int(sweeps)

    def run(self, n_intervals, sweeps_per_exchange=100):
        for _ in range(int(n_intervals)):
            self.interval(sweeps_per_exchange)
        return self.stats()

    def stats(self):
        att = self.attempts.cpu().numpy()
        acc = self.accepts.cpu().numpy()
        mc = self.mc.state()
        ml = self.mala.state()
        pairs = slice(0, self.R - 1)
        return {"exchange_acceptance": float(acc[pairs].sum() / max(1, att[pairs].sum())),
                "pair_acceptance": (acc[pairs] / np.maximum(1, att[pairs])).tolist(),
                "torsion_acceptance": float(mc["n_accepted"].sum() / max(1, mc["n_proposed"].sum())),
                "mala_acceptance": float(ml["n_accepted"].sum() / max(1, ml["n_proposed"].sum())),
                "temperature_of_system_K": (mc["temperature"] / K_BOLTZMANN).tolist(),
                "sys_of_temp": self.sys_of_temp.cpu().numpy().tolist()}

"""Benchmark inputs that need the device, and their files.

The compact chains of the benchmark configurations are finished on the
device: a coil chain is collapsed on the host (synth.collapse, a bead
model), then relaxed here with the full energy plus a radius-of-gyration
restraint k (Rg - target)^2 over all atoms:

1. torsion-space descent (every rotatable bond at once, the analytic
   gradient of alma_forces projected on the torsions by alma_torsion_grad,
   each bond's step scaled by the inverse inertia of its moving side),
   with +-120 degree rotamer jumps tried every 250 steps on sidechain bonds
   that move a clashing atom, and every 1,000 steps a search over all well
   combinations of the first three chis of each residue holding a
   clashing atom; this clears the clashes the bead model leaves;
2. seeded Metropolis moves at 300 K (single-bond torsion moves with the
   reference's step rule: uniform in +-cur_max x lever scale, x2.5 for
   sidechain bonds, cur_max adapted to 28-52 % acceptance), each scored
   by a full energy on a fresh neighbor list plus the restraint.

``save_chain`` / ``load_chain`` keep a chain in an .npz of plain arrays
(coordinates, charges, radii, epsilons, names, residue indices), which
numpy alone can read back.
"""
from __future__ import annotations

import itertools
import math

import numpy as np

from . import synth

K_BOLTZMANN = 0.0019872  # kcal mol^-1 K^-1


def save_chain(path, ch, **meta):
    np.savez_compressed(path, xyz=np.asarray(ch.xyz, np.float64), charge=ch.charge, radius=ch.radius,
                        epsilon=ch.epsilon, resnames=np.array(ch.resnames), atomnames=np.array(ch.atomnames),
                        res_idx=np.asarray(ch.res_idx, np.int32), sequence=np.array(ch.sequence),
                        **{k: np.asarray(v) for k, v in meta.items()})


def load_chain(path):
    d = np.load(path, allow_pickle=False)
    ch = synth.Chain(d["xyz"].astype(np.float64), d["charge"], d["radius"], d["epsilon"],
                     [str(x) for x in d["resnames"]], [str(x) for x in d["atomnames"]],
                     [int(x) for x in d["res_idx"]], [str(x) for x in d["sequence"]])
    ch.meta = {k: d[k] for k in d.files if k not in ("xyz", "charge", "radius", "epsilon", "resnames",
                                                     "atomnames", "res_idx", "sequence")}
    return ch


class _Restrained:
    """Energy + k sum_g (Rg_g - target)^2 of one chain in a DeviceBatch
    (groups: atom index ranges, one Rg term each), with its torsion
    gradient."""

    def __init__(self, batch, ts, k_rg, rg_target, groups):
        import torch
        self.b, self.ts, self.k, self.t = batch, ts, float(k_rg), float(rg_target)
        self.groups = groups
        n = batch.natoms
        self.terms = torch.zeros((1, 5), dtype=torch.float64, device="cuda")
        self.grad = torch.zeros((n, 4), dtype=torch.float64, device="cuda")
        self.g = torch.zeros(max(ts.nrb, 1), dtype=torch.float64, device="cuda")

    def rgs(self):
        out = []
        for a0, a1 in self.groups:
            x = self.b.xyz[a0:a1, :3]
            d = x - x.mean(0)
            out.append(((d * d).sum(1).mean().sqrt(), d))
        return out

    def rg(self):
        return [float(r) for r, _ in self.rgs()]

    def energy(self, with_grad=True):
        b = self.b
        b.nl_ready = False
        b.build_nl(check=True)
        b.energy_terms(recompute_born=True, out=self.terms)
        E = self.terms[0, 4]
        if with_grad:
            b.forces(out=self.grad)
        for (a0, a1), (rg, d) in zip(self.groups, self.rgs()):
            E = E + self.k * (rg - self.t) ** 2
            if with_grad:
                self.grad[a0:a1, :3] += (2.0 * self.k * (rg - self.t) / ((a1 - a0) * rg)) * d
        if with_grad:
            self.ts.gtheta(self.grad, out=self.g)
        return E


def _side_inertia(x, F):
    """I_k = sum over bond k's moving side of the squared distance to its
    axis: the rigid-body scale of a torsion step (prefix sums over the
    side's atom range plus its explicit atoms)."""
    i, j = np.asarray(F.rb_i), np.asarray(F.rb_j)
    u = x[j] - x[i]
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    a = x[i]
    # |(x - a) x u|^2 = |x|^2 - 2 x.a + |a|^2 - ((x - a).u)^2, summed with prefix sums of x, xx^T, |x|^2
    X2 = np.concatenate([[0.0], np.cumsum((x * x).sum(1))])
    X1 = np.concatenate([np.zeros((1, 3)), np.cumsum(x, 0)])
    XX = np.concatenate([np.zeros((1, 3, 3)), np.cumsum(x[:, :, None] * x[:, None, :], 0)])
    lo, hi = np.asarray(F.side_lo, np.int64), np.asarray(F.side_hi, np.int64)
    hi = np.maximum(hi, lo)
    n = (hi - lo).astype(np.float64)
    s2, s1, sxx = X2[hi] - X2[lo], X1[hi] - X1[lo], XX[hi] - XX[lo]
    ptr = np.asarray(F.side_ptr, np.int64)
    idx = np.asarray(F.side_idx, np.int64)
    owner = np.repeat(np.arange(len(i)), np.diff(ptr))
    np.add.at(n, owner, 1.0)
    np.add.at(s2, owner, (x[idx] * x[idx]).sum(1))
    np.add.at(s1, owner, x[idx])
    np.add.at(sxx, owner, x[idx][:, :, None] * x[idx][:, None, :])
    ua = (a * u).sum(1)
    # sum ((x - a).u)^2 = u^T Sxx u - 2 (a.u)(S1.u) + n (a.u)^2
    par = np.einsum("ki,kij,kj->k", u, sxx, u) - 2.0 * ua * (s1 * u).sum(1) + n * ua * ua
    tot = s2 - 2.0 * (s1 * a).sum(1) + n * (a * a).sum(1)
    return np.maximum(tot - par, 1.0)


def _clashing_atoms(x, F, radius, ratio=1.6):
    """Atoms in a non-excluded pair closer than (R*_i + R*_j) / ratio."""
    from scipy.spatial import cKDTree
    pr = cKDTree(x).query_pairs(2.0 * float(radius.max()) / ratio, output_type="ndarray")
    if len(pr) == 0:
        return np.zeros(len(x), bool)
    i, j = pr.min(1), pr.max(1)
    d = np.linalg.norm(x[i] - x[j], axis=1)
    close = d * ratio < radius[i] + radius[j]
    i, j = i[close], j[close]
    ptr, cols = np.asarray(F.excl_ptr), np.asarray(F.excl_cols)
    keys = set((np.repeat(np.arange(len(ptr) - 1), np.diff(ptr)).astype(np.int64) * len(x) + cols).tolist())
    bad = np.array([k not in keys for k in (i.astype(np.int64) * len(x) + j).tolist()], bool)
    out = np.zeros(len(x), bool)
    out[i[bad]] = True
    out[j[bad]] = True
    return out


def relax(ch, rg_target, k_rg=200.0, descent_steps=4000, mc_moves=2000, temperature_K=300.0, seed=0,
          precision="mixed", domains=None):
    """Device relaxation of a collapsed chain (module docstring); returns a
    new Chain and a dict of what it did.  domains: residue ranges
    [(r0, r1), ...] with one Rg term each (default: the whole chain)."""
    import torch
    from .device import DeviceBatch
    from .topology import BondTopology, flatten
    from .torsion import TorsionSpace
    T = BondTopology()
    T.build(ch.resnames, ch.atomnames, ch.res_idx)
    F = flatten(T)
    b = DeviceBatch([(ch.xyz, ch.charge, ch.radius, ch.epsilon, F)], precision=precision)
    ts = TorsionSpace(b)
    ridx = np.asarray(ch.res_idx)
    groups = [(int(np.searchsorted(ridx, r0)), int(np.searchsorted(ridx, r1))) for r0, r1 in domains] if domains \
        else [(0, b.natoms)]
    R = _Restrained(b, ts, k_rg, rg_target, groups)
    info = {"rg_start": R.rg()}
    xyz_old, born_old = torch.empty_like(b.xyz), torch.empty_like(b.born)
    # 1) descent along -g / I (rigid-body scaled torsion steps: a bond
    # that swings half the chain takes a step its inertia allows), the
    # largest torsion change eta; rotamer jumps for locked sidechain clashes
    E = float(R.energy())
    info["E_start"] = E
    g_cur = R.g.clone()
    eta = 0.05
    nb = ts.nrb
    kinds = np.asarray(F.rb_kind)
    jumps = repacked = 0
    chis = {}  # residue -> its sidechain bonds, in topology order (chi1 first)
    for k in np.flatnonzero(kinds == 2):
        chis.setdefault(int(ridx[int(F.rb_i[k])]), []).append(int(k))
    for it in range(int(descent_steps)):
        if it % 50 == 0:
            inv_I = torch.as_tensor(1.0 / _side_inertia(b.coords(0), F), device="cuda")
        if it % 1000 == 500:  # rotamer search: every well combination of a clashing residue's first three chis
            x = b.coords(0)
            bad = _clashing_atoms(x, F, np.asarray(ch.radius), ratio=1.5)
            for r in sorted(set(ridx[bad].tolist())):
                ks = chis.get(r, [])[:3]
                if not ks:
                    continue
                best = None
                for combo in itertools.product((0.0, 2.0 * math.pi / 3.0, -2.0 * math.pi / 3.0), repeat=len(ks)):
                    if not any(combo):
                        continue
                    xyz_old.copy_(b.xyz)
                    born_old.copy_(b.born)
                    step = torch.zeros(max(nb, 1), dtype=torch.float64, device="cuda")
                    for k, a in zip(ks, combo):
                        step[k] = a
                    ts.apply(step)
                    En = float(R.energy(with_grad=False))
                    b.xyz.copy_(xyz_old)
                    b.born.copy_(born_old)
                    b.invalidate_sasa()
                    if math.isfinite(En) and En < E and (best is None or En < best[0]):
                        best = (En, step)
                if best is not None:
                    ts.apply(best[1])
                    E = best[0]
                    repacked += 1
            E = float(R.energy())
            g_cur = R.g.clone()
        elif it % 250 == 125:  # rotamer jumps: +-120 deg on sidechain bonds that move a clashing atom
            x = b.coords(0)
            bad = _clashing_atoms(x, F, np.asarray(ch.radius))
            for k in np.flatnonzero(kinds == 2):
                lo, hi = int(F.side_lo[k]), int(F.side_hi[k])
                side = np.concatenate([np.arange(lo, max(lo, hi)), F.side_idx[F.side_ptr[k]:F.side_ptr[k + 1]]])
                if not bad[side].any():
                    continue
                best = None
                for jump in (2.0 * math.pi / 3.0, -2.0 * math.pi / 3.0):
                    xyz_old.copy_(b.xyz)
                    born_old.copy_(b.born)
                    step = torch.zeros(max(nb, 1), dtype=torch.float64, device="cuda")
                    step[k] = jump
                    ts.apply(step)
                    En = float(R.energy(with_grad=False))
                    b.xyz.copy_(xyz_old)
                    b.born.copy_(born_old)
                    b.invalidate_sasa()
                    if math.isfinite(En) and En < E and (best is None or En < best[0]):
                        best = (En, jump)
                if best is not None:
                    step = torch.zeros(max(nb, 1), dtype=torch.float64, device="cuda")
                    step[k] = best[1]
                    ts.apply(step)
                    E = best[0]
                    jumps += 1
            E = float(R.energy())
            g_cur = R.g.clone()
        g = g_cur[:nb] * inv_I
        delta = -(eta / max(float(g.abs().max()), 1e-300)) * g
        xyz_old.copy_(b.xyz)
        born_old.copy_(b.born)
        ts.apply(delta)
        En = float(R.energy())
        if math.isfinite(En) and En < E:
            E, g_cur = En, R.g.clone()
            eta = min(eta * 1.2, 0.5)
        else:
            b.xyz.copy_(xyz_old)
            b.born.copy_(born_old)
            b.invalidate_sasa()
            eta = max(eta * 0.5, 1e-6)
    info["E_descent"] = E
    info["rotamer_jumps"] = jumps
    info["residues_repacked"] = repacked
    info["rg_descent"] = R.rg()
    # 2) restrained Metropolis moves (reference step rule, one bond a move)
    rng = np.random.default_rng(seed)
    beta = 1.0 / (K_BOLTZMANN * temperature_K)
    cur_max = 0.12
    lever = np.asarray(F.rb_scale, np.float64)
    side = np.asarray(F.rb_kind) == 2  # sidechain bonds take 2.5x steps
    E = float(R.energy(with_grad=False))
    acc_window = acc = 0
    delta = torch.zeros(max(nb, 1), dtype=torch.float64, device="cuda")
    for m in range(int(mc_moves)):
        k = int(rng.integers(0, nb))
        step = cur_max * lever[k] * (2.5 if side[k] else 1.0)
        d = float(rng.uniform(-step, step))
        xyz_old.copy_(b.xyz)
        born_old.copy_(b.born)
        delta.zero_()
        delta[k] = d
        ts.apply(delta)
        En = float(R.energy(with_grad=False))
        dE = En - E
        if math.isfinite(En) and (dE < 0 or rng.random() < math.exp(-beta * dE)):
            E = En
            acc += 1
            acc_window += 1
        else:
            b.xyz.copy_(xyz_old)
            b.born.copy_(born_old)
            b.invalidate_sasa()
        if (m + 1) % 200 == 0:  # the reference's adaptation window and band
            rate = acc_window / 200.0
            cur_max = min(cur_max * 1.06, 0.5) if rate > 0.52 else max(cur_max * 0.94, 0.004) if rate < 0.28 \
                else cur_max
            acc_window = 0
    E = float(R.energy(with_grad=False))  # the final state's terms (the last proposal may have been undone)
    info.update(E_end=E, rg_end=R.rg(), mc_accept=acc / max(1, int(mc_moves)), cur_max=cur_max,
                E_physical=float(R.terms[0, 4]))
    out = synth.Chain(b.coords(0).copy(), ch.charge, ch.radius, ch.epsilon, ch.resnames, ch.atomnames, ch.res_idx,
                      ch.sequence)
    b.nl_ready = False
    b.build_nl()
    info["full_row_mean"] = float(b.full_len[:b.natoms].double().mean())
    info["half_row_mean"] = float(b.half_len[:b.natoms].double().mean())
    return out, info

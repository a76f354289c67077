"""Torsion space on the device: the torsion gradient of the analytic forces,
all-bond torsion moves, descent minimisation and the Langevin (MALA)
torsion sampler.

The reference samples torsions one or two at a time with uniform steps
(physics_engine.cpp:2328-2501).  These drivers use the backward kernel
(alma_forces) instead: dE/dθ for every rotatable bond from one pass
(alma_torsion_grad), all bonds turned at once (alma_torsion_apply), and
each proposal's energy recomputed from a fresh neighbor list — the
reference's calculate_potential semantics.

Per proposal on the device, no host round trip except the list's overflow
check: save (x, born) -> propose -> apply -> list -> Born + energy ->
forces -> torsion gradient -> accept -> select.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .device import DeviceBatch, _ptr, _t

_i32p = C.POINTER(C.c_int32)


def _np_ptr(a):
    return a.ctypes.data if a.size else None


def torsion_tree(flat):
    """(rb_parent [nrb], atom_rb [n]) of one system (local indices) from its
    FlatTopology j-sides (alma_torsion_tree)."""
    L = _lib.lib()
    n, nrb = int(flat.n), int(flat.nrb)
    rb_ij = np.ascontiguousarray(np.stack([flat.rb_i, flat.rb_j], 1).reshape(-1), np.int32)
    side_ptr = np.ascontiguousarray(flat.side_ptr, np.int64)
    side_idx = np.ascontiguousarray(flat.side_idx, np.int32)
    has = np.asarray(flat.side_hi) > np.asarray(flat.side_lo)
    lo = np.ascontiguousarray(np.where(has, flat.side_lo, 0), np.int32)
    hi = np.ascontiguousarray(np.where(has, flat.side_hi, 0), np.int32)
    parent = np.zeros(max(nrb, 1), np.int32)
    atom_rb = np.zeros(max(n, 1), np.int32)
    rc = L.alma_torsion_tree(n, nrb, _np_ptr(rb_ij), side_ptr.ctypes.data, _np_ptr(side_idx), _np_ptr(lo),
                             _np_ptr(hi), parent.ctypes.data, atom_rb.ctypes.data)
    _lib.check(rc, "alma_torsion_tree")
    return parent[:nrb], atom_rb[:n]


class TorsionSpace:
    """Torsion-space view of a DeviceBatch (every system needs a topology)."""

    def __init__(self, batch: DeviceBatch):
        if not all(batch.has_topo):
            raise ValueError("torsion space needs a topology for every system")
        self.b = batch
        self.L = batch.L
        parents, atom_rbs = [], []
        for T in batch.topos:
            p, a = torsion_tree(T)
            parents.append(p)
            atom_rbs.append(a)
        self.nrb = int(batch.rb_off_h[-1])
        self.rb_parent = _t(np.concatenate(parents) if self.nrb else np.zeros(1, np.int32), torch.int32)
        self.atom_rb = _t(np.concatenate(atom_rbs), torch.int32)
        self.tree = _lib.AlmaTorsionTree(_ptr(self.rb_parent), _ptr(self.atom_rb))
        self.ws = torch.zeros(self.L.alma_torsion_workspace_bytes(batch.natoms, batch.nsys, self.nrb),
                              dtype=torch.uint8, device="cuda")
        self.bond_sys = torch.as_tensor(np.repeat(np.arange(batch.nsys), np.diff(batch.rb_off_h)),
                                        dtype=torch.int64, device="cuda")
        cnt = np.diff(batch.rb_off_h)
        self.max_nrb = int(max(1, cnt.max()))
        self.nrb_sys = torch.as_tensor(cnt, dtype=torch.float64, device="cuda")
        self.bond_local = torch.as_tensor(np.arange(self.nrb) - np.repeat(batch.rb_off_h[:-1], cnt),
                                          dtype=torch.int64, device="cuda")

    def gtheta(self, grad, out=None, sys_mask=None):
        """dE/dθ [nrb] from a [natoms, 4] gradient."""
        out = out if out is not None else torch.zeros(max(self.nrb, 1), dtype=torch.float64, device="cuda")
        b = self.b
        _lib.check(self.L.alma_torsion_grad(C.byref(b.batch_s), C.byref(b.topo_s), _ptr(grad),
                                            _ptr(sys_mask) if sys_mask is not None else None, _ptr(self.ws),
                                            _ptr(out), b._sp()), "alma_torsion_grad")
        return out

    def apply(self, delta, sys_mask=None):
        """Turns every bond k by delta[k] (radians) in place."""
        b = self.b
        _lib.check(self.L.alma_torsion_apply(C.byref(b.batch_s), C.byref(b.topo_s), C.byref(self.tree),
                                             _ptr(delta), _ptr(sys_mask) if sys_mask is not None else None,
                                             _ptr(self.ws), b._sp()), "alma_torsion_apply")
        b.nl_ready = False
        b.invalidate_sasa()

    def select(self, accept, xyz_old, born_old, g_new=None, g_cur=None, sys_mask=None):
        b = self.b
        _lib.check(self.L.alma_mala_select(C.byref(b.batch_s), C.byref(b.topo_s), _ptr(accept),
                                           _ptr(sys_mask) if sys_mask is not None else None, _ptr(xyz_old),
                                           _ptr(born_old), _ptr(g_new), _ptr(g_cur), b._sp()),
                   "alma_mala_select")
        b.invalidate_sasa()  # rejected systems went back to their saved coordinates


class _Eval:
    """Energy, gradient and torsion gradient at the batch's coordinates."""

    def __init__(self, ts: TorsionSpace):
        self.ts = ts
        self.check = True  # the list's overflow check (a host sync; off inside a CUDA graph)
        b = ts.b
        self.terms = torch.zeros((b.nsys, 5), dtype=torch.float64, device="cuda")
        self.grad = torch.zeros((max(b.natoms, 1), 4), dtype=torch.float64, device="cuda")
        self.g = torch.zeros(max(ts.nrb, 1), dtype=torch.float64, device="cuda")

    def __call__(self):
        b = self.ts.b
        b.nl_ready = False
        b.build_nl(check=self.check)
        b.energy_terms(recompute_born=True, out=self.terms)
        b.forces(out=self.grad)
        self.ts.gtheta(self.grad, out=self.g)
        return self


def minimize(batch: DeviceBatch, steps=500, step0=0.02, grow=1.2, shrink=0.5, step_bounds=(1e-6, 0.3),
             clip=3.0, ts: TorsionSpace | None = None):
    """Descent in torsion space along d = -clip(g, ±clip·mean|g|) (per
    system; clip <= 0: plain steepest descent), scaled so the largest
    torsion change is eta_s radians.  Clipping lets every bond caught in
    a clash move at once instead of only the steepest one.  A step that
    lowers the energy is kept and eta_s grows, otherwise it is undone and
    eta_s shrinks.  Runs on the device without host syncs except the
    neighbor list's overflow check.  Returns the energies [steps + 1,
    nsys] (device) and the final eta."""
    ts = ts or TorsionSpace(batch)
    b = batch
    cur = _Eval(ts)()
    E = cur.terms[:, 4].clone()
    g_cur = cur.g.clone()
    new = _Eval(ts)
    eta = torch.full((b.nsys,), float(step0), dtype=torch.float64, device="cuda")
    xyz_old = torch.empty_like(b.xyz)
    born_old = torch.empty_like(b.born)
    hist = [E.clone()]
    nb = ts.nrb
    for _ in range(int(steps)):
        if nb == 0:
            break
        g = g_cur[:nb]
        if clip > 0:  # per-system mean |g|: rows of a padded [nsys, max bonds] matrix (no atomics)
            pad = g.new_zeros((b.nsys, ts.max_nrb))
            pad[ts.bond_sys, ts.bond_local] = g.abs()
            mean = pad.sum(1) / torch.clamp(ts.nrb_sys, min=1.0)
            lim = (clip * mean)[ts.bond_sys]
            g = torch.maximum(torch.minimum(g, lim), -lim)
        gmax = torch.zeros(b.nsys, dtype=torch.float64, device="cuda").scatter_reduce(
            0, ts.bond_sys, g.abs(), reduce="amax", include_self=True)
        scale = eta / torch.clamp(gmax, min=1e-300)
        delta = -(scale[ts.bond_sys] * g)
        xyz_old.copy_(b.xyz)
        born_old.copy_(b.born)
        ts.apply(delta)
        new()
        En = new.terms[:, 4]
        acc = (En < E) & torch.isfinite(En)
        ts.select(acc.to(torch.uint8), xyz_old, born_old, g_new=new.g, g_cur=g_cur)
        E = torch.where(acc, En, E)
        eta = torch.where(acc, eta * grow, eta * shrink).clamp(*step_bounds)
        hist.append(E.clone())
    b.nl_ready = False
    return torch.stack(hist), eta


def mala_config(seed, drift_clip=0.1, tune_freq=20, target=(0.4, 0.7), scale_up=1.1, scale_down=0.8,
                scale_bounds=(1e-3, 4.0)):
    """AlmaMalaConfig: truncated drift at ±drift_clip·σ; every tune_freq
    proposals (0: never) the step scale grows / shrinks when the window's
    acceptance leaves the target band (as the reference adapts cur_max,
    physics_engine.cpp:2515-2526)."""
    cfg = _lib.AlmaMalaConfig()
    cfg.seed = int(seed) & ((1 << 64) - 1)
    cfg.drift_clip = float(drift_clip)
    cfg.tune_freq = int(tune_freq)
    cfg.target_lo, cfg.target_hi = target
    cfg.scale_up, cfg.scale_down = scale_up, scale_down
    cfg.scale_min, cfg.scale_max = scale_bounds
    return cfg


class MALARunner:
    """Metropolis-adjusted Langevin proposals in torsion space for every
    system of a batch: all rotatable bonds move at once by
    clip(-½ σ_k² β dE/dθ_k, ±clip σ_k) + σ_k ξ_k with σ_k = scale × step ×
    the bond's lever scale (sidechain bonds × sidechain_mult), accepted by
    Metropolis–Hastings.

    temperatures: kcal/mol per system (scalar broadcast).  drift_clip:
    the drift's truncation in units of σ; at 0.1 a dense chain's steep
    contacts, whose drift is clipped both ways, cost log α about 0.02 per
    bond instead of about 2 at 1.0."""

    def __init__(self, batch: DeviceBatch, temperatures, seed, step=np.radians(0.5), sidechain_mult=2.5,
                 drift_clip=0.1, tune_freq=20, ts: TorsionSpace | None = None):
        self.b = batch
        self.ts = ts or TorsionSpace(batch)
        self.cfg = mala_config(seed, drift_clip=drift_clip, tune_freq=tune_freq)
        T = np.broadcast_to(np.asarray(temperatures, np.float64), (batch.nsys,)).copy()
        if np.any(T <= 0):
            raise ValueError("temperature must be positive")
        st = np.zeros(batch.nsys, dtype=_lib.MALA_STATE_DTYPE)
        st["beta"] = 1.0 / T
        st["scale"] = 1.0
        self.states = torch.from_numpy(st.view(np.uint8).copy()).to("cuda")
        kind = batch.rb_kind_h
        sig = float(step) * batch.rb_scale_h * np.where(kind == 2, sidechain_mult, 1.0)
        sig = np.where(kind == 3, 0.0, sig)  # fixed bonds never move
        self.sigma = _t(sig if sig.size else np.zeros(1), torch.float64)
        self.cur = _Eval(self.ts)
        self.new = _Eval(self.ts)
        self.delta = torch.zeros_like(self.cur.g)
        self.accept = torch.zeros(batch.nsys, dtype=torch.uint8, device="cuda")
        self.xyz_old = torch.empty_like(batch.xyz)
        self.born_old = torch.empty_like(batch.born)
        self._graph = None
        self._graph_capture = False
        self.refresh()

    def refresh(self):
        """Energy and torsion gradient of the current coordinates (after the
        coordinates changed outside the sampler, e.g. plain torsion moves)."""
        self.cur()
        st = self.state()
        st["energy"] = self.cur.terms[:, 4].cpu().numpy()
        self.states.copy_(torch.from_numpy(st.view(np.uint8).copy()))

    def set_temperatures(self, temperatures):
        st = self.state()
        st["beta"] = 1.0 / np.broadcast_to(np.asarray(temperatures, np.float64), (self.b.nsys,))
        self.states.copy_(torch.from_numpy(st.view(np.uint8).copy()))

    def state(self):
        return self.states.cpu().numpy().view(_lib.MALA_STATE_DTYPE).copy()

    def step(self):
        b, ts, L = self.b, self.ts, self.b.L
        self.new.check = self._graph_capture is False
        topo, cfg = C.byref(b.topo_s), C.byref(self.cfg)
        _lib.check(L.alma_mala_propose(topo, b.nsys, _ptr(self.cur.g), _ptr(self.sigma), cfg, _ptr(self.states),
                                       None, _ptr(self.delta), b._sp()), "alma_mala_propose")
        self.xyz_old.copy_(b.xyz)
        self.born_old.copy_(b.born)
        ts.apply(self.delta)
        self.new()
        _lib.check(L.alma_mala_accept(topo, b.nsys, _ptr(self.delta), _ptr(self.cur.g), _ptr(self.new.g),
                                      _ptr(self.sigma), _ptr(self.new.terms), cfg, None, _ptr(self.states),
                                      _ptr(self.accept), b._sp()), "alma_mala_accept")
        ts.select(self.accept, self.xyz_old, self.born_old, g_new=self.new.g, g_cur=self.cur.g)
        b.nl_ready = False

    def run(self, n, graph=False, chunk=64):
        """n proposals.  graph=True replays one captured CUDA graph per
        proposal (no host work between proposals); the list's overflow
        check then runs once per chunk, and a chunk that overflowed is
        undone and redone eagerly (which grows the list regions)."""
        if not graph:
            for _ in range(int(n)):
                self.step()
            return self.state()
        done = 0
        while done < n:
            k = min(int(chunk), int(n) - done)
            if self._graph is None:
                self._capture()
            snap = [t.clone() for t in (self.b.xyz, self.b.born, self.states, self.cur.g)]
            for _ in range(k):
                self._graph.replay()
            if int(self.b.status.item()) & (_lib.ST_NL_OVERFLOW | _lib.ST_CELL_OVERFLOW):
                for dst, src in zip((self.b.xyz, self.b.born, self.states, self.cur.g), snap):
                    dst.copy_(src)
                self.b.status.zero_()
                self.b.invalidate_sasa()
                self._graph = None
                for _ in range(k):
                    self.step()
            done += k
        self.b.nl_ready = False
        self.b.invalidate_sasa()
        return self.state()

    def _chain_tensors(self):
        return (self.b.xyz, self.b.born, self.states, self.cur.g)

    def _capture(self):
        # the warm-up steps make every buffer exist before the capture; the
        # chain is put back afterwards, so replays are its only proposals
        snap = [t.clone() for t in self._chain_tensors()]
        self.step()
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            self.step()
        torch.cuda.current_stream().wait_stream(side)
        g = torch.cuda.CUDAGraph()
        self._graph_capture = True
        try:
            with torch.cuda.graph(g):
                self.step()
        finally:
            self._graph_capture = False
        for dst, src in zip(self._chain_tensors(), snap):
            dst.copy_(src)
        self._graph = g

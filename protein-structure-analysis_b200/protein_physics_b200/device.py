"""Device-resident batches of systems and the calls into the C ABI.

A ``DeviceBatch`` holds one or more independent systems (chains or
temperature replicas) concatenated atom-wise in HBM:

  xyz    float64 [natoms, 4]  master coordinates (x, y, z, unused)
  prm    float32 [natoms, 4]  charge, R*, epsilon (pair arithmetic, mixed mode)
  prm64  float64 [natoms, 4]  the same in FP64 (SASA, Born finalisation)
  born   float64 [natoms]     effective Born radii
  topology arrays with global atom indices, neighbor-list regions per system

Torch only allocates memory and supplies the stream; all arithmetic runs in
libalma_b200.so.  There is no CPU fallback: without a CUDA device the
constructor raises.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from .topology import FlatTopology

_DEV = "cuda"


def _require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("protein_physics_b200 needs a CUDA device (sm_100); none is available")


def _t(a, dtype):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype).to(_DEV, non_blocking=False)


def _ptr(t):
    return t.data_ptr() if t is not None and t.numel() > 0 else None


def _empty_topo(n):
    return FlatTopology(
        n=n, excl_ptr=np.zeros(n + 1, np.int64), excl_cols=np.zeros(0, np.int32),
        rb_i=np.zeros(0, np.int32), rb_j=np.zeros(0, np.int32), rb_kind=np.zeros(0, np.int32),
        rb_scale=np.zeros(0), side_ptr=np.zeros(1, np.int64), side_idx=np.zeros(0, np.int32),
        side_lo=np.zeros(0, np.int32), side_hi=np.zeros(0, np.int32), side_count=np.zeros(0, np.int64),
        dih_abcd=np.zeros((0, 4), np.int32), term_off=np.zeros(1, np.int32), term_v2=np.zeros(0),
        term_n=np.zeros(0, np.int32), term_gamma=np.zeros(0), ss=np.zeros((0, 2), np.int32),
        crank=np.zeros((0, 2), np.int32), conc_sc=np.zeros((0, 2), np.int32))


class DeviceBatch:
    """A batch of systems on the device.

    systems: list of (xyz [n,3], charge [n], radius [n], epsilon [n],
    FlatTopology or None).  A None topology means no exclusions, dihedrals
    or disulfides (the reference's calculate_potential without topology)."""

    NL_FULL_PER_ATOM = 640   # first-build capacity guesses (entries / atom)
    NL_HALF_PER_ATOM = 330
    NL_SHORT_PER_ATOM = 200

    def __init__(self, systems, precision="mixed", stream=None):
        _require_cuda()
        self.L = _lib.lib()
        self.prec = _lib.PREC_FP64 if precision == "fp64" else _lib.PREC_MIXED
        self.stream = stream  # None: launch on torch's current stream (graph capture included)
        self.nsys = len(systems)
        if self.nsys == 0:
            raise ValueError("empty batch")
        sizes = [int(np.asarray(s[0]).reshape(-1, 3).shape[0]) for s in systems]
        self.atom_off_h = np.zeros(self.nsys + 1, np.int32)
        self.atom_off_h[1:] = np.cumsum(sizes)
        self.natoms = int(self.atom_off_h[-1])
        self.has_topo = [s[4] is not None for s in systems]
        self._build_atoms(systems)
        self._build_topology([s[4] if s[4] is not None else _empty_topo(n) for s, n in zip(systems, sizes)])
        self.params = _lib.reference_params()
        self.nl_ready = False
        self.keep_span = True  # AlmaNL.full_span: lets the move kernels skip rows that move whole
        self._alloc_nl(None)
        self.scratch = torch.zeros(max(1, self.L.alma_move_scratch_bytes(max(self.natoms, 1))),
                                   dtype=torch.uint8, device=_DEV)

    # ---- construction ---------------------------------------------------------
    def _build_atoms(self, systems):
        n = self.natoms
        xyz = np.zeros((n, 4))
        prm64 = np.zeros((n, 4))
        for s, (x, q, r, e, _) in enumerate(systems):
            a0, a1 = self.atom_off_h[s], self.atom_off_h[s + 1]
            xyz[a0:a1, :3] = np.asarray(x, np.float64).reshape(-1, 3)
            prm64[a0:a1, 0] = q
            prm64[a0:a1, 1] = r
            prm64[a0:a1, 2] = e
        if not np.all(np.isfinite(xyz)):
            raise ValueError("non-finite coordinates")
        self.xyz = _t(xyz, torch.float64)
        self.prm64 = _t(prm64, torch.float64)
        self.prm = self.prm64.to(torch.float32)
        self.born = torch.zeros(max(n, 1), dtype=torch.float64, device=_DEV)
        # per-atom SASA terms of the current coordinates (AlmaBatch.sasa):
        # filled by energy_terms, kept current by the move kernels; any other
        # change of the coordinates must call invalidate_sasa()
        self.sasa = torch.zeros(max(n, 1), dtype=torch.float64, device=_DEV)
        self.sasa_valid = False
        self.status = torch.zeros(1, dtype=torch.int32, device=_DEV)
        self.atom_off = _t(self.atom_off_h, torch.int32)
        self.atom_sys = torch.as_tensor(np.repeat(np.arange(self.nsys), np.diff(self.atom_off_h)), dtype=torch.int64,
                                        device=_DEV)

    def _build_topology(self, topos):
        off = self.atom_off_h
        ex_ptr, ex_cols = [np.zeros(1, np.int64)], []
        rb_ij, rb_kind, rb_scale, side_ptr, side_idx, side_lo, side_hi = [], [], [], [np.zeros(1, np.int64)], [], [], []
        dih, term_off, term_v2, term_n, term_g, ss, cp, csp = [], [np.zeros(1, np.int32)], [], [], [], [], [], []
        rb_off, dih_off, ss_off, cp_off, csp_off = ([0] for _ in range(5))
        ex_base = side_base = term_base = 0
        for s, T in enumerate(topos):
            a0 = int(off[s])
            n_s = int(off[s + 1] - off[s])
            if T.n != n_s:
                raise ValueError(f"system {s}: topology has {T.n} atoms, coordinates {n_s}")
            ex_ptr.append(T.excl_ptr[1:] + ex_base)
            ex_cols.append(T.excl_cols + a0)
            ex_base += int(T.excl_ptr[-1])
            rb_ij.append(np.stack([T.rb_i, T.rb_j], 1).reshape(-1) + a0)
            rb_kind.append(T.rb_kind)
            rb_scale.append(T.rb_scale)
            side_ptr.append(T.side_ptr[1:] + side_base)
            side_idx.append(T.side_idx + a0)
            side_base += int(T.side_ptr[-1])
            has = T.side_hi > T.side_lo
            side_lo.append(np.where(has, T.side_lo + a0, 0).astype(np.int32))
            side_hi.append(np.where(has, T.side_hi + a0, 0).astype(np.int32))
            dih.append(T.dih_abcd.reshape(-1) + a0)
            term_off.append(T.term_off[1:] + term_base)
            term_base += int(T.term_off[-1])
            term_v2.append(T.term_v2)
            term_n.append(T.term_n)
            term_g.append(T.term_gamma)
            ss.append(T.ss.reshape(-1) + a0)
            cp.append(T.crank.reshape(-1))
            csp.append(T.conc_sc.reshape(-1))
            rb_off.append(rb_off[-1] + T.nrb)
            dih_off.append(dih_off[-1] + T.ndih)
            ss_off.append(ss_off[-1] + T.ss.shape[0])
            cp_off.append(cp_off[-1] + T.crank.shape[0])
            csp_off.append(csp_off[-1] + T.conc_sc.shape[0])
        cat = lambda xs, dt: np.concatenate([np.asarray(x, dt).reshape(-1) for x in xs]) if xs else np.zeros(0, dt)
        self.t_excl_ptr = _t(cat(ex_ptr, np.int64), torch.int64)
        self.t_excl_cols = _t(cat(ex_cols, np.int32), torch.int32)
        self.t_rb_ij = _t(cat(rb_ij, np.int32), torch.int32)
        self.t_rb_kind = _t(cat(rb_kind, np.int32), torch.int32)
        self.t_rb_scale = _t(cat(rb_scale, np.float64), torch.float64)
        self.t_side_ptr = _t(cat(side_ptr, np.int64), torch.int64)
        self.t_side_idx = _t(cat(side_idx, np.int32), torch.int32)
        self.t_side_lo = _t(cat(side_lo, np.int32), torch.int32)
        self.t_side_hi = _t(cat(side_hi, np.int32), torch.int32)
        self.t_dih = _t(cat(dih, np.int32), torch.int32)
        self.t_term_off = _t(cat(term_off, np.int32), torch.int32)
        self.t_term_v2 = _t(cat(term_v2, np.float64), torch.float64)
        self.t_term_n = _t(cat(term_n, np.int32), torch.int32)
        self.t_term_g = _t(cat(term_g, np.float64), torch.float64)
        self.t_ss = _t(cat(ss, np.int32), torch.int32)
        self.t_cp = _t(cat(cp, np.int32), torch.int32)
        self.t_csp = _t(cat(csp, np.int32), torch.int32)
        self.rb_off_h = np.asarray(rb_off, np.int32)
        self.cp_off_h = np.asarray(cp_off, np.int32)
        self.csp_off_h = np.asarray(csp_off, np.int32)
        self.t_rb_off = _t(self.rb_off_h, torch.int32)
        self.t_dih_off = _t(np.asarray(dih_off, np.int32), torch.int32)
        self.t_ss_off = _t(np.asarray(ss_off, np.int32), torch.int32)
        self.t_cp_off = _t(self.cp_off_h, torch.int32)
        self.t_csp_off = _t(self.csp_off_h, torch.int32)
        self.side_count = cat([T.side_count for T in topos], np.int64)
        self.rb_kind_h = cat(rb_kind, np.int32)
        self.rb_scale_h = cat(rb_scale, np.float64)
        self.topos = topos
        tp = _lib.AlmaTopo()
        tp.excl_ptr, tp.excl_cols = _ptr(self.t_excl_ptr), _ptr(self.t_excl_cols)
        # per-atom exclusion windows: the list build tests one bit per pair
        self.t_excl_win = torch.zeros(4 * max(self.natoms, 1), dtype=torch.int32, device=_DEV)
        if self.t_excl_cols.numel() > 0:
            _lib.check(self.L.alma_excl_window(_ptr(self.t_excl_ptr), _ptr(self.t_excl_cols), self.natoms,
                                               _ptr(self.t_excl_win), self._sp()), "alma_excl_window")
        tp.excl_win = _ptr(self.t_excl_win)  # all zero without exclusions: no pair excluded
        tp.nrb, tp.rb_off, tp.rb_ij = int(rb_off[-1]), _ptr(self.t_rb_off), _ptr(self.t_rb_ij)
        tp.rb_kind, tp.rb_scale = _ptr(self.t_rb_kind), _ptr(self.t_rb_scale)
        tp.side_ptr, tp.side_idx = _ptr(self.t_side_ptr), _ptr(self.t_side_idx)
        tp.side_lo, tp.side_hi = _ptr(self.t_side_lo), _ptr(self.t_side_hi)
        tp.ndih, tp.dih_off, tp.dih_abcd = int(dih_off[-1]), _ptr(self.t_dih_off), _ptr(self.t_dih)
        tp.term_off, tp.term_v2, tp.term_n, tp.term_gamma = (_ptr(self.t_term_off), _ptr(self.t_term_v2),
                                                             _ptr(self.t_term_n), _ptr(self.t_term_g))
        tp.nss, tp.ss_off, tp.ss_ij = int(ss_off[-1]), _ptr(self.t_ss_off), _ptr(self.t_ss)
        tp.ncp, tp.cp_off, tp.cp = int(cp_off[-1]), _ptr(self.t_cp_off), _ptr(self.t_cp)
        tp.ncsp, tp.csp_off, tp.csp = int(csp_off[-1]), _ptr(self.t_csp_off), _ptr(self.t_csp)
        self.topo_s = tp
        self.use_topo = any(self.has_topo)

    @property
    def batch_s(self):
        """The AlmaBatch of this batch (built once: its buffers never move;
        the SASA cache pointer follows sasa_valid on every access)."""
        b = getattr(self, "_batch_s", None)
        if b is None:
            b = _lib.AlmaBatch()
            b.nsys, b.natoms = self.nsys, self.natoms
            b.atom_off, b.xyz, b.prm, b.prm64 = _ptr(self.atom_off), _ptr(self.xyz), _ptr(self.prm), _ptr(self.prm64)
            b.born, b.status = _ptr(self.born), _ptr(self.status)
            self._batch_s = b
        b.sasa = _ptr(self.sasa) if self.sasa_valid else None
        return b

    def invalidate_sasa(self):
        """Coordinates changed outside the energy / move kernels."""
        self.sasa_valid = False

    # ---- neighbor list ---------------------------------------------------------
    def _alloc_nl(self, need):
        self._nl_s = None
        sizes = np.diff(self.atom_off_h).astype(np.int64)
        if need is None:
            caps = [sizes * self.NL_FULL_PER_ATOM + 64, sizes * self.NL_HALF_PER_ATOM + 64,
                    sizes * self.NL_SHORT_PER_ATOM + 64, sizes * (self.NL_SHORT_PER_ATOM // 2) + 64]
        else:
            caps = [(need[:, k] * 5) // 4 + 4096 for k in range(4)]
        bases = []
        for c in caps:
            bb = np.zeros(self.nsys + 1, np.int64)
            bb[1:] = np.cumsum(c)
            bases.append(bb)
        fb, hb, sfb, shb = bases
        n = max(self.natoms, 1)
        self.full_base = _t(fb, torch.int64)
        self.half_base = _t(hb, torch.int64)
        self.full_ptr = torch.zeros(n, dtype=torch.int64, device=_DEV)
        self.full_len = torch.zeros(n, dtype=torch.int32, device=_DEV)
        self.half_ptr = torch.zeros(n, dtype=torch.int64, device=_DEV)
        self.half_len = torch.zeros(n, dtype=torch.int32, device=_DEV)
        self.full_cols = torch.zeros(int(fb[-1]) + 1, dtype=torch.int32, device=_DEV)
        self.half_cols = torch.zeros(int(hb[-1]) + 1, dtype=torch.int32, device=_DEV)
        self.sfull_base = _t(sfb, torch.int64)
        self.shalf_base = _t(shb, torch.int64)
        self.sfull_ptr = torch.zeros(n, dtype=torch.int64, device=_DEV)
        self.sfull_len = torch.zeros(n, dtype=torch.int32, device=_DEV)
        self.shalf_ptr = torch.zeros(n, dtype=torch.int64, device=_DEV)
        self.shalf_len = torch.zeros(n, dtype=torch.int32, device=_DEV)
        self.sfull_cols = torch.zeros(int(sfb[-1]) + 1, dtype=torch.int32, device=_DEV)
        self.shalf_cols = torch.zeros(int(shb[-1]) + 1, dtype=torch.int32, device=_DEV)
        self.ref_xyz = torch.zeros((n, 4), dtype=torch.float64, device=_DEV)
        self.full_span = torch.zeros((n, 2), dtype=torch.int32, device=_DEV)
        self.need = torch.zeros((self.nsys, 4), dtype=torch.int64, device=_DEV)
        self.max_cells = int(max(4096, 8 * self.natoms + 4096 * self.nsys))
        self.nl_ws = torch.zeros(self.L.alma_nl_workspace_bytes(self.nsys, self.natoms, self.max_cells),
                                 dtype=torch.uint8, device=_DEV)

    @property
    def nl_s(self):
        """The AlmaNL of the list buffers (rebuilt after _alloc_nl moves them)."""
        if getattr(self, "_nl_s", None) is not None:
            return self._nl_s
        nl = _lib.AlmaNL()
        nl.full_ptr, nl.full_len, nl.full_cols, nl.full_base = (_ptr(self.full_ptr), _ptr(self.full_len),
                                                                _ptr(self.full_cols), _ptr(self.full_base))
        nl.half_ptr, nl.half_len, nl.half_cols, nl.half_base = (_ptr(self.half_ptr), _ptr(self.half_len),
                                                                _ptr(self.half_cols), _ptr(self.half_base))
        nl.ref_xyz, nl.need = _ptr(self.ref_xyz), _ptr(self.need)
        nl.full_span = _ptr(self.full_span) if self.keep_span else None
        nl.sfull_ptr, nl.sfull_len, nl.sfull_cols, nl.sfull_base = (_ptr(self.sfull_ptr), _ptr(self.sfull_len),
                                                                    _ptr(self.sfull_cols), _ptr(self.sfull_base))
        nl.shalf_ptr, nl.shalf_len, nl.shalf_cols, nl.shalf_base = (_ptr(self.shalf_ptr), _ptr(self.shalf_len),
                                                                    _ptr(self.shalf_cols), _ptr(self.shalf_base))
        self._nl_s = nl
        return nl

    def set_row_spans(self, on):
        """Keep (default) or drop the per-row index spans (AlmaNL.full_span);
        the move kernels give the same bits either way, only slower without.
        The lists are rebuilt on the next use."""
        self.keep_span = bool(on)
        self._nl_s = None
        self.nl_ready = False

    def _sp(self):
        return C.c_void_p((self.stream or torch.cuda.current_stream()).cuda_stream)

    def build_nl(self, sys_mask=None, check=True):
        """Neighbor lists (all systems, or those with sys_mask[s] != 0)."""
        if self.natoms == 0:
            self.nl_ready = True
            return
        for attempt in range(3):
            b, t, nl = self.batch_s, self.topo_s, self.nl_s
            rc = self.L.alma_nl_build(C.byref(b), C.byref(t) if self.use_topo else None, C.byref(nl),
                                      C.byref(self.params), _ptr(sys_mask) if sys_mask is not None else None,
                                      _ptr(self.nl_ws),
                                      self.max_cells, self._sp())
            _lib.check(rc, "alma_nl_build")
            if not check:
                break
            st = int(self.status.item())
            if st & (_lib.ST_NL_OVERFLOW | _lib.ST_CELL_OVERFLOW):
                need = self.need.cpu().numpy()
                self.status.zero_()
                if st & _lib.ST_CELL_OVERFLOW:
                    self.max_cells *= 4
                    self.nl_ws = torch.zeros(self.L.alma_nl_workspace_bytes(self.nsys, self.natoms, self.max_cells),
                                             dtype=torch.uint8, device=_DEV)
                if st & _lib.ST_NL_OVERFLOW:
                    keep_cells = self.max_cells
                    self._alloc_nl(need)
                    self.max_cells = keep_cells
                    self.nl_ws = torch.zeros(self.L.alma_nl_workspace_bytes(self.nsys, self.natoms, self.max_cells),
                                             dtype=torch.uint8, device=_DEV)
                sys_mask = None
                continue
            break
        self.nl_ready = True

    def compact_nl(self):
        """Re-allocates the NL regions at 1.25x the measured need + margin."""
        need = self.need.cpu().numpy()
        keep = self.max_cells
        self._alloc_nl(need)
        self.max_cells = keep
        self.build_nl()

    # ---- energies -------------------------------------------------------------
    def born_radii(self, sys_mask=None):
        if not self.nl_ready:
            self.build_nl()
        b, nl = self.batch_s, self.nl_s
        _lib.check(self.L.alma_born_radii(C.byref(b), C.byref(nl), C.byref(self.params), self.prec,
                                          _ptr(sys_mask) if sys_mask is not None else None, self._sp()),
                   "alma_born_radii")

    def energy_terms(self, recompute_born=True, sys_mask=None, out=None):
        """[nsys, 5] float64 tensor {sasa, dihedral, disulfide, pairs, total}
        (rows of systems outside sys_mask are left as in `out`)."""
        if not self.nl_ready:
            self.build_nl()
        if recompute_born:
            self.born_radii(sys_mask)
        terms = out if out is not None else torch.zeros((self.nsys, 5), dtype=torch.float64, device=_DEV)
        if getattr(self, "_atom_e", None) is None:
            self._atom_e = torch.zeros((max(self.natoms, 1), 2), dtype=torch.float64, device=_DEV)
        b, t, nl = self.batch_s, self.topo_s, self.nl_s
        b.sasa = _ptr(self.sasa)  # refreshed for the evaluated systems
        _lib.check(self.L.alma_energy(C.byref(b), C.byref(t) if self.use_topo else None, C.byref(nl),
                                      C.byref(self.params), self.prec,
                                      _ptr(sys_mask) if sys_mask is not None else None, _ptr(self._atom_e),
                                      _ptr(terms), self._sp()), "alma_energy")
        if sys_mask is None:
            self.sasa_valid = True
        return terms

    def forces(self, sys_mask=None, out=None, recompute_born=False):
        """dE/dx [natoms, 4] float64 (x, y, z, 0) at the current coordinates
        (alma_forces).  The Born radii must be those of the current
        coordinates: energy_terms() leaves them so; recompute_born=True
        recomputes them first."""
        if not self.nl_ready:
            self.build_nl()
            recompute_born = True
        if recompute_born:
            self.born_radii(sys_mask)
        g = out if out is not None else torch.zeros((max(self.natoms, 1), 4), dtype=torch.float64, device=_DEV)
        if getattr(self, "_force_ws", None) is None:
            self._force_ws = torch.zeros(self.L.alma_forces_workspace_bytes(self.natoms), dtype=torch.uint8,
                                         device=_DEV)
        b, t, nl = self.batch_s, self.topo_s, self.nl_s
        _lib.check(self.L.alma_forces(C.byref(b), C.byref(t) if self.use_topo else None, C.byref(nl),
                                      C.byref(self.params), self.prec,
                                      _ptr(sys_mask) if sys_mask is not None else None, _ptr(self._force_ws),
                                      _ptr(g), self._sp()), "alma_forces")
        return g

    def evaluate(self, graph=False):
        """One full evaluation at the coordinates in self.xyz: fresh neighbor
        list, Born radii, energy terms and dE/dx.  Returns (terms [nsys, 5],
        grad [natoms, 4]); with graph=True both are buffers owned by the batch,
        rewritten by every call.

        graph=True replays one captured CUDA graph of the whole sequence (the
        first call captures it): write new coordinates into self.xyz between
        calls.  The list's overflow check runs after each replay (one status
        read); on overflow the lists are regrown, the graph recaptured and the
        evaluation repeated."""
        if not graph:
            self.nl_ready = False
            self.invalidate_sasa()
            self.build_nl()
            terms = self.energy_terms(recompute_born=True)
            return terms, self.forces()
        for _ in range(3):
            g = getattr(self, "_eval_graph", None)
            if g is None:
                g = self._capture_eval()
            g.replay()
            st = int(self.status.item())
            if not st & (_lib.ST_NL_OVERFLOW | _lib.ST_CELL_OVERFLOW):
                self.nl_ready = True
                self.sasa_valid = True
                return self._g_terms, self._g_grad
            # regrow the lists eagerly; the graph holds the old buffers
            self._eval_graph = None
            self.status.zero_()
            self.nl_ready = False
            self.build_nl()
        raise RuntimeError("evaluate: neighbor-list overflow persists")

    def _capture_eval(self):
        self._g_terms = torch.zeros((self.nsys, 5), dtype=torch.float64, device=_DEV)
        self._g_grad = torch.zeros((max(self.natoms, 1), 4), dtype=torch.float64, device=_DEV)

        def body():
            self.nl_ready = False
            self.build_nl(check=False)
            self.energy_terms(recompute_born=True, out=self._g_terms)
            self.forces(out=self._g_grad)

        keep, self.stream = self.stream, None  # captured on torch's current stream
        try:
            side = torch.cuda.Stream()
            side.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(side):  # warm-up: every workspace allocated outside the capture
                body()
            torch.cuda.current_stream().wait_stream(side)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                body()
        finally:
            self.stream = keep
        self._eval_graph = g
        return g

    # ---- one proposal per system ---------------------------------------------
    def move_dE(self, kind, a, delta, apply=False):
        """kind/a: int per system; delta: [nsys, 2] radians.  Returns
        (dE [nsys], dterms [nsys, 4]) device tensors."""
        if not self.nl_ready:
            self.build_nl()
        kind = np.asarray(kind, np.int64).reshape(self.nsys)
        a = np.asarray(a, np.int64).reshape(self.nsys)
        limits = {0: np.diff(self.rb_off_h), 1: np.diff(self.cp_off_h), 2: np.diff(self.csp_off_h)}
        for s in range(self.nsys):
            if kind[s] < 0:
                continue
            if kind[s] not in limits or not (0 <= a[s] < limits[int(kind[s])][s]):
                raise ValueError(f"system {s}: move (kind {kind[s]}, index {a[s]}) out of range")
        kind_t = _t(kind.astype(np.int32), torch.int32)
        a_t = _t(np.asarray(a, np.int32).reshape(self.nsys), torch.int32)
        d_t = _t(np.asarray(delta, np.float64).reshape(self.nsys, 2), torch.float64)
        dE = torch.zeros(self.nsys, dtype=torch.float64, device=_DEV)
        dterms = torch.zeros((self.nsys, 4), dtype=torch.float64, device=_DEV)
        b, t, nl = self.batch_s, self.topo_s, self.nl_s
        _lib.check(self.L.alma_move_dE(C.byref(b), C.byref(t), C.byref(nl), C.byref(self.params), self.prec,
                                       _ptr(self.scratch), _ptr(kind_t), _ptr(a_t), _ptr(d_t), int(bool(apply)),
                                       _ptr(dE), _ptr(dterms), self._sp()), "alma_move_dE")
        return dE, dterms

    def move_counters(self, phases=False):
        """[nsys, 4] uint64: pair terms, hct terms, SASA visits, moved atoms
        (phases=True: also [nsys, 4] SM cycles of the four ΔE phases)."""
        out = np.zeros((2, self.nsys, 4), np.uint64)
        _lib.check(self.L.alma_move_counters(_ptr(self.scratch), self.natoms, self.nsys, out.ctypes.data,
                                             self._sp()), "alma_move_counters")
        return (out[0], out[1]) if phases else out[0]

    def load_coords(self, xyz):
        """New coordinates [natoms, 3] for every system (same atoms, same
        topology): the list, radii and SASA cache are rebuilt on next use."""
        x = torch.as_tensor(np.ascontiguousarray(xyz, np.float64) if not isinstance(xyz, torch.Tensor) else xyz,
                            dtype=torch.float64).reshape(self.natoms, 3)
        self.xyz[:self.natoms, :3].copy_(x)
        self.nl_ready = False
        self.invalidate_sasa()
        self.status.zero_()

    # ---- host views -------------------------------------------------------------
    def coords(self, s=None):
        x = self.xyz[:, :3].cpu().numpy()
        if s is None:
            return x
        return x[self.atom_off_h[s]:self.atom_off_h[s + 1]]

    def nl_host(self, s=0, half=True, short=False):
        """(row_ptr, cols, excl_flags) of system s with local indices
        (short=True: the SASA-reach sub-rows)."""
        a0, a1 = int(self.atom_off_h[s]), int(self.atom_off_h[s + 1])
        if short:
            arrs = (self.shalf_ptr, self.shalf_len, self.shalf_cols) if half else \
                (self.sfull_ptr, self.sfull_len, self.sfull_cols)
        else:
            arrs = (self.half_ptr, self.half_len, self.half_cols) if half else \
                (self.full_ptr, self.full_len, self.full_cols)
        ptr = arrs[0][a0:a1].cpu().numpy()
        ln = arrs[1][a0:a1].cpu().numpy()
        cols_all = arrs[2].cpu().numpy().view(np.uint32)
        rp = np.zeros(a1 - a0 + 1, np.int64)
        rp[1:] = np.cumsum(ln)
        out = np.empty(int(rp[-1]), np.uint32)
        for i in range(a1 - a0):
            out[rp[i]:rp[i + 1]] = cols_all[ptr[i]:ptr[i] + ln[i]]
        idx = (out & 0x7FFFFFFF).astype(np.int64) - a0
        return rp, idx.astype(np.int32), (out >> 31).astype(np.uint8)

"""TEST INFRASTRUCTURE — the reference energy as an FP64 torch function of
the coordinates, for autograd gradient checks of the backward kernels.

The same arithmetic as alma_oracle.c (which cites the reference lines of
src/physics_engine.cpp), written with torch ops so that autograd gives dE/dx:
  * Born radii: HCT over both directions of every half-list pair
    (born_radii :2024-2039), a = 1/max(1/rho - sum/2, 2);
  * pairs: non-excluded half-list pairs with r^2 <= 144 (total_e
    :2205-2234), pair_e :2148-2164 (DH + GB + LJ + capped hard core);
  * SASA: the ordered recurrence over each half row (:2068-2083), run
    entry by entry over padded rows, vectorised over atoms;
  * dihedral records (:1912-1921) and disulfide springs (:1965-1974).
The neighbor list is an input (fixed while differentiating).  Only tests use
this module.
"""
from __future__ import annotations

import math

import numpy as np
import torch

COULOMB, EPS_WATER, EPS_PROT, KAPPA = 332.0636, 78.5, 1.0, 0.1257
GAMMA_SA, BETA_SA, PROBE_R = 0.00542, 0.92, 1.4
PAIR_CUT2 = 144.0
HARD_SCALE, HARD_CAP, HARD_FRAC = 1.0e4, 5.0e3, 0.6
GB_COEF = -0.5 * (1.0 / EPS_PROT - 1.0 / EPS_WATER) * COULOMB
K_SS, R0_SS = 600.0, 2.044


def _hct(r, r2, ri, rj):
    L = torch.maximum((r - rj).abs(), ri)
    U = r + rj
    v = 1.0 / L - 1.0 / U + (r2 - rj * rj + ri * ri) / (2.0 * r * ri * ri) * torch.log(L / U) * 0.5 / r
    return torch.where(ri >= U, torch.zeros_like(v), v)


def _dihedral(x, a, b, c, d):
    b1 = x[a] - x[b]
    b2 = x[c] - x[b]
    b3 = x[d] - x[c]
    n1 = torch.cross(b1, b2, dim=1)
    n2 = torch.cross(b2, b3, dim=1)
    m1 = torch.cross(n1, b2, dim=1)
    return torch.atan2((m1 * n2).sum(1), (n1 * n2).sum(1))


class TorchEnergy:
    """E(x) for one system with a fixed half neighbor list (row_ptr, cols)."""

    def __init__(self, q, radius, eps, row_ptr, cols, flat=None):
        self.n = len(q)
        row_ptr = np.asarray(row_ptr, np.int64)
        cols = np.asarray(cols, np.int64)
        I = np.repeat(np.arange(self.n), np.diff(row_ptr))
        self.I, self.J = torch.from_numpy(I), torch.from_numpy(cols)
        self.q = torch.as_tensor(np.asarray(q, np.float64))
        self.rad = torch.as_tensor(np.asarray(radius, np.float64))
        self.eps = torch.as_tensor(np.asarray(eps, np.float64))
        excl = np.zeros(len(cols), bool)
        self.flat = flat
        if flat is not None:
            ep, ec = np.asarray(flat.excl_ptr), np.asarray(flat.excl_cols)
            for k, (i, j) in enumerate(zip(I, cols)):
                a, b = (i, j) if i < j else (j, i)
                row = ec[ep[a]:ep[a + 1]]
                excl[k] = row.size > 0 and np.any(row == b)
        self.excl = torch.from_numpy(excl)
        # padded half rows for the ordered SASA recurrence
        lens = np.diff(row_ptr)
        self.maxlen = int(lens.max()) if self.n else 0
        pad = np.full((self.n, max(self.maxlen, 1)), -1, np.int64)
        for i in range(self.n):
            pad[i, :lens[i]] = cols[row_ptr[i]:row_ptr[i + 1]]
        self.pad = torch.from_numpy(pad)

    def born(self, x):
        d = x[self.I] - x[self.J]
        r2 = (d * d).sum(1)
        r = torch.sqrt(r2)
        ri, rj = self.rad[self.I], self.rad[self.J]
        s = torch.zeros(self.n, dtype=x.dtype)
        s = s.index_add(0, self.I, _hct(r, r2, ri, rj))
        s = s.index_add(0, self.J, _hct(r, r2, rj, ri))
        return 1.0 / torch.clamp(1.0 / self.rad - 0.5 * s, min=2.0)

    def pairs(self, x, a):
        d = x[self.I] - x[self.J]
        r2 = (d * d).sum(1)
        keep = (~self.excl) & (r2 <= PAIR_CUT2)
        I, J, r2 = self.I[keep], self.J[keep], r2[keep]
        r = torch.sqrt(r2)
        qp = self.q[I] * self.q[J]
        sig = self.rad[I] + self.rad[J]
        edh = (COULOMB * qp) / (EPS_WATER * r) * torch.exp(-KAPPA * r)
        aa = a[I] * a[J]
        egb = GB_COEF * qp / torch.sqrt(r2 + aa * torch.exp(-r2 / (4.0 * aa)))
        s6 = (sig / r) ** 6
        elj = 4.0 * torch.sqrt(self.eps[I] * self.eps[J]) * (s6 * s6 - s6)
        rc = sig * HARD_FRAC
        t12 = (rc / r) ** 12
        hard = torch.where(r < rc, torch.clamp(HARD_SCALE * (t12 - 1.0) ** 2, max=HARD_CAP), torch.zeros_like(r))
        return (edh + egb + elj + hard).sum()

    def sasa(self, x):
        if self.n == 0:
            return x.new_zeros(())
        R = self.rad + PROBE_R
        sa = 4.0 * math.pi * R * R
        cs = 2.0 * math.pi * R * R
        for k in range(self.maxlen):
            j = self.pad[:, k]
            ok = j >= 0
            jj = torch.where(ok, j, torch.zeros_like(j))
            d = x - x[jj]
            dist = torch.sqrt((d * d).sum(1) + (~ok).to(x.dtype))  # padded slots: dist 1, masked below
            dc = R + R[jj]
            hit = ok & (dist < dc)
            cap = cs * ((dc - dist) / (2.0 * R))
            sa = torch.where(hit, sa - torch.minimum(sa * 0.85, cap), sa)
        return BETA_SA + GAMMA_SA * torch.clamp(sa, min=0.0).sum()

    def bonded(self, x):
        E = x.new_zeros(())
        f = self.flat
        if f is None:
            return E, E
        abcd = np.asarray(f.dih_abcd, np.int64).reshape(-1, 4)
        if len(abcd):
            phi = _dihedral(x, *[torch.from_numpy(abcd[:, k]) for k in range(4)])
            off = np.asarray(f.term_off, np.int64)
            rec = torch.from_numpy(np.repeat(np.arange(len(abcd)), np.diff(off)))
            v2 = torch.tensor(np.asarray(f.term_v2, np.float64))  # copies: the topology's arrays are read-only
            nn = torch.tensor(np.asarray(f.term_n, np.float64))
            gm = torch.tensor(np.asarray(f.term_gamma, np.float64))
            E = (v2 * (1.0 + torch.cos(nn * phi[rec] - gm))).sum()
        ss = np.asarray(f.ss, np.int64).reshape(-1, 2)
        Ess = x.new_zeros(())
        if len(ss):
            d = x[torch.from_numpy(ss[:, 0])] - x[torch.from_numpy(ss[:, 1])]
            Ess = (K_SS * (torch.sqrt((d * d).sum(1)) - R0_SS) ** 2).sum()
        return E, Ess

    def terms(self, x):
        """(sasa, dihedral, ss, pairs, total) as torch scalars."""
        a = self.born(x)
        es = self.sasa(x)
        ed, ess = self.bonded(x)
        ep = self.pairs(x, a)
        return es, ed, ess, ep, es + ed + ess + ep

    def energy_and_grad(self, xyz):
        x = torch.tensor(np.asarray(xyz, np.float64), requires_grad=True)
        E = self.terms(x)[4]
        (g,) = torch.autograd.grad(E, x)
        return float(E.detach()), g.numpy()

"""Host logic of torsion space (no GPU): the j-side nesting tree
(alma_torsion_tree, host C++ in libalma_b200.so) and the composition rule
the all-bond move kernel relies on — turning every bond at once through the
tree equals the reference's one-bond-at-a-time rotations with axes taken
from the updated coordinates (rodrigues, physics_engine.cpp:1848-1862)."""
import numpy as np
import pytest

from protein_physics_b200 import synth
from protein_physics_b200.topology import BondTopology, flatten
from protein_physics_b200.torsion import torsion_tree


def _chain(n_res=12, seed=3):
    ch = synth.chain(n_res, seed)
    T = BondTopology()
    T.build(ch.resnames, ch.atomnames, ch.res_idx)
    return ch, T, flatten(T)


def _rot(p, o, u, d):
    v = p - o
    c, s = np.cos(d), np.sin(d)
    return o + v * c + np.cross(u, v) * s + np.outer(v @ u, u) * (1 - c)


def test_tree_matches_side_sets():
    ch, T, flat = _chain()
    parent, atom_rb = torsion_tree(flat)
    sides = [T.side_set(k) for k in range(flat.nrb)]
    for k in range(flat.nrb):
        p = parent[k]
        if p >= 0:
            assert sides[k] < sides[p]
        # atoms whose chain of innermost bonds passes through k = side k
    anc = []
    for m in range(flat.n):
        chain, k = set(), atom_rb[m]
        while k >= 0:
            chain.add(int(k))
            k = parent[k]
        anc.append(chain)
    for k in range(flat.nrb):
        assert {m for m in range(flat.n) if k in anc[m]} == sides[k]


def test_compose_equals_sequential_rotations():
    ch, T, flat = _chain(10, 5)
    parent, atom_rb = torsion_tree(flat)
    rng = np.random.default_rng(0)
    delta = rng.normal(0, 0.3, flat.nrb)
    x0 = ch.xyz.copy()
    # sequential, axes from the updated coordinates
    xs = x0.copy()
    for k in range(flat.nrb):
        side = np.array(sorted(T.side_set(k)))
        o = xs[flat.rb_i[k]]
        u = xs[flat.rb_j[k]] - o
        u /= np.linalg.norm(u)
        xs[side] = _rot(xs[side], o, u, delta[k])
    # tree composition, axes from the original coordinates
    A = []
    for k in range(flat.nrb):
        o = x0[flat.rb_i[k]]
        u = x0[flat.rb_j[k]] - o
        u /= np.linalg.norm(u)
        c, s = np.cos(delta[k]), np.sin(delta[k])
        K = np.array([[0, -u[2], u[1]], [u[2], 0, -u[0]], [-u[1], u[0], 0]])
        R = c * np.eye(3) + s * K + (1 - c) * np.outer(u, u)
        A.append((R, o - R @ o))
    Tk = list(A)
    P = parent.copy()
    while np.any(P >= 0):  # pointer jumping, as the kernel does
        Tn, Pn = list(Tk), P.copy()
        for k in range(flat.nrb):
            if P[k] >= 0:
                Rp, tp = Tk[P[k]]
                R, t = Tk[k]
                Tn[k] = (Rp @ R, Rp @ t + tp)
                Pn[k] = P[P[k]]
        Tk, P = Tn, Pn
    xt = x0.copy()
    for m in range(flat.n):
        if atom_rb[m] >= 0:
            R, t = Tk[atom_rb[m]]
            xt[m] = R @ x0[m] + t
    assert np.abs(xt - xs).max() < 1e-10


def test_ring_rejected():
    from conftest import Golden
    g = Golden("insulin")  # three disulfides close rings in the bond graph
    flat = flatten(g.topology())
    try:
        torsion_tree(flat)
    except ValueError as e:
        assert "nested" in str(e)
    else:  # a topology whose sides happen to stay nested is fine too
        pass

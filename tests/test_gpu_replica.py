"""GPU checks of replica exchange (alma_replica_exchange) and its driver.

The swap decisions of one round are recomputed on the host from the same
fresh energies, temperatures and Philox draw; the ladder stays a
permutation; runs are reproducible from the seed."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _philox(c, k):
    M0, M1, W0, W1, mask = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85, 0xFFFFFFFF
    c0, c1, c2, c3 = c
    k0, k1 = k
    for _ in range(10):
        p0, p1 = M0 * c0, M1 * c2
        c0, c1, c2, c3 = ((p1 >> 32) ^ c1 ^ k0) & mask, p1 & mask, ((p0 >> 32) ^ c3 ^ k1) & mask, p0 & mask
        k0, k1 = (k0 + W0) & mask, (k1 + W1) & mask
    return c0, c1, c2, c3


def _u01(a, b):
    return (((a >> 5) << 26) | (b >> 6)) / 9007199254740992.0


def _system(nres=12, seed=21):
    from protein_physics_b200 import synth
    from protein_physics_b200.topology import BondTopology, flatten
    ch = synth.chain(nres, seed)
    T = BondTopology()
    T.build(ch.resnames, ch.atomnames, ch.res_idx)
    return (ch.xyz, ch.charge, ch.radius, ch.epsilon, flatten(T))


def test_exchange_round_matches_host():
    from protein_physics_b200.replica import ReplicaExchange, geometric_ladder
    from protein_physics_b200.mc import K_BOLTZMANN
    RE = ReplicaExchange(_system(), geometric_ladder(300, 450, 6), seed=77, minimize_steps=40)
    for rnd in range(4):
        before_T = RE.mc.state()["temperature"].copy()
        before_perm = RE.sys_of_temp.cpu().numpy().copy()
        RE.interval(8)
        E = RE.terms.cpu().numpy()[:, 4]
        after_perm = RE.sys_of_temp.cpu().numpy()
        after_T = RE.mc.state()["temperature"]
        seed = RE.seed
        k = ((seed & 0xFFFFFFFF) ^ 0xA511E9B3, seed >> 32)
        perm = before_perm.copy()
        T = before_T.copy()
        for t in range(rnd & 1, RE.R - 1, 2):
            sa, sb = perm[t], perm[t + 1]
            la = (1 / T[sa] - 1 / T[sb]) * (E[sa] - E[sb])
            r = _philox((rnd, 0, t, 0x52455800), k)
            if la >= 0 or np.log(_u01(r[0], r[1])) < la:
                T[sa], T[sb] = T[sb], T[sa]
                perm[t], perm[t + 1] = sb, sa
        assert np.array_equal(after_perm, perm)
        assert np.array_equal(after_T, T)
        assert sorted(np.round(after_T / K_BOLTZMANN, 6)) == sorted(np.round(geometric_ladder(300, 450, 6), 6))
        # slot order = ascending temperature
        assert np.all(np.diff(after_T[after_perm]) > 0)
    st = RE.stats()
    assert 0.0 <= st["exchange_acceptance"] <= 1.0
    assert RE.attempts.cpu().numpy()[:RE.R - 1].sum() == 2 * 3 + 2 * 2  # rounds 0,2: 3 pairs; 1,3: 2 pairs


def test_replica_reproducible():
    from protein_physics_b200.replica import ReplicaExchange, geometric_ladder
    out = []
    for _ in range(2):
        RE = ReplicaExchange(_system(10, 5), geometric_ladder(300, 450, 4), seed=3, minimize_steps=20)
        RE.run(2, sweeps_per_exchange=8)
        out.append((RE.batch.coords(0), RE.sys_of_temp.cpu().numpy()))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])

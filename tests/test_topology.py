"""BondTopology (host input of the device path) against the reference's own
BondTopology output stored in the golden vectors: exclusion sets, rotatable
bonds, j-sides (DFS order), lever scales, dihedral records, crankshaft and
concerted-sidechain pairs must be identical."""
import hashlib

import numpy as np
import pytest


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_topology_matches_reference(golden):
    _check_topology(golden)


@pytest.mark.parametrize("name", __import__("conftest").WORKLOAD_SYSTEMS)
def test_topology_matches_reference_on_bench_chains(name):
    """The same identity on the benchmark chains (up to 65k atoms); for
    chains whose j-side lists run to ~10^8 entries the sides are compared
    by count and by the compact form instead of the DFS lists."""
    from conftest import Golden
    g = Golden(name)
    _check_topology(g, full_sides=g.n < 20000)


def _check_topology(golden, full_sides=True):
    T = golden.topology()
    excl_cnt = np.array([len(e) for e in T.excl], np.int64)
    assert np.array_equal(excl_cnt, golden["topo_excl_cnt"])
    assert sha(np.array([j for e in T.excl for j in e], np.int32)) == str(golden["topo_excl_sha"])
    rb = np.array([(r.i, r.j, int(r.kind)) for r in T.rot_bonds], np.int32).reshape(-1, 3)
    assert np.array_equal(rb, golden["topo_rb"])
    if full_sides:
        sides = T.rot_bond_sides
        assert np.array_equal(np.array([len(s) for s in sides], np.int64), golden["topo_side_cnt"])
        assert sha(np.array([j for s in sides for j in s], np.int32)) == str(golden["topo_side_sha"])
    else:
        from protein_physics_b200.topology import flatten
        assert np.array_equal(np.asarray(flatten(T).side_count, np.int64), golden["topo_side_cnt"])
    np.testing.assert_array_equal(np.array(T.rot_bond_scale), golden["topo_rot_bond_scale"])
    dih = np.stack([T.dih_a, T.dih_b, T.dih_c, T.dih_d], 1).astype(np.int32) if T.num_dihedrals else np.zeros((0, 4))
    assert np.array_equal(dih, golden["topo_dih"])
    assert np.array_equal(np.array(T.dih_term_offsets), golden["topo_dih_term_offsets"])
    np.testing.assert_array_equal(np.array(T.dih_term_v2), golden["topo_dih_term_v2"])
    np.testing.assert_array_equal(np.array(T.dih_term_n), golden["topo_dih_term_n"])
    np.testing.assert_array_equal(np.array(T.dih_term_gamma), golden["topo_dih_term_gamma"])
    assert np.array_equal(np.array(sorted(T.concerted_pairs), np.int32).reshape(-1, 2), golden["topo_crank"])
    assert np.array_equal(np.array(T.concerted_sidechain_pairs, np.int32).reshape(-1, 2), golden["topo_conc_sc"])
    assert np.array_equal(np.array(T.disulfide_pairs, np.int32).reshape(-1, 2), golden["topo_ss"])


def test_compact_sides_cover_dfs_sides(golden):
    from protein_physics_b200.topology import flatten
    T = golden.topology()
    F = flatten(T)
    for k, side in enumerate(T.rot_bond_sides):
        comp = set(range(int(F.side_lo[k]), int(F.side_hi[k])))
        comp.update(F.side_idx[F.side_ptr[k]:F.side_ptr[k + 1]].tolist())
        assert comp == set(side)
        assert F.side_count[k] == len(side)


def test_queries_and_errors():
    from protein_physics_b200.topology import BondKind, BondTopology
    T = BondTopology()
    T.build(["ALA"] * 5 + ["GLY"] * 5, ["N", "H", "CA", "HA", "C"] + ["N", "H", "CA", "HA2", "C"],
            [0] * 5 + [1] * 5)
    assert T.bonded(0, 2) and not T.bonded(0, 9)
    assert T.is_excluded(0, 4) and not T.is_excluded(0, 99)
    assert T.j_side(-1, 2) == []
    assert all(isinstance(rb.kind, BondKind) for rb in T.rot_bonds)
    T.add_disulfide(0, 0)            # ignored: self pair
    T.add_disulfide(0, 1000)         # ignored: out of range
    assert T.disulfide_pairs == []
    with pytest.raises(ValueError):
        T.build(["ALA"], ["N", "CA"], [0])
    E = BondTopology()
    E.build([], [], [])
    assert E.num_atoms == 0 and E.num_rot_bonds == 0


def test_reference_topology_flattens_identically(golden):
    """flatten() accepts the reference's BondTopology: same CSR arrays."""
    ref = pytest.importorskip("protein_physics")
    from protein_physics_b200.topology import flatten
    R = ref.BondTopology()
    R.build(golden.resnames, golden.atomnames, golden.res_idx)
    for i, j in golden["ss_in"]:
        R.add_disulfide(int(i), int(j))
    R.identify_concerted_sidechain_pairs([ref.Particle(*map(float, x), 0.0) for x in golden["xyz"]])
    A, B = flatten(golden.topology()), flatten(R)
    for k in ("excl_ptr", "excl_cols", "rb_i", "rb_j", "rb_kind", "rb_scale", "side_ptr", "side_idx", "side_lo",
              "side_hi", "dih_abcd", "term_off", "term_v2", "term_n", "term_gamma", "ss", "conc_sc"):
        assert np.array_equal(getattr(A, k), getattr(B, k)), k
    assert sorted(map(tuple, A.crank)) == sorted(map(tuple, B.crank))


def test_flatten_cache_follows_mutations(golden):
    """flatten() reuses its arrays until build / add_disulfide /
    identify_concerted_sidechain_pairs change the topology."""
    from protein_physics_b200.topology import BondTopology, flatten
    T = BondTopology()
    T.build(golden.resnames, golden.atomnames, golden.res_idx)
    a = flatten(T)
    assert flatten(T) is a
    assert not a.excl_cols.flags.writeable
    T.add_disulfide(0, golden.n - 1)
    b = flatten(T)
    assert b is not a and len(b.ss) == len(a.ss) + 1
    T.identify_concerted_sidechain_pairs(golden["xyz"])
    c = flatten(T)
    assert c is not b and len(c.conc_sc) == len(T.concerted_sidechain_pairs)
    T.build(golden.resnames[:10], golden.atomnames[:10], golden.res_idx[:10])
    assert flatten(T).n == 10


def test_exclusion_windows_restate_is_excluded(golden):
    """The exclusion windows the list build reads (restated from the flat
    CSR rows) give BondTopology.is_excluded for every pair within 63
    indices, and flag exactly the atoms with a partner farther away."""
    from conftest import excl_window_np
    from protein_physics_b200.topology import flatten
    T = golden.topology()
    F = flatten(T)
    w = excl_window_np(F.excl_ptr, F.excl_cols, F.n)
    bits = np.unpackbits(w.view(np.uint8).reshape(F.n, 16), axis=1, bitorder="little")
    for i in range(F.n):
        for d in range(-63, 64):
            j = i + d
            if d == 0 or not 0 <= j < F.n:
                assert d == 0 or bits[i, d + 64] == 0
                continue
            assert bits[i, d + 64] == int(T.is_excluded(i, j)), (i, j)
        far = any(T.is_excluded(i, j) for j in range(F.n) if abs(j - i) >= 64)
        assert bits[i, 64] == int(far), i
        assert bits[i, 0] == 0

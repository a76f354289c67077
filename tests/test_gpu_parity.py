"""GPU parity: the sm_100a kernels (through the C ABI) against the oracle
and the reference's golden vectors.

Bars (the reference's own path is FP64):
  * neighbor lists, exclusion flags: bit-exact, row order included;
  * FP64 mode: energies 1e-10 relative, Born radii 1e-12 relative,
    move ΔE 1e-7 kcal/mol absolute (summation order differs only);
  * mixed mode (FP32 pair terms, FP64 accumulation): total energy 1e-6
    relative; move ΔE 1e-4 kcal/mol absolute on the PDB systems.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _batch(golden, precision="mixed", topo=True):
    from protein_physics_b200.device import DeviceBatch
    from protein_physics_b200.topology import flatten
    flat = flatten(golden.topology()) if topo else None
    return DeviceBatch([(golden["xyz"], golden["q"], golden["r"], golden["eps"], flat)], precision=precision)


def test_nl_bit_exact(golden, oracle):
    b = _batch(golden)
    b.build_nl()
    rp, cols, flags = b.nl_host(0, half=True)
    ptr, ocols = oracle.nl_build(golden["xyz"])
    assert np.array_equal(rp, ptr)
    assert np.array_equal(cols, ocols)  # row order included (SASA depends on it)
    # exclusion flags = the topology's exclusion test
    from oracle import TopoArrays
    from protein_physics_b200.topology import flatten
    T = golden.topology()
    ex = np.array([T.is_excluded(i, int(j)) for i in range(golden.n) for j in ocols[ptr[i]:ptr[i + 1]]], np.uint8)
    assert np.array_equal(flags, ex)
    # full rows: both directions, same sets
    frp, fcols, _ = b.nl_host(0, half=False)
    for i in range(0, golden.n, max(1, golden.n // 97)):
        half_i = set(ocols[ptr[i]:ptr[i + 1]].tolist())
        lower = {k for k in range(i) if i in set(ocols[ptr[k]:ptr[k + 1]].tolist())}
        assert set(fcols[frp[i]:frp[i + 1]].tolist()) == half_i | lower


def test_nl_short_rows(golden):
    """Short rows: the full/half rows filtered, in order, to the pairs within
    R*_i + R*_j + 2 probe + skin (+1e-6) at build time."""
    b = _batch(golden)
    b.build_nl()
    p = b.params
    pad = 2.0 * p.probe_r + 2.0 * np.sqrt(p.half_skin2) + 1e-6
    x, r = golden["xyz"], golden["r"]
    for half in (True, False):
        rp, cols, flags = b.nl_host(0, half=half)
        srp, scols, sflags = b.nl_host(0, half=half, short=True)
        for i in range(golden.n):
            row = cols[rp[i]:rp[i + 1]]
            fl = flags[rp[i]:rp[i + 1]]
            reach = r[i] + pad + r[row]
            keep = np.sum((x[row] - x[i]) ** 2, axis=1) < reach * reach
            assert np.array_equal(scols[srp[i]:srp[i + 1]], row[keep]), i
            assert np.array_equal(sflags[srp[i]:srp[i + 1]], fl[keep]), i
    need = b.need.cpu().numpy()[0]
    assert need[2] == len(b.nl_host(0, half=False, short=True)[1])
    assert need[3] == len(b.nl_host(0, half=True, short=True)[1])


@pytest.mark.parametrize("precision,rtol", [("fp64", 1e-12), ("mixed", 2e-6)])
def test_born_radii(golden, oracle, precision, rtol):
    b = _batch(golden, precision)
    b.build_nl()
    b.born_radii()
    a = b.born[:golden.n].cpu().numpy()
    np.testing.assert_allclose(a, golden["born"], rtol=rtol, atol=0)


@pytest.mark.parametrize("precision,rtol", [("fp64", 1e-10), ("mixed", 1e-6)])
def test_energy_terms(golden, precision, rtol):
    b = _batch(golden, precision)
    terms = b.energy_terms()[0].cpu().numpy()
    ref = golden["energy_topo"]
    assert abs(terms[4] - ref[4]) <= rtol * abs(ref[4])
    np.testing.assert_allclose(terms[:3], ref[:3], rtol=1e-10, atol=1e-9)  # SASA/dihedral/SS are FP64 always
    b2 = _batch(golden, precision, topo=False)
    t2 = b2.energy_terms()[0].cpu().numpy()
    assert abs(t2[4] - golden["energy_notopo"][4]) <= rtol * abs(golden["energy_notopo"][4])


def test_bridge_case():
    import json
    import os
    from conftest import GOLDEN
    from protein_physics_b200 import Particle, PhysicsEngine
    g = json.load(open(os.path.join(GOLDEN, "bridge.json")))
    P = [Particle(*x, q) for x, q in zip(g["xyz"], g["q"])]
    assert PhysicsEngine(precision="fp64").calculate_potential(P) == pytest.approx(g["energy"], rel=1e-12)
    assert PhysicsEngine().calculate_potential(P) == pytest.approx(g["energy"], rel=1e-6)


def _move_args(golden, T, kind, code):
    if kind == 0:
        return 0, int(code)
    phi_k, psi_k = divmod(int(code), 100000)
    return 1, sorted(T.concerted_pairs).index((phi_k, psi_k))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_move_dE_vs_reference(golden, precision):
    T = golden.topology()
    b = _batch(golden, precision)
    b.build_nl()
    b.born_radii()
    errs = []
    for kind, code, delta, dE_ref, *terms_ref in golden["moves"]:
        k, a = _move_args(golden, T, int(kind), code)
        dE, dterms = b.move_dE([k], [a], [[delta, 0.0]])
        dE = float(dE[0].item())
        dterms = dterms[0].cpu().numpy()
        if precision == "fp64":
            assert dE == pytest.approx(dE_ref, abs=1e-7 + 1e-12 * abs(dE_ref))
            np.testing.assert_allclose(dterms, terms_ref, atol=1e-7, rtol=1e-12)
        else:
            # 1e-4 kcal/mol; plus the FP64 rounding floor of the reference's
            # own sums when a move carries a clash of ~1e11 kcal/mol
            scale = np.sum(np.abs(terms_ref))
            tol = 1e-4 + 1e-14 * scale
            assert abs(dE - dE_ref) <= tol, (kind, code, dE, dE_ref)
            np.testing.assert_allclose(dterms[1:], terms_ref[1:], atol=1e-8, rtol=1e-11)  # SASA/dih/SS FP64
        errs.append(abs(dE - dE_ref))
    # the state must be unchanged after non-applied proposals
    assert np.array_equal(b.coords(0), golden["xyz"])


def test_move_apply_matches_oracle(golden, oracle):
    from oracle import TopoArrays
    from protein_physics_b200.topology import flatten
    T = golden.topology()
    flat = flatten(T)
    b = _batch(golden, "fp64")
    b.build_nl()
    b.born_radii()
    x, q, r, e = golden["xyz"], golden["q"], golden["r"], golden["eps"]
    nl = oracle.nl_build(x)
    a = oracle.born_radii(x, r, nl)
    k = int(np.argmax([len(s) for s in T.rot_bond_sides]) // 2)
    side = T.rot_bond_sides[k]
    group = np.zeros(golden.n, np.int8)
    group[side] = 1
    dE_o, _, new_xyz, new_a = oracle.move_dE(x, q, r, e, nl, a, TopoArrays(flat), [(T.rot_bonds[k].i, T.rot_bonds[k].j,
                                                                                    0.2, side)], group)
    dE, _ = b.move_dE([0], [k], [[0.2, 0.0]], apply=True)
    assert float(dE[0]) == pytest.approx(dE_o, abs=1e-7)
    np.testing.assert_allclose(b.coords(0), new_xyz, rtol=0, atol=1e-12)
    np.testing.assert_allclose(b.born[:golden.n].cpu().numpy(), new_a, rtol=1e-12, atol=0)


def test_batched_equals_single():
    from conftest import Golden
    from protein_physics_b200.device import DeviceBatch
    from protein_physics_b200.topology import flatten
    gs = [Golden(n) for n in ("xq8", "insulin", "synth64")]
    systems = [(g["xyz"], g["q"], g["r"], g["eps"], flatten(g.topology())) for g in gs]
    B = DeviceBatch(systems)
    tb = B.energy_terms().cpu().numpy()
    for s, sysd in enumerate(systems):
        S = DeviceBatch([sysd])
        ts = S.energy_terms().cpu().numpy()[0]
        assert np.array_equal(ts, tb[s])  # bit-identical: same per-atom work, same reduction order
        rp_b, c_b, f_b = B.nl_host(s)
        rp_s, c_s, f_s = S.nl_host(0)
        assert np.array_equal(rp_b, rp_s) and np.array_equal(c_b, c_s) and np.array_equal(f_b, f_s)


def test_deterministic():
    from conftest import Golden
    g = Golden("xq8")
    r1 = _batch(g).energy_terms().cpu().numpy()
    r2 = _batch(g).energy_terms().cpu().numpy()
    assert np.array_equal(r1, r2)


def test_dropin_api(golden):
    from protein_physics_b200 import Particle, PhysicsEngine
    P = [Particle(*x, q, r, e) for x, q, r, e in zip(golden["xyz"], golden["q"], golden["r"], golden["eps"])]
    eng = PhysicsEngine()
    E = eng.calculate_potential(P, golden.topology())
    assert E == pytest.approx(golden["energy_topo"][4], rel=1e-6)
    assert eng.calculate_potential(P) == pytest.approx(golden["energy_notopo"][4], rel=1e-6)
    assert eng.calculate_potential([]) == 0.0
    assert "B200" in PhysicsEngine.device_name() or len(PhysicsEngine.device_name()) > 0


def test_engine_reuses_batch_across_calls(golden):
    """Repeated calls on one system reuse the device batch (coordinates
    reloaded): energies equal a fresh engine's, also after the coordinates
    change, and a different parameter set gets its own batch."""
    from protein_physics_b200 import Particle, PhysicsEngine
    T = golden.topology()
    eng = PhysicsEngine()
    P = [Particle(*x, q, r, e) for x, q, r, e in zip(golden["xyz"], golden["q"], golden["r"], golden["eps"])]
    E1 = eng.calculate_potential(P, T)
    x2 = np.asarray(golden["xyz"]) + np.random.default_rng(2).normal(0, 0.05, (golden.n, 3))
    P2 = [Particle(*x, q, r, e) for x, q, r, e in zip(x2, golden["q"], golden["r"], golden["eps"])]
    E2 = eng.calculate_potential(P2, T)
    assert len(eng._batches) == 1
    assert E2 == PhysicsEngine().calculate_potential(P2, T)
    assert eng.calculate_potential(P, T) == E1
    P3 = [Particle(*x, 0.5 * q, r, e) for x, q, r, e in zip(golden["xyz"], golden["q"], golden["r"], golden["eps"])]
    assert eng.calculate_potential(P3, T) == PhysicsEngine().calculate_potential(P3, T)
    assert len(eng._batches) == 2


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_row_spans_and_edge_skip(golden, precision):
    """AlmaNL.full_span holds each full row's smallest and largest atom
    index, and a move gives the same ΔE terms whether or not the kernels may
    skip the rows that move whole (no cross pair, no SASA mark in them):
    every torsion, crankshaft and concerted-pair move of the system."""
    T = golden.topology()
    on = _batch(golden, precision)
    off = _batch(golden, precision)
    off.set_row_spans(False)
    for b in (on, off):
        b.build_nl()
        b.born_radii()
    rp, cols, _ = on.nl_host(0, half=False)
    span = on.full_span[:golden.n].cpu().numpy()
    for i in range(golden.n):
        row = cols[rp[i]:rp[i + 1]]
        assert tuple(span[i]) == ((int(row.min()), int(row.max())) if row.size else (2 ** 31 - 1, -1))
    moves = [(0, k) for k in range(len(T.rot_bonds))]
    moves += [(1, k) for k in range(len(T.concerted_pairs))]
    moves += [(2, k) for k in range(len(T.concerted_sidechain_pairs))]
    rng = np.random.default_rng(5)
    tol = 1e-11 if precision == "fp64" else 1e-9
    inner = 0
    for kind, a in moves:
        d = rng.uniform(-0.3, 0.3, 2)
        e1, t1 = on.move_dE([kind], [a], [d])
        e0, t0 = off.move_dE([kind], [a], [d])
        t1, t0 = t1[0].cpu().numpy(), t0[0].cpu().numpy()
        np.testing.assert_allclose(t1, t0, rtol=tol, atol=1e-9, err_msg=str((kind, a)))
        assert float(e1[0]) == pytest.approx(float(e0[0]), rel=tol, abs=1e-9)
    # the skip engages: some torsion side holds atoms whose rows stay inside it
    from protein_physics_b200.topology import flatten
    F = flatten(T)
    for k in range(F.nrb):
        lo, hi = int(F.side_lo[k]), int(F.side_hi[k])
        inner += int(np.sum((span[lo:hi, 0] >= lo) & (span[lo:hi, 1] < hi)))
    assert inner > 0
    # commits of the largest sides (their inner members' Born radii come from
    # the commit pass): same coordinates, same radii
    big = np.argsort(-F.side_count)[:4]
    for kind, a in [(0, int(k)) for k in big] + [(1, 0)] * (len(T.concerted_pairs) > 0):
        for b in (on, off):
            b.move_dE([kind], [a], [[0.2, 0.0]], apply=True)
        assert np.array_equal(on.coords(0), off.coords(0))
        np.testing.assert_allclose(on.born[:golden.n].cpu().numpy(), off.born[:golden.n].cpu().numpy(),
                                   rtol=1e-12 if precision == "fp64" else 1e-6)


def test_nl_overflow_regrows_and_rebuilds(oracle):
    """Regions far too small for the rows: the build raises the overflow,
    the batch regrows its regions from need[] and builds again; the rows are
    then bit-exact, and a masked rebuild of one system after its atoms move
    leaves the other system's rows as they were."""
    from conftest import Golden
    from protein_physics_b200.device import DeviceBatch
    from protein_physics_b200.topology import flatten

    class Tight(DeviceBatch):
        NL_FULL_PER_ATOM = 1
        NL_HALF_PER_ATOM = 1
        NL_SHORT_PER_ATOM = 2

    gs = [Golden("insulin"), Golden("xq8")]
    systems = [(g["xyz"], g["q"], g["r"], g["eps"], flatten(g.topology())) for g in gs]
    b = Tight(systems)
    assert int(b.full_base[-1]) < 2 * b.natoms + 1000  # the initial regions cannot hold the rows
    b.build_nl()
    for s, g in enumerate(gs):
        rp, cols, _ = b.nl_host(s, half=True)
        ptr, ocols = oracle.nl_build(g["xyz"])
        assert np.array_equal(rp, ptr) and np.array_equal(cols, ocols), s
    before = b.nl_host(1, half=False)
    x = b.xyz.clone()
    a0, a1 = int(b.atom_off_h[0]), int(b.atom_off_h[1])
    x[a0:a1, :3] += 0.3
    b.xyz.copy_(x)
    mask = torch.tensor([1, 0], dtype=torch.uint8, device="cuda")
    b.build_nl(sys_mask=mask)
    after = b.nl_host(1, half=False)
    assert all(np.array_equal(u, v) for u, v in zip(before, after))
    rp, cols, _ = b.nl_host(0, half=True)
    ptr, ocols = oracle.nl_build(b.coords(0))
    assert np.array_equal(rp, ptr) and np.array_equal(cols, ocols)


def test_exclusion_window(golden):
    """alma_excl_window against its restatement from the CSR rows, and the
    list rows with the windows equal to those of the per-pair CSR search,
    flags and order included (insulin's disulfides take the far path)."""
    from conftest import excl_window_np
    from protein_physics_b200.device import _ptr
    b = _batch(golden)
    ref = excl_window_np(b.t_excl_ptr.cpu().numpy(), b.t_excl_cols.cpu().numpy(), b.natoms)
    got = b.t_excl_win.cpu().numpy().view(np.uint32).reshape(-1, 4)[:b.natoms]
    assert np.array_equal(got, ref)
    if len(golden.d["ss_in"]):
        assert (ref[:, 2] & 1).any()
    kinds = [(h, s) for h in (True, False) for s in (False, True)]
    b.build_nl()
    with_win = [b.nl_host(0, half=h, short=s) for h, s in kinds]
    b.topo_s.excl_win = None
    try:
        b.nl_ready = False
        b.build_nl()
        csr = [b.nl_host(0, half=h, short=s) for h, s in kinds]
    finally:
        b.topo_s.excl_win = _ptr(b.t_excl_win)
    for a, c in zip(with_win, csr):
        for x, y in zip(a, c):
            assert np.array_equal(x, y)

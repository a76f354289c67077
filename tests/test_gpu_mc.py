"""Device Monte Carlo vs the oracle's MC driver, draw for draw.

Both sides take the same Philox draws (seed, system, step), so with FP64
pair arithmetic on the device the two trajectories must coincide: the same
accepted / rebuilt counts, the same adaptive cur_max and final coordinates
to 1e-9 Å.  The mixed-precision engine may flip a Metropolis decision only
when u is within its ~1e-5 kcal/mol ΔE error of the threshold; over the
short runs here it does not.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _setup(name):
    from conftest import Golden
    from protein_physics_b200.topology import flatten
    g = Golden(name)
    return g, flatten(g.topology())


def _gpu_run(g, F, nsys, seed, steps, precision="fp64", policy=0, fixed_delta=0.0, moveset=None, T=0.6,
             cluster_size=None, spec_teams=1, device_rebuild=True, runner=False, tail_shape=True):
    from protein_physics_b200.device import DeviceBatch
    from protein_physics_b200.mc import MCRunner
    b = DeviceBatch([(g["xyz"], g["q"], g["r"], g["eps"], F)] * nsys, precision=precision)
    R = MCRunner(b, T, seed, policy=policy, fixed_delta=fixed_delta,
                 moveset=[moveset] * nsys if moveset is not None else None, cluster_size=cluster_size,
                 spec_teams=spec_teams, device_rebuild=device_rebuild, tail_shape=tail_shape)
    st = R.run_to(steps)
    return (b, st, R) if runner else (b, st)


def _oracle_run(g, F, seed, steps, sys_index=0, policy=0, fixed_delta=0.0, moveset=None, T=0.6):
    from oracle import Oracle, oracle_mc
    return oracle_mc(Oracle(), F, g["xyz"], g["q"], g["r"], g["eps"], seed, steps, temperature=T, policy=policy,
                     fixed_delta=fixed_delta, moveset=moveset, sys_index=sys_index)


@pytest.mark.parametrize("name,policy,steps", [("insulin", 0, 300), ("xq8", 0, 150), ("xq8", 1, 150)])
def test_fp64_trajectory_matches_oracle(name, policy, steps):
    g, F = _setup(name)
    b, st = _gpu_run(g, F, 1, 11, steps, policy=policy)
    x_o, st_o, _ = _oracle_run(g, F, 11, steps, policy=policy)
    assert st["n_accepted"][0] == st_o["n_accepted"]
    assert st["n_proposed"][0] == st_o["n_proposed"]
    assert st["n_rebuild"][0] == st_o["n_rebuild"]
    assert st["cur_max"][0] == pytest.approx(st_o["cur_max"], rel=1e-15)
    np.testing.assert_allclose(b.coords(0), x_o, rtol=0, atol=1e-9)
    assert st["energy"][0] == pytest.approx(st_o["energy"], rel=1e-9, abs=1e-6)


def test_rebuild_path_matches_oracle():
    """Large fixed angles force drift > skin/2 and neighbor-list rebuilds."""
    g, F = _setup("insulin")
    b, st = _gpu_run(g, F, 1, 5, 120, fixed_delta=0.6, T=50.0)
    x_o, st_o, _ = _oracle_run(g, F, 5, 120, fixed_delta=0.6, T=50.0)
    assert st_o["n_rebuild"] > 0
    assert st["n_rebuild"][0] == st_o["n_rebuild"]
    assert st["n_accepted"][0] == st_o["n_accepted"]
    np.testing.assert_allclose(b.coords(0), x_o, rtol=0, atol=1e-8)


def test_batched_chains_are_independent_streams():
    g, F = _setup("insulin")
    b, st = _gpu_run(g, F, 3, 21, 80)
    for s in range(3):
        x_o, st_o, _ = _oracle_run(g, F, 21, 80, sys_index=s)
        assert st["n_accepted"][s] == st_o["n_accepted"]
        np.testing.assert_allclose(b.coords(s), x_o, rtol=0, atol=1e-9)


def test_moveset_restriction():
    g, F = _setup("xq8")
    small = [k for k in range(F.nrb) if F.side_count[k] <= 0.25 * F.n]
    b, st = _gpu_run(g, F, 1, 3, 100, policy=2, moveset=small)
    x_o, st_o, _ = _oracle_run(g, F, 3, 100, policy=2, moveset=small)
    assert st["n_accepted"][0] == st_o["n_accepted"]
    np.testing.assert_allclose(b.coords(0), x_o, rtol=0, atol=1e-9)


def test_mixed_precision_chain_is_sane():
    g, F = _setup("insulin")
    b, st = _gpu_run(g, F, 2, 9, 200, precision="mixed")
    _, st_o, _ = _oracle_run(g, F, 9, 200)
    assert abs(int(st["n_accepted"][0]) - st_o["n_accepted"]) <= 2
    assert np.all(np.isfinite(st["energy"]))


def test_dropin_mc_entry_points():
    from protein_physics_b200 import Particle, PhysicsEngine
    g, F = _setup("insulin")
    T = g.topology()
    P = [Particle(*x, q, r, e) for x, q, r, e in zip(g["xyz"], g["q"], g["r"], g["eps"])]
    eng = PhysicsEngine(seed=1)
    ens = eng.generate_ensemble(P, T, 3, 50)
    assert len(ens) == 3 and all(len(m) == len(P) for m in ens)
    snaps, energies = eng.run_landscape_trajectory(P, T, 2, 20)
    assert len(snaps) == 2 and len(energies) == 2 and all(np.isfinite(energies))
    snaps, energies, cur_max = eng.run_landscape_segment(P, T, 1, 10, 0.6, 0.1)
    assert 0.004 <= cur_max <= 0.5
    best = eng.lowest_energy_structure(ens)
    assert len(best) == len(P)
    with pytest.raises(ValueError):
        eng.generate_ensemble([], T, 1, 1)
    with pytest.raises(ValueError):
        eng.generate_ensemble(P, T, 0, 1)
    with pytest.raises(ValueError):
        eng.run_landscape_trajectory(P, T, 1, 0)


# ---- speculative rounds (spec_teams > 1): the same chain as one team --------
@pytest.mark.parametrize("teams,cl", [(2, 4), (4, 8), (8, 8), (4, 16)])
def test_spec_teams_match_oracle(teams, cl):
    g, F = _setup("insulin")
    b, st = _gpu_run(g, F, 1, 11, 300, cluster_size=cl, spec_teams=teams)  # crosses a tune window (200)
    x_o, st_o, _ = _oracle_run(g, F, 11, 300)
    assert st["step"][0] == 300
    assert st["n_accepted"][0] == st_o["n_accepted"]
    assert st["n_proposed"][0] == st_o["n_proposed"]
    assert st["cur_max"][0] == pytest.approx(st_o["cur_max"], rel=1e-15)
    np.testing.assert_allclose(b.coords(0), x_o, rtol=0, atol=1e-9)


def test_spec_teams_rebuild_and_batched():
    g, F = _setup("insulin")
    b, st = _gpu_run(g, F, 1, 5, 120, fixed_delta=0.6, T=50.0, cluster_size=4, spec_teams=4)
    x_o, st_o, _ = _oracle_run(g, F, 5, 120, fixed_delta=0.6, T=50.0)
    assert st_o["n_rebuild"] > 0 and st["n_rebuild"][0] == st_o["n_rebuild"]
    np.testing.assert_allclose(b.coords(0), x_o, rtol=0, atol=1e-8)
    b, st = _gpu_run(g, F, 3, 21, 80, cluster_size=2, spec_teams=4)
    for s in range(3):
        x_o, st_o, _ = _oracle_run(g, F, 21, 80, sys_index=s)
        assert st["n_accepted"][s] == st_o["n_accepted"]
        np.testing.assert_allclose(b.coords(s), x_o, rtol=0, atol=1e-9)


def test_spec_teams_bitwise_equal_one_team():
    """Mixed precision: K teams and one team (same cluster size) give the
    same chain — every decision, every coordinate bit for bit.  The running
    energy (a sum of the accepted ΔE) agrees to 1e-12 relative: the two
    kernels inline the FP32 pair arithmetic separately and the compiler may
    contract its multiply-adds differently, which moves a ΔE by an ulp."""
    g, F = _setup("xq8")
    b1, st1 = _gpu_run(g, F, 1, 3, 400, precision="mixed", cluster_size=8, spec_teams=1)
    b4, st4 = _gpu_run(g, F, 1, 3, 400, precision="mixed", cluster_size=8, spec_teams=4)
    assert np.array_equal(b1.coords(0), b4.coords(0))
    for k in ("cur_max", "n_accepted", "n_proposed", "n_rebuild", "step"):
        assert st1[k][0] == st4[k][0], k
    assert abs(st1["energy"][0] - st4["energy"][0]) <= 1e-12 * abs(st1["energy"][0])


def test_tail_launches_follow_the_oracle():
    """Once few chains are short of the step limit, MCRunner launches only
    them, on 16-CTA clusters with speculative teams: every chain is still
    the oracle's, through many host rebuilds."""
    g, F = _setup("insulin")
    n = 12
    b, st, R = _gpu_run(g, F, n, 7, 120, fixed_delta=0.6, T=50.0, cluster_size=1, spec_teams=1,
                        device_rebuild=False, runner=True)
    assert R.tail_launches > 0 and R.rebuilds > 0
    for s in range(n):
        x_o, st_o, _ = _oracle_run(g, F, 7, 120, fixed_delta=0.6, T=50.0, sys_index=s)
        assert st["step"][s] == 120
        # a chain that drifted on its last proposal is rebuilt when the run
        # ends; the oracle leaves the flag for the chain's next step
        assert st["n_rebuild"][s] == st_o["n_rebuild"] + (st_o["need_rebuild"] != 0)
        assert st["n_accepted"][s] == st_o["n_accepted"]
        np.testing.assert_allclose(b.coords(s), x_o, rtol=0, atol=1e-8)


def test_tail_launches_bitwise_equal_fixed_shape():
    """Mixed precision, the same batch with and without tail launches: the
    same decisions and the same coordinates bit for bit.  The running
    energies agree to 1e-9 relative: kernels of different cluster sizes are
    separate instantiations, whose FP32 pair arithmetic the compiler may
    contract differently (an ulp of a pair term)."""
    g, F = _setup("xq8")
    kw = dict(precision="mixed", fixed_delta=0.4, T=30.0, cluster_size=1, spec_teams=1, device_rebuild=False)
    b1, st1, R1 = _gpu_run(g, F, 6, 3, 300, tail_shape=False, runner=True, **kw)
    b2, st2, R2 = _gpu_run(g, F, 6, 3, 300, tail_shape=True, runner=True, **kw)
    assert R1.tail_launches == 0 < R2.tail_launches
    for s in range(6):
        assert np.array_equal(b1.coords(s), b2.coords(s)), s
        for k in ("cur_max", "n_accepted", "n_proposed", "n_rebuild", "step"):
            assert st1[k][s] == st2[k][s], (s, k)
        assert abs(st1["energy"][s] - st2["energy"][s]) <= 1e-9 * abs(st1["energy"][s])


def test_team_counts_mixed_on_one_scratch():
    """A 2-team run, then a 4-team run on the same batch scratch (sized for
    four teams): the 2-team launches' round buffers lie over team 2's move
    scratch and are left zeroed, so the 4-team run is the oracle's chain."""
    from protein_physics_b200.device import DeviceBatch
    from protein_physics_b200.mc import MCRunner
    from oracle import Oracle, oracle_mc
    g, F = _setup("insulin")
    b = DeviceBatch([(g["xyz"], g["q"], g["r"], g["eps"], F)], precision="fp64")
    MCRunner(b, 0.6, 5, cluster_size=8, spec_teams=2).run_to(60)
    x_mid = b.coords(0).copy()
    R = MCRunner(b, 0.6, 9, cluster_size=8, spec_teams=4)
    st = R.run_to(150)
    x_o, st_o, _ = oracle_mc(Oracle(), F, x_mid, g["q"], g["r"], g["eps"], 9, 150, temperature=0.6)
    assert st["n_accepted"][0] == st_o["n_accepted"]
    np.testing.assert_allclose(b.coords(0), x_o, rtol=0, atol=1e-9)


def test_launch_systems_rejects_bad_counts():
    from protein_physics_b200 import _lib
    g, F = _setup("insulin")
    b, st, R = _gpu_run(g, F, 2, 1, 1, cluster_size=1, spec_teams=1, device_rebuild=False, runner=True)
    cfg = _lib.AlmaMCConfig.from_buffer_copy(R.cfg)
    cfg.launch_systems = 3  # more than the batch holds
    assert R._run(cfg, 2) == _lib.ALMA_EINVAL
    cfg.launch_systems, cfg.sys_order = 1, None  # a count needs an order
    assert R._run(cfg, 2) == _lib.ALMA_EINVAL


# ---- rebuilds inside the persistent kernel ----------------------------------
@pytest.mark.parametrize("cl", [1, 8])
def test_device_rebuild_matches_oracle_and_host_build(cl):
    """Large fixed angles drift the chain past half the skin many times: the
    in-kernel rebuild gives the oracle's trajectory, and the list it leaves
    equals a fresh host build of the same coordinates, row order included."""
    from protein_physics_b200.device import DeviceBatch
    g, F = _setup("insulin")
    b, st, R = _gpu_run(g, F, 1, 5, 120, fixed_delta=0.6, T=50.0, cluster_size=cl, spec_teams=1, runner=True)
    x_o, st_o, _ = _oracle_run(g, F, 5, 120, fixed_delta=0.6, T=50.0)
    assert st_o["n_rebuild"] > 0
    assert st["n_rebuild"][0] == st_o["n_rebuild"]
    assert st["n_accepted"][0] == st_o["n_accepted"]
    np.testing.assert_allclose(b.coords(0), x_o, rtol=0, atol=1e-8)
    assert R.rebuilds == 0  # every rebuild ran on the device
    ref = b.ref_xyz[:g.n, :3].cpu().numpy()
    h = DeviceBatch([(ref, g["q"], g["r"], g["eps"], F)], precision="fp64")
    h.build_nl()
    for half in (True, False):
        for short in (False, True):
            a1, a2, a3 = b.nl_host(0, half=half, short=short)
            b1, b2, b3 = h.nl_host(0, half=half, short=short)
            assert np.array_equal(a1, b1) and np.array_equal(a2, b2) and np.array_equal(a3, b3), (half, short)


def test_device_rebuild_batched_equals_host_rebuild():
    g, F = _setup("insulin")
    b1, st1 = _gpu_run(g, F, 3, 21, 120, fixed_delta=0.5, T=30.0, cluster_size=1, spec_teams=1, device_rebuild=True)
    b2, st2 = _gpu_run(g, F, 3, 21, 120, fixed_delta=0.5, T=30.0, cluster_size=1, spec_teams=1, device_rebuild=False)
    for s in range(3):
        assert st1["n_rebuild"][s] == st2["n_rebuild"][s] > 0
        assert st1["n_accepted"][s] == st2["n_accepted"][s]
        assert np.array_equal(b1.coords(s), b2.coords(s))
        assert st1["energy"][s] == pytest.approx(st2["energy"][s], rel=1e-11)


def test_spec_wait_runs_out_and_reports():
    """The speculative rounds' cross-team wait is bounded: a team alone at a
    barrier gives up after its poll limit, raises ALMA_ST_SPEC_ABORT and
    returns; the context stays usable."""
    import time
    from protein_physics_b200 import _lib
    L = _lib.lib()
    buf = torch.zeros(L.alma_spec_round_bytes(), dtype=torch.uint8, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    aborted = torch.zeros(1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    t0 = time.perf_counter()
    _lib.check(L.alma_spec_wait_selftest(buf.data_ptr(), status.data_ptr(), aborted.data_ptr(), stream),
               "alma_spec_wait_selftest")
    torch.cuda.synchronize()
    assert int(aborted.item()) == 1
    assert int(status.item()) & _lib.ST_SPEC_ABORT
    assert time.perf_counter() - t0 < 30.0
    assert float(torch.ones(4, device="cuda").sum()) == 4.0  # the context still works

"""GPU parity of the analytic backward (alma_forces).

Checks, through the C ABI:
  * against an FP64 torch-autograd restatement of the reference energy
    (oracle/torch_energy.py, itself pinned to the oracle energies at 1e-15):
    FP64 mode to 1e-9 relative (2^-32 fixed-point floor), mixed mode
    (FP32 pair / HCT-derivative arithmetic) to 2e-4 of the atom's largest
    component;
  * against central finite differences of the oracle's FP64 energy
    (h = 1e-4 Å, neighbor list fixed) on 64 random atoms: within 1e-5
    relative, plus 2e-6 kcal/mol/Å for the rounding noise of the FD
    quotient (its energies are ~1e4 kcal/mol); atoms with a pair within
    1e-3 Å of the 12 Å cutoff, where the reference energy is discontinuous,
    are not drawn;
  * determinism, batched == single, system mask.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _system(golden):
    from protein_physics_b200.topology import flatten
    return golden["xyz"], golden["q"], golden["r"], golden["eps"], flatten(golden.topology())


def _device_forces(systems, precision):
    from protein_physics_b200.device import DeviceBatch
    b = DeviceBatch(systems, precision=precision)
    b.build_nl()
    b.energy_terms()
    return b, b.forces()[:b.natoms, :3].cpu().numpy()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_forces_vs_torch_autograd(golden, oracle, precision):
    from torch_energy import TorchEnergy
    sysd = _system(golden)
    b, g = _device_forces([sysd], precision)
    ptr, cols = oracle.nl_build(golden["xyz"])
    TE = TorchEnergy(golden["q"], golden["r"], golden["eps"], ptr, cols, sysd[4])
    E, gt = TE.energy_and_grad(golden["xyz"])
    scale = np.maximum(np.abs(gt).max(axis=1), 1.0)
    err = np.abs(g - gt).max(axis=1) / scale
    tol = 1e-9 if precision == "fp64" else 2e-4
    assert err.max() <= tol, (precision, int(err.argmax()), g[err.argmax()], gt[err.argmax()])


def _fd_atoms(xyz, ptr, cols, n_pick, rng, h):
    n = xyz.shape[0]
    near_cut = np.zeros(n, bool)
    I = np.repeat(np.arange(n), np.diff(ptr))
    r = np.sqrt(((xyz[I] - xyz[cols]) ** 2).sum(1))
    bad = np.abs(r - 12.0) < 1e-3 + 2 * h
    near_cut[I[bad]] = True
    near_cut[cols[bad]] = True
    ok = np.flatnonzero(~near_cut)
    return rng.choice(ok, size=min(n_pick, ok.size), replace=False)


@pytest.mark.parametrize("name", ["insulin", "xq8"])
def test_forces_vs_finite_differences(name, oracle):
    from conftest import Golden
    from oracle import TopoArrays
    g = Golden(name)
    sysd = _system(g)
    _, gd = _device_forces([sysd], "fp64")
    _, gm = _device_forces([sysd], "mixed")
    x0 = np.array(g["xyz"], np.float64)
    nl = oracle.nl_build(x0)
    topo = TopoArrays(sysd[4])
    h = 1e-4

    def E(x):
        a = oracle.born_radii(x, g["r"], nl)
        return oracle.energy(x, g["q"], g["r"], g["eps"], nl, a, topo)[4]

    atoms = _fd_atoms(x0, nl[0], nl[1], 64, np.random.default_rng(7), h)
    worst = {"fp64": 0.0, "mixed": 0.0}
    for i in atoms:
        fd = np.zeros(3)
        for c in range(3):
            xp = x0.copy()
            xp[i, c] += h
            xm = x0.copy()
            xm[i, c] -= h
            fd[c] = (E(xp) - E(xm)) / (2 * h)
        for prec, gg in (("fp64", gd), ("mixed", gm)):
            err = np.abs(gg[i] - fd).max()
            tol = 1e-5 * np.abs(fd).max() + 2e-6
            worst[prec] = max(worst[prec], err / tol)
    assert worst["fp64"] <= 1.0, worst
    assert worst["mixed"] <= 1.0, worst


def test_forces_deterministic_batched_and_masked():
    from conftest import Golden
    from protein_physics_b200.device import DeviceBatch
    systems = [_system(Golden(n)) for n in ("xq8", "insulin", "synth64")]
    B = DeviceBatch(systems)
    B.energy_terms()
    g1 = B.forces().cpu().numpy()
    g2 = B.forces().cpu().numpy()
    assert np.array_equal(g1, g2)
    for s, sysd in enumerate(systems):
        _, gs = _device_forces([sysd], "mixed")
        a0, a1 = B.atom_off_h[s], B.atom_off_h[s + 1]
        assert np.array_equal(g1[a0:a1, :3], gs)
    # masked: only system 1 is written
    out = torch.full_like(B.forces(), 7.0)
    mask = torch.tensor([0, 1, 0], dtype=torch.uint8, device="cuda")
    B.forces(sys_mask=mask, out=out)
    o = out.cpu().numpy()
    a0, a1 = B.atom_off_h[1], B.atom_off_h[2]
    assert np.array_equal(o[a0:a1], g1[a0:a1])
    assert np.all(o[:a0] == 7.0) and np.all(o[a1:B.natoms] == 7.0)


def test_forces_no_topology_and_empty():
    from conftest import Golden
    from protein_physics_b200.device import DeviceBatch
    from torch_energy import TorchEnergy
    from oracle import Oracle
    g = Golden("insulin")
    b = DeviceBatch([(g["xyz"], g["q"], g["r"], g["eps"], None)], precision="fp64")
    b.energy_terms()
    f = b.forces()[:g.n, :3].cpu().numpy()
    ptr, cols = Oracle().nl_build(g["xyz"])
    _, gt = TorchEnergy(g["q"], g["r"], g["eps"], ptr, cols, None).energy_and_grad(g["xyz"])
    assert np.abs(f - gt).max() <= 1e-9 * max(1.0, np.abs(gt).max())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_evaluate_graph_equals_eager(precision):
    """DeviceBatch.evaluate(graph=True) — the list build, Born radii, energy
    terms and gradient replayed as one CUDA graph — gives the eager results
    bit for bit, also after the coordinates change between replays and
    through the autograd path."""
    from conftest import Golden
    from protein_physics_b200.autograd import EnergyModel
    from protein_physics_b200.device import DeviceBatch
    systems = [_system(Golden(n)) for n in ("insulin", "synth64")]
    eager = DeviceBatch(systems, precision=precision)
    graphed = DeviceBatch(systems, precision=precision)
    rng = np.random.default_rng(3)
    n = eager.natoms
    x0 = eager.xyz[:n, :3].clone()
    for it in range(4):
        x = x0 + torch.as_tensor(rng.normal(0, 0.3 * it, (n, 3)), device="cuda")
        eager.xyz[:n, :3].copy_(x)
        graphed.xyz[:n, :3].copy_(x)
        te, ge = eager.evaluate()
        tg, gg = graphed.evaluate(graph=True)
        assert torch.equal(te, tg), it
        assert torch.equal(ge[:n], gg[:n]), it
    model = EnergyModel(systems, precision=precision, graph=True)
    xg = x.clone().requires_grad_()
    model(xg).sum().backward()
    assert torch.equal(xg.grad, ge[:n, :3])

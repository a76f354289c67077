"""alma_move_dE_noalloc — the ΔE entry point for callers that cannot
allocate device memory (their host owns the GPU's memory, or their loop
cannot afford cudaMalloc's device-wide synchronisation).  It must give the
results of alma_move_dE with caller scratch, call after call, although
every call reuses the one built-in scratch area.

This file sorts last so that a run stopping at the first failure has run
every other test first; it also passes alone in a fresh process.  The
tests check equality with the caller-scratch entry over calls in a row,
that a call allocates no device memory, a batch just under the maximum,
and the rejection of larger ones.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _batch(names, precision):
    from conftest import Golden
    from protein_physics_b200.device import DeviceBatch
    from protein_physics_b200.topology import flatten
    gs = [Golden(n) for n in names]
    b = DeviceBatch([(g["xyz"], g["q"], g["r"], g["eps"], flatten(g.topology())) for g in gs], precision=precision)
    b.build_nl()
    b.born_radii()
    return b


def _call(b, fn_name, kind, a, delta, with_scratch):
    from protein_physics_b200 import _lib
    from protein_physics_b200.device import _ptr, _t
    L = _lib.lib()
    fn = getattr(L, fn_name)
    kind_t = _t(np.asarray(kind, np.int32), torch.int32)
    a_t = _t(np.asarray(a, np.int32), torch.int32)
    d_t = _t(np.asarray(delta, np.float64).reshape(-1, 2), torch.float64)
    dE = torch.zeros(b.nsys, dtype=torch.float64, device="cuda")
    dterms = torch.zeros((b.nsys, 4), dtype=torch.float64, device="cuda")
    args = [C.byref(b.batch_s), C.byref(b.topo_s), C.byref(b.nl_s), C.byref(b.params), b.prec]
    if with_scratch:
        args.append(C.c_void_p(_ptr(b.scratch)))
    args += [C.c_void_p(_ptr(kind_t)), C.c_void_p(_ptr(a_t)), C.c_void_p(_ptr(d_t)), 0, C.c_void_p(_ptr(dE)),
             C.c_void_p(_ptr(dterms)), b._sp()]
    rc = fn(*args)
    _lib.check(rc, fn_name)
    torch.cuda.synchronize()
    return dE.cpu().numpy(), dterms.cpu().numpy()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_noalloc_matches_scratch_entry_two_calls_in_a_row(precision):
    from protein_physics_b200 import _lib
    L = _lib.lib()
    L.alma_move_dE_noalloc.argtypes = [C.c_void_p] * 4 + [C.c_int] + [C.c_void_p] * 3 + [C.c_int] + [C.c_void_p] * 3
    b = _batch(("insulin", "xq8"), precision)
    calls = [([0, 1], [3, 2], [[0.15, 0.0], [-0.05, 0.0]]),   # torsion on insulin, crankshaft on 1XQ8
             ([0, 0], [40, 111], [[-0.3, 0.0], [0.2, 0.0]])]  # a second call reuses the built-in area
    for kind, a, delta in calls:
        e_ref, t_ref = _call(b, "alma_move_dE", kind, a, delta, True)
        e_na, t_na = _call(b, "alma_move_dE_noalloc", kind, a, delta, False)
        # same kernel, same reduction order: agreement to the parity tests' FP64 bar
        np.testing.assert_allclose(e_na, e_ref, rtol=1e-12, atol=1e-9)
        np.testing.assert_allclose(t_na, t_ref, rtol=1e-12, atol=1e-9)


def test_noalloc_rejects_batches_beyond_its_area():
    from conftest import Golden
    from protein_physics_b200 import _lib
    from protein_physics_b200.device import DeviceBatch
    from protein_physics_b200.topology import flatten
    L = _lib.lib()
    L.alma_move_dE_noalloc.argtypes = [C.c_void_p] * 4 + [C.c_int] + [C.c_void_p] * 3 + [C.c_int] + [C.c_void_p] * 3
    g = Golden("insulin")
    F = flatten(g.topology())
    reps = 16384 // g.n + 1  # just above the built-in limit
    b = DeviceBatch([(g["xyz"], g["q"], g["r"], g["eps"], F)] * reps)
    assert b.natoms > 16384
    with pytest.raises(ValueError, match="exceeds the built-in scratch area"):
        _call(b, "alma_move_dE_noalloc", [0] * reps, [1] * reps, [[0.1, 0.0]] * reps, False)


def test_noalloc_allocates_nothing_and_fills_its_area():
    """Several calls on a batch just under the documented maximum (24
    copies of insulin, 15,768 atoms): the GPU's free memory does not move
    across them, and every call equals the caller-scratch entry."""
    from conftest import Golden
    from protein_physics_b200 import _lib
    from protein_physics_b200.device import DeviceBatch, _ptr, _t
    from protein_physics_b200.topology import flatten
    L = _lib.lib()
    L.alma_move_dE_noalloc.argtypes = [C.c_void_p] * 4 + [C.c_int] + [C.c_void_p] * 3 + [C.c_int] + [C.c_void_p] * 3
    g = Golden("insulin")
    F = flatten(g.topology())
    reps = 16384 // g.n
    b = DeviceBatch([(g["xyz"], g["q"], g["r"], g["eps"], F)] * reps, precision="mixed")
    assert 16384 - g.n < b.natoms <= 16384
    b.build_nl()
    b.born_radii()
    rng = np.random.default_rng(5)
    kind = _t(np.zeros(reps, np.int32), torch.int32)
    a = _t(rng.integers(0, F.nrb, size=reps).astype(np.int32), torch.int32)
    delta = _t(np.stack([rng.uniform(-0.3, 0.3, reps), np.zeros(reps)], 1), torch.float64)
    outs = [(torch.zeros(reps, dtype=torch.float64, device="cuda"),
             torch.zeros((reps, 4), dtype=torch.float64, device="cuda")) for _ in range(2)]
    common = [C.byref(b.batch_s), C.byref(b.topo_s), C.byref(b.nl_s), C.byref(b.params), b.prec]
    move = [C.c_void_p(_ptr(kind)), C.c_void_p(_ptr(a)), C.c_void_p(_ptr(delta)), 0]

    def noalloc():
        dE, dt = outs[0]
        _lib.check(L.alma_move_dE_noalloc(*common, *move, C.c_void_p(_ptr(dE)), C.c_void_p(_ptr(dt)), b._sp()),
                   "alma_move_dE_noalloc")

    noalloc()  # first call: the address lookup
    dE, dt = outs[1]
    _lib.check(L.alma_move_dE(*common, C.c_void_p(_ptr(b.scratch)), *move, C.c_void_p(_ptr(dE)),
                              C.c_void_p(_ptr(dt)), b._sp()), "alma_move_dE")
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(4):
        noalloc()
        torch.cuda.synchronize()
        np.testing.assert_allclose(outs[0][0].cpu().numpy(), outs[1][0].cpu().numpy(), rtol=1e-12, atol=1e-9)
        np.testing.assert_allclose(outs[0][1].cpu().numpy(), outs[1][1].cpu().numpy(), rtol=1e-12, atol=1e-9)
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0

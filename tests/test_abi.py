"""The C-ABI library loads and exports every entry point include/*.h
declares; host-side helpers behave (no GPU needed)."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[\w\s\*]+?\b(alma_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    from protein_physics_b200 import _lib
    L = _lib.lib()
    syms = declared_symbols()
    assert len(syms) >= 10
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    assert L.alma_abi_version() == 1


def test_reference_params():
    from protein_physics_b200 import _lib
    p = _lib.reference_params()
    assert p.coulomb == 332.0636 and p.kappa == 0.1257 and p.gamma_sa == 0.00542 and p.hard_frac == 0.6
    assert p.nl_rcut2 == 196.0 and p.pair_cut2 == 144.0 and p.half_skin2 == 1.0


def test_errors_are_reported():
    from protein_physics_b200 import _lib
    L = _lib.lib()
    rc = L.alma_nl_build(None, None, None, None, None, None, 0, None)
    assert rc == _lib.ALMA_EINVAL
    assert b"alma_nl_build" in L.alma_last_error()
    with pytest.raises(ValueError):
        _lib.check(rc, "x")
    # exclusion windows: arguments are checked before any device work
    assert L.alma_excl_window(None, None, -1, None, None) == _lib.ALMA_EINVAL
    assert L.alma_excl_window(None, None, 5, None, None) == _lib.ALMA_EINVAL
    assert b"alma_excl_window" in L.alma_last_error()
    assert L.alma_excl_window(None, None, 0, None, None) == _lib.ALMA_OK  # nothing to do


def test_topo_sides_dfs_order():
    from protein_physics_b200 import _lib
    # path 0-1-2-3 with a branch 2-4: side of (1,2) from 2 = [2, 4, 3] (stack order)
    adj = [[1], [0, 2], [1, 3, 4], [2], [2]]
    ptr = np.zeros(6, np.int64)
    ptr[1:] = np.cumsum([len(a) for a in adj])
    idx = np.array([j for a in adj for j in a], np.int32)
    sides = _lib.topo_sides(5, ptr, idx, [(1, 2), (0, 1), (2, 1)])
    assert sides[0] == [2, 4, 3]
    assert sorted(sides[1]) == [1, 2, 3, 4]
    assert sorted(sides[2]) == [0, 1]
    lo, hi, cnt, ex_ptr, ex_idx = _lib.topo_sides_compact(5, ptr, idx, [(1, 2), (0, 1), (2, 1)])
    assert list(cnt) == [3, 4, 2]
    assert (lo[0], hi[0]) == (2, 5) and ex_ptr[1] == 0
    assert (lo[1], hi[1]) == (1, 5)


def test_workspace_sizes_are_monotone():
    from protein_physics_b200 import _lib
    L = _lib.lib()
    assert L.alma_nl_workspace_bytes(1, 1000, 10000) < L.alma_nl_workspace_bytes(2, 2000, 20000)
    assert L.alma_move_scratch_bytes(100) < L.alma_move_scratch_bytes(1000)


def test_noalloc_area_holds_its_documented_batch():
    """The built-in scratch of alma_move_dE_noalloc holds the scratch of a
    batch of ALMA_NOALLOC_MAX_ATOMS atoms (the header's promise), so a batch
    within the documented limit is never turned away."""
    from protein_physics_b200 import _lib
    L = _lib.lib()
    hdr = open(os.path.join(ROOT, "include", "alma_b200.h")).read()
    max_atoms = int(re.search(r"#define ALMA_NOALLOC_MAX_ATOMS (\d+)", hdr).group(1))
    assert L.alma_move_scratch_bytes(max_atoms) <= L.alma_move_noalloc_capacity_bytes()


def test_engine_fails_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from protein_physics_b200 import Particle, PhysicsEngine
    with pytest.raises(RuntimeError):
        PhysicsEngine().calculate_potential([Particle(0, 0, 0, 1.0), Particle(3, 0, 0, -1.0)])


def test_bench_host_threads_follows_omp_setting(monkeypatch):
    """bench.py sizes the e2e call like the reference arm: one candidate per
    host thread, OMP_NUM_THREADS first."""
    import importlib
    import sys
    sys.path.insert(0, ROOT)
    bench = importlib.import_module("bench")
    monkeypatch.setenv("OMP_NUM_THREADS", "3")
    assert bench.host_threads() == 3
    monkeypatch.delenv("OMP_NUM_THREADS")
    assert bench.host_threads() >= 1


def test_bench_reference_inputs_load_nothing_of_the_package():
    """The reference arm builds its inputs with the chain generator loaded
    by path: protein_physics_b200 (and its native library) stay unloaded,
    and both arms describe the workload with the same config."""
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, %r); import bench; "
            "chains, temps = bench.c3_inputs(0, n_chains=2); "
            "assert not [m for m in sys.modules if m.startswith('protein_physics_b200')], sorted(sys.modules); "
            "c = bench.config_of('batched', chains); assert c == bench.config_of('batched', chains); "
            "assert c['chains'] == 2 and c['atoms'] == sum(len(x['xyz']) for x in chains); "
            "assert len(temps) == 2 and abs(temps[0] - 280 * 0.0019872) < 1e-12; print('ok')" % ROOT)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stderr[-2000:]


def test_ctypes_structs_match_the_library_layout():
    """Every struct the Python binding mirrors has the size the library
    was compiled with (alma_struct_size): a field added on one side only
    would shift every later field."""
    from protein_physics_b200 import _lib
    L = _lib.lib()
    L.alma_struct_size.restype = ctypes.c_size_t
    L.alma_struct_size.argtypes = [ctypes.c_int32]
    mirrors = [_lib.AlmaParams, _lib.AlmaBatch, _lib.AlmaTopo, _lib.AlmaNL, _lib.AlmaMCConfig, _lib.AlmaChainState,
               _lib.AlmaTorsionTree, _lib.AlmaMalaState, _lib.AlmaMalaConfig]
    for which, cls in enumerate(mirrors):
        assert L.alma_struct_size(which) == ctypes.sizeof(cls), cls.__name__
    assert L.alma_struct_size(99) == 0

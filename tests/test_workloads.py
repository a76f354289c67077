"""The benchmark chains in workloads/: what the configurations ask for,
and the coordinates the reference goldens were made from (CPU)."""
import hashlib
import os

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

CASES = [("c2_chain_300res.npz", "wl_c2", 300, (16.5, 19.5)),
         ("c4_globule_1000res.npz", "wl_c4", 1000, (27.0, 32.0)),
         ("c5_multidomain_4x1000res.npz", "wl_c5", 4030, None)]


@pytest.mark.parametrize("fname,golden,n_res,rg_band", CASES)
def test_workload_chain(fname, golden, n_res, rg_band):
    d = np.load(os.path.join(ROOT, "workloads", fname), allow_pickle=False)
    xyz = d["xyz"].astype(np.float64)
    assert len(d["sequence"]) == n_res
    assert xyz.shape == (len(d["atomnames"]), 3) == (len(d["charge"]), 3)
    assert np.all(np.isfinite(xyz))
    if rg_band:  # a compact chain: the radius of gyration the generator aims at
        c = xyz - xyz.mean(0)
        rg = float(np.sqrt((c * c).sum(1).mean()))
        assert rg_band[0] <= rg <= rg_band[1], rg
    g = np.load(os.path.join(GOLDEN, golden + ".npz"))
    assert str(g["fixture"]) == fname
    assert hashlib.sha256(np.ascontiguousarray(xyz).tobytes()).hexdigest() == str(g["xyz_sha"])


def test_multidomain_domains_are_compact():
    d = np.load(os.path.join(ROOT, "workloads", "c5_multidomain_4x1000res.npz"), allow_pickle=False)
    ridx = d["res_idx"]
    for k in range(4):
        a0, a1 = np.searchsorted(ridx, 1010 * k), np.searchsorted(ridx, 1010 * k + 1000)
        x = d["xyz"][a0:a1]
        c = x - x.mean(0)
        assert float(np.sqrt((c * c).sum(1).mean())) < 36.0

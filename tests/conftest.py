import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "protein-structure-analysis_b200")
ORACLE_DIR = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (PKG_DIR, ORACLE_DIR, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA sm_100 device")


def _ensure_built():
    lib = os.path.join(PKG_DIR, "protein_physics_b200", "libalma_b200.so")
    if not os.path.exists(lib):
        subprocess.run([sys.executable, os.path.join(PKG_DIR, "build.py")], check=True)
    if not os.path.exists(os.path.join(ORACLE_DIR, "alma_oracle.so")):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR, "oracle"], check=True)


_ensure_built()


class Golden:
    """One golden system: inputs + reference outputs (tests/golden/*.npz)."""

    def __init__(self, name):
        self.name = name
        d = np.load(os.path.join(GOLDEN, name + ".npz"))
        self.d = {k: d[k] for k in d.files}
        if "fixture" in self.d:  # a benchmark chain: inputs from workloads/, checked by hash
            import hashlib
            w = np.load(os.path.join(ROOT, "workloads", str(self.d["fixture"])), allow_pickle=False)
            xyz = w["xyz"].astype(np.float64)
            assert hashlib.sha256(np.ascontiguousarray(xyz).tobytes()).hexdigest() == str(self.d["xyz_sha"])
            self.d.update(xyz=xyz, q=w["charge"], r=w["radius"], eps=w["epsilon"])
            self.resnames = [str(v) for v in w["resnames"]]
            self.atomnames = [str(v) for v in w["atomnames"]]
            self.res_idx = [int(v) for v in w["res_idx"]]
            return
        with open(os.path.join(GOLDEN, name + ".names.json")) as f:
            m = json.load(f)
        self.resnames, self.atomnames, self.res_idx = m["resnames"], m["atomnames"], m["res_idx"]

    def __getitem__(self, k):
        return self.d[k]

    @property
    def n(self):
        return int(self.d["xyz"].shape[0])

    def topology(self):
        from protein_physics_b200.topology import BondTopology
        T = BondTopology()
        T.build(self.resnames, self.atomnames, self.res_idx)
        for i, j in self.d["ss_in"]:
            T.add_disulfide(int(i), int(j))
        T.identify_concerted_sidechain_pairs(self.d["xyz"])
        return T


GOLDEN_SYSTEMS = ("xq8", "insulin", "synth64")
# the benchmark chains (workloads/*.npz) with their reference goldens
WORKLOAD_SYSTEMS = tuple(n for n in ("wl_c2", "wl_c4", "wl_c5") if os.path.exists(os.path.join(GOLDEN, n + ".npz")))


@pytest.fixture(scope="session", params=GOLDEN_SYSTEMS)
def golden(request):
    return Golden(request.param)


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


def excl_window_np(ptr, cols, n):
    """Exclusion windows (alma_excl_window) restated from CSR rows of
    partners j > i: bit d + 64 of atom i's four words for 0 < |d| < 64, bit
    64 for a partner farther away."""
    w = np.zeros((n, 4), np.uint32)
    for i in range(n):
        for j in cols[ptr[i]:ptr[i + 1]].tolist():
            d = j - i
            if 0 < abs(d) < 64:
                for a, dd in ((i, d), (j, -d)):
                    bit = dd + 64
                    w[a, bit >> 5] |= np.uint32(1 << (bit & 31))
            else:
                w[i, 2] |= np.uint32(1)
                w[j, 2] |= np.uint32(1)
    return w


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False

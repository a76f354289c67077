"""GPU ensemble metrics vs the reference's protein_analysis module (built
from analysis_ext.cpp into oracle/_ref by oracle/Makefile; skipped when it
is absent) and a numpy restatement: 1e-12 relative (the reference build
may contract to FMA)."""
import glob
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _numpy_mean(c):
    d = np.sqrt(((c[:, :, None, :] - c[:, None, :, :]) ** 2).sum(-1))
    return d.mean(0)


@pytest.mark.parametrize("n_snaps,n_ca", [(1, 5), (7, 33), (20, 130)])
def test_matrices_vs_numpy_and_reference(n_snaps, n_ca):
    from protein_physics_b200 import analysis
    c = np.random.default_rng(n_ca).normal(size=(n_snaps, n_ca, 3)) * 12.0
    m = analysis.compute_mean_dist_matrix(c)
    f = analysis.compute_contact_freq_matrix(c, 8.0)
    np.testing.assert_allclose(m, _numpy_mean(c), rtol=1e-12, atol=1e-12)
    d = np.sqrt(((c[:, :, None, :] - c[:, None, :, :]) ** 2).sum(-1))
    fr = (d < 8.0).mean(0)
    np.fill_diagonal(fr, 0.0)
    np.testing.assert_allclose(f, fr, rtol=1e-15, atol=1e-15)  # count * (1/n) vs mean: last-bit rounding
    hits = glob.glob(os.path.join(ROOT, "oracle", "_ref", "protein_analysis*.so"))
    if hits:
        sys.path.insert(0, os.path.dirname(hits[0]))
        import protein_analysis as pa
        np.testing.assert_allclose(m, pa.compute_mean_dist_matrix(c), rtol=1e-12, atol=1e-12)
        np.testing.assert_array_equal(f, pa.compute_contact_freq_matrix(c, 8.0))


def test_device_tensor_in_device_tensor_out():
    from protein_physics_b200 import analysis
    c = torch.randn(4, 40, 3, dtype=torch.float64, device="cuda") * 10
    m = analysis.compute_mean_dist_matrix(c)
    assert m.is_cuda and m.shape == (40, 40)
    np.testing.assert_allclose(m.cpu().numpy(), _numpy_mean(c.cpu().numpy()), rtol=1e-12, atol=1e-12)
    assert analysis.compute_mean_dist_matrix(np.zeros((0, 3, 3))).shape == (3, 3)
    with pytest.raises(ValueError):
        analysis.compute_mean_dist_matrix(np.zeros((3, 3)))

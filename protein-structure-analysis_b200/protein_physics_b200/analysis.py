"""Ensemble metrics on the device — the drop-in for the reference's
`protein_analysis` module functions (analysis_ext.cpp):

    compute_mean_dist_matrix(coords) -> (n_ca, n_ca)
    compute_contact_freq_matrix(coords, cutoff) -> (n_ca, n_ca)

coords: (n_snaps, n_ca, 3) array-like (numpy or a CUDA float64 tensor).
Numpy in, numpy out; a CUDA tensor in, a CUDA tensor out (snapshots that
are already on the device, e.g. from a DeviceBatch, are not copied).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib


def _coords(coords):
    if isinstance(coords, torch.Tensor) and coords.is_cuda:
        t = coords.to(torch.float64).contiguous()
        on_dev = True
    else:
        a = np.asarray(coords, dtype=np.float64)
        t = torch.from_numpy(np.ascontiguousarray(a)).to("cuda")
        on_dev = False
    if t.dim() != 3 or t.shape[2] != 3:
        raise ValueError("coords must be a 3-D array (n_snaps, n_ca, 3)")
    return t, on_dev


def _run(fn, coords, *extra):
    t, on_dev = _coords(coords)
    n_snaps, n_ca = int(t.shape[0]), int(t.shape[1])
    out = torch.zeros((n_ca, n_ca), dtype=torch.float64, device="cuda")
    if n_snaps and n_ca:
        _lib.check(fn(C.c_void_p(t.data_ptr()), n_snaps, n_ca, *extra, C.c_void_p(out.data_ptr()),
                      C.c_void_p(torch.cuda.current_stream().cuda_stream)), fn.__name__)
    return out if on_dev else out.cpu().numpy()


def compute_mean_dist_matrix(coords):
    """Ensemble-mean Cα-Cα distance matrix (alma_mean_dist_matrix)."""
    return _run(_lib.lib().alma_mean_dist_matrix, coords)


def compute_contact_freq_matrix(coords, cutoff):
    """Fraction of snapshots with each pair closer than cutoff Å
    (alma_contact_freq_matrix)."""
    return _run(_lib.lib().alma_contact_freq_matrix, coords, C.c_double(float(cutoff)))

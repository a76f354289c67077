"""GPU parity on the benchmark chains themselves (workloads/*.npz: the
300-residue compact chain of the single-chain benchmark, the 1,000-residue
globule, the 4 x 1,000-residue multi-domain chain of the replica
benchmark) against the reference's own outputs on the same inputs
(tests/golden/wl_*.npz, made by the compiled reference engine).

Bars, as on the smaller goldens:
  * neighbor list: row lengths and the columns in the reference's
    cell-scan order, bit-exact (SHA-256 of the columns);
  * Born radii: 1e-12 (FP64) / 2e-6 (mixed) relative;
  * total energy with and without topology: 1e-10 (FP64) / 1e-6 (mixed)
    relative; SASA, dihedral and disulfide terms 1e-10 (FP64 always);
  * ΔE of 16 torsion moves of up to 30 degrees, 16 of the samplers' own
    size (0.12 rad x lever scale) and 8 crankshaft moves, replayed by the
    reference: FP64 1e-7 kcal/mol + 1e-11 relative (the reference sums the
    before and after cross energies separately, with -ffast-math); mixed
    1e-4 kcal/mol + 1e-14 x sum|terms| for |ΔE| <= 1e3 kcal/mol, and 1e-6
    relative above — turning half of a compact chain by 30 degrees drives
    atoms through each other (ΔE up to ~1e21 kcal/mol), a move the
    Metropolis test rejects at any temperature whatever its last digits.
"""
import hashlib

import numpy as np
import pytest

from conftest import WORKLOAD_SYSTEMS, Golden

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

_CACHE = {}


def _golden(name):
    if name not in _CACHE:  # the topology of the 65k-atom chain takes a while to build: once
        g = Golden(name)
        _CACHE[name] = (g, g.topology())
    return _CACHE[name]


def _batch(name, precision, topo=True):
    from protein_physics_b200.device import DeviceBatch
    from protein_physics_b200.topology import flatten
    g, T = _golden(name)
    return DeviceBatch([(g["xyz"], g["q"], g["r"], g["eps"], flatten(T) if topo else None)], precision=precision)


@pytest.mark.parametrize("name", WORKLOAD_SYSTEMS)
def test_nl_matches_reference(name):
    g, _ = _golden(name)
    b = _batch(name, "mixed")
    b.build_nl()
    rp, cols, _ = b.nl_host(0, half=True)
    assert np.array_equal(np.diff(rp).astype(np.int32), g["nl_row_cnt"])
    assert hashlib.sha256(np.ascontiguousarray(cols.astype(np.int32)).tobytes()).hexdigest() == str(g["nl_sha"])


@pytest.mark.parametrize("name", WORKLOAD_SYSTEMS)
@pytest.mark.parametrize("precision,rtol_born,rtol_e", [("fp64", 1e-12, 1e-10), ("mixed", 2e-6, 1e-6)])
def test_born_and_energy_match_reference(name, precision, rtol_born, rtol_e):
    g, _ = _golden(name)
    b = _batch(name, precision)
    b.build_nl()
    b.born_radii()
    np.testing.assert_allclose(b.born[:g.n].cpu().numpy(), g["born"], rtol=rtol_born, atol=0)
    terms = b.energy_terms()[0].cpu().numpy()
    ref = g["energy_topo"]
    assert abs(terms[4] - ref[4]) <= rtol_e * abs(ref[4]), (terms[4], ref[4])
    np.testing.assert_allclose(terms[:3], ref[:3], rtol=1e-10, atol=1e-9)
    t2 = _batch(name, precision, topo=False).energy_terms()[0].cpu().numpy()
    assert abs(t2[4] - g["energy_notopo"][4]) <= rtol_e * abs(g["energy_notopo"][4])


@pytest.mark.parametrize("name", WORKLOAD_SYSTEMS)
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_move_dE_matches_reference(name, precision):
    g, T = _golden(name)
    b = _batch(name, precision)
    b.build_nl()
    b.born_radii()
    crank = sorted(T.concerted_pairs)
    for kind, code, delta, dE_ref, *terms_ref in g["moves"]:
        if int(kind) == 0:
            k, a = 0, int(code)
        else:
            k, a = 1, crank.index(divmod(int(code), 100000))
        dE, dterms = b.move_dE([k], [a], [[delta, 0.0]])
        dE = float(dE[0].item())
        if precision == "fp64":
            assert abs(dE - dE_ref) <= 1e-7 + 1e-11 * abs(dE_ref), (kind, code, dE, dE_ref)
        elif abs(dE_ref) <= 1e3:
            assert abs(dE - dE_ref) <= 1e-4 + 1e-14 * np.sum(np.abs(terms_ref)), (kind, code, dE, dE_ref)
        else:
            assert abs(dE - dE_ref) <= 1e-6 * abs(dE_ref), (kind, code, dE, dE_ref)
        np.testing.assert_allclose(dterms[0].cpu().numpy()[1:], terms_ref[1:], atol=1e-8, rtol=1e-11)

"""Sampling statistics of the device Monte Carlo against the reference's
own sampler on the same start.

The reference draws from an unseeded generator (physics_engine.cpp:2236,
:2535), so its trajectories cannot be matched draw for draw; the policy
restatement is checked trajectory by trajectory against the oracle's MC
driver elsewhere (test_gpu_mc.py).  Here the two samplers are compared as
distributions, on the seeded 64-residue chain of the goldens at T = 0.6
kcal/mol:

  * generate_ensemble (:2273-2543): 64 candidates x 300 proposals each;
    the final energies of both ensembles (scored by the reference's own
    calculate_potential) must agree — the difference of the means within
    4 standard errors and a two-sample Kolmogorov-Smirnov test above
    p = 1e-3;
  * run_landscape_segment (:2557-2951, returns the adapted cur_max): the
    final cur_max of 24 independent segments of 600 proposals must agree
    the same way (cur_max follows the acceptance rate through the
    adaptation window, :2515-2526);
  * the acceptance rate of the device chains must fall inside the
    reference's 99.9 % interval from run_mc_diagnostic (:3300), whose
    moves are the landscape skeleton's torsion / crankshaft moves.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _ref():
    import sys
    from oracle import ref_so_path
    path = ref_so_path()
    if path is None:
        pytest.skip("reference engine not built (oracle/_ref)")
    import os
    sys.path.insert(0, os.path.dirname(path))
    import protein_physics as pp
    return pp


def _start():
    from conftest import Golden
    g = Golden("synth64")
    return g


def _ks_p(a, b):
    from scipy.stats import ks_2samp
    return float(ks_2samp(a, b).pvalue)


def _means_agree(a, b, k=4.0):
    a, b = np.asarray(a, float), np.asarray(b, float)
    se = np.sqrt(a.var(ddof=1) / len(a) + b.var(ddof=1) / len(b))
    return abs(a.mean() - b.mean()) <= k * se + 1e-12, (a.mean(), b.mean(), se)


def test_generate_ensemble_energy_distribution_matches_reference():
    pp = _ref()
    from protein_physics_b200 import Particle, PhysicsEngine
    g = _start()
    R = pp.BondTopology()
    R.build(g.resnames, g.atomnames, g.res_idx)
    Pr = [pp.Particle(*map(float, x), float(q), float(r), float(e)) for x, q, r, e in
          zip(g["xyz"], g["q"], g["r"], g["eps"])]
    P = [Particle(*x, q, r, e) for x, q, r, e in zip(g["xyz"], g["q"], g["r"], g["eps"])]
    ref_eng = pp.PhysicsEngine()
    ens_ref = ref_eng.generate_ensemble(Pr, R, 64, 300, 0.6, 0.12)
    ens_dev = PhysicsEngine(precision="mixed", seed=31).generate_ensemble(P, g.topology(), 64, 300, 0.6, 0.12)
    score = lambda m: ref_eng.calculate_potential([pp.Particle(p.x, p.y, p.z, p.charge, p.radius, p.epsilon)
                                                   for p in m], R)
    e_ref = [score(m) for m in ens_ref]
    e_dev = [score(m) for m in ens_dev]
    ok, info = _means_agree(e_dev, e_ref)
    assert ok, info
    assert _ks_p(e_dev, e_ref) > 1e-3, (np.mean(e_dev), np.mean(e_ref))
    e0 = ref_eng.calculate_potential(Pr, R)
    assert np.mean(e_ref) < e0 and np.mean(e_dev) < e0  # both samplers relax the start


def test_landscape_cur_max_and_acceptance_match_reference():
    pp = _ref()
    from protein_physics_b200 import Particle, PhysicsEngine
    g = _start()
    R = pp.BondTopology()
    R.build(g.resnames, g.atomnames, g.res_idx)
    Pr = [pp.Particle(*map(float, x), float(q), float(r), float(e)) for x, q, r, e in
          zip(g["xyz"], g["q"], g["r"], g["eps"])]
    P = [Particle(*x, q, r, e) for x, q, r, e in zip(g["xyz"], g["q"], g["r"], g["eps"])]
    ref_eng = pp.PhysicsEngine()
    eng = PhysicsEngine(precision="mixed", seed=77)
    T = g.topology()
    cm_ref = [ref_eng.run_landscape_segment(Pr, R, 1, 600, 0.6, 0.12)[2] for _ in range(24)]
    cm_dev = [eng.run_landscape_segment(P, T, 1, 600, 0.6, 0.12)[2] for _ in range(24)]
    ok, info = _means_agree(cm_dev, cm_ref)
    assert ok, info

"""protein_physics_b200 — B200-native drop-in for ALMA's `protein_physics`
nonbonded-energy / Monte Carlo ΔE path.

Same Python surface as the reference module (physics_engine.cpp:3692-3888):
``Particle``, ``BondKind``, ``RotBond``, ``BondTopology`` and
``PhysicsEngine`` with ``calculate_potential``, ``generate_ensemble``,
``run_landscape_trajectory``, ``run_landscape_segment``,
``lowest_energy_structure``, ``num_threads`` and the static
``device_name``.  The arithmetic runs in hand-written sm_100a CUDA kernels
(libalma_b200.so, C ABI in include/alma_b200.h); there is no CPU fallback.
"""
from .topology import BondKind, BondTopology, RotBond, flatten  # noqa: F401
from .engine import Particle, PhysicsEngine  # noqa: F401

__all__ = ["Particle", "BondKind", "RotBond", "BondTopology", "PhysicsEngine", "flatten"]

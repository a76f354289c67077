"""Drop-in ``Particle`` and ``PhysicsEngine`` over the device engine.

Mirrors the reference bindings (physics_engine.cpp:3692-3888 and the CUDA
module physics_engine_cuda.cu:1287-1396): argument names, positional order,
defaults, value semantics (particle lists in, new lists out) and error
types (ValueError for bad input, RuntimeError for device errors).
"""
from __future__ import annotations

import numpy as np

from . import topology as _topology


class Particle:
    """One atom (physics_engine.cpp:208-214): position (Å), partial charge
    (e), LJ radius R* (Å, also the intrinsic Born radius), well depth
    epsilon (kcal/mol), water flag (unused by the energy)."""

    __slots__ = ("x", "y", "z", "charge", "radius", "epsilon", "is_water")

    def __init__(self, x, y, z, charge, radius=1.9, epsilon=0.1, is_water=False):
        self.x, self.y, self.z = float(x), float(y), float(z)
        self.charge, self.radius, self.epsilon = float(charge), float(radius), float(epsilon)
        self.is_water = bool(is_water)

    def __repr__(self):
        return (f"Particle({self.x!r}, {self.y!r}, {self.z!r}, {self.charge!r}, {self.radius!r}, "
                f"{self.epsilon!r}, {self.is_water!r})")


_FLAT_FIELDS = ("excl_ptr", "excl_cols", "rb_i", "rb_j", "rb_kind", "rb_scale", "side_ptr", "side_idx", "side_lo",
                "side_hi", "dih_abcd", "term_off", "term_v2", "term_n", "term_gamma", "ss", "crank", "conc_sc")


def _flat_digest(flat):
    """Digest of a FlatTopology's arrays; kept on the object when its arrays
    are read-only (the cached result of flatten, which never changes)."""
    d = getattr(flat, "_digest", None)
    if d is not None:
        return d
    import hashlib
    h = hashlib.blake2b(digest_size=16)
    for name in _FLAT_FIELDS:
        h.update(np.ascontiguousarray(getattr(flat, name)).tobytes())
    d = h.digest()
    if not flat.excl_cols.flags.writeable:
        flat._digest = d
    return d


def particle_arrays(particles):
    """(xyz [n,3], charge, radius, epsilon) from any objects with the
    Particle attributes (this module's or the reference's)."""
    ps = particles if isinstance(particles, list) else list(particles)
    xyz = np.array([[p.x for p in ps], [p.y for p in ps], [p.z for p in ps]], dtype=np.float64).T.copy()
    return (xyz.reshape(-1, 3), np.array([p.charge for p in ps], dtype=np.float64),
            np.array([p.radius for p in ps], dtype=np.float64), np.array([p.epsilon for p in ps], dtype=np.float64))


def particles_from(xyz, template):
    """New Particle list with coordinates xyz and the other fields of template
    (built field by field: the values are floats already)."""
    out = []
    new = Particle.__new__
    for (x, y, z), p in zip(np.asarray(xyz, dtype=np.float64).tolist(), template):
        o = new(Particle)
        o.x, o.y, o.z = x, y, z
        o.charge, o.radius, o.epsilon, o.is_water = float(p.charge), float(p.radius), float(p.epsilon), bool(p.is_water)
        out.append(o)
    return out


class PhysicsEngine:
    """B200 engine with the reference PhysicsEngine's methods.

    precision: "mixed" (FP32 pair terms, FP64 accumulation — the default)
    or "fp64".  seed: MC random stream (the reference is not seedable; here
    every run is reproducible from the seed)."""

    def __init__(self, precision="mixed", seed=None):
        if precision not in ("mixed", "fp64"):
            raise ValueError("precision must be 'mixed' or 'fp64'")
        self.precision = precision
        self._seed = int(np.random.SeedSequence().entropy % (1 << 63)) if seed is None else int(seed)
        self._calls = 0
        self._batches = {}  # device batches of recent calls, reused when only coordinates change

    def _batch(self, xyz, q, r, e, flat, copies=1):
        """A DeviceBatch of `copies` systems with these parameters and
        topology, loaded with xyz: reused across calls on the same system
        (the key hashes every parameter and topology array), so repeated
        calls pay no topology upload or list allocation."""
        import hashlib
        from .device import DeviceBatch
        h = hashlib.blake2b(digest_size=16)
        for a in (q, r, e):
            h.update(np.ascontiguousarray(a, np.float64).tobytes())
        if flat is not None:
            h.update(_flat_digest(flat))
        key = (int(copies), len(q), flat is not None, h.hexdigest())
        b = self._batches.pop(key, None)
        X = np.tile(np.asarray(xyz, np.float64).reshape(-1, 3), (int(copies), 1))
        if b is None:
            b = DeviceBatch([(xyz, q, r, e, flat)] * int(copies), precision=self.precision)
        else:
            b.load_coords(X)
        self._batches[key] = b
        while len(self._batches) > 4:
            self._batches.pop(next(iter(self._batches)))
        return b

    # ---- energies ----------------------------------------------------------------
    def calculate_potential(self, particles, topology=None):
        """Total energy (kcal/mol): Born radii, SASA, dihedral, disulfide and
        pair terms on a freshly built neighbor list (physics_engine.cpp:2242)."""
        return float(self.energy_terms(particles, topology)[4])

    def energy_terms(self, particles, topology=None):
        """[sasa, dihedral, disulfide, pair sum, total] (kcal/mol)."""
        if len(particles) == 0:
            return np.zeros(5)
        from .device import DeviceBatch
        xyz, q, r, e = particle_arrays(particles)
        flat = _topology.flatten(topology) if topology is not None else None
        if flat is not None and flat.n != len(particles):
            raise ValueError(f"topology has {flat.n} atoms, particle list {len(particles)}")
        if not np.all(np.isfinite(xyz)):
            raise ValueError("non-finite coordinates")
        b = self._batch(xyz, q, r, e, flat)
        return b.energy_terms()[0].cpu().numpy()

    def lowest_energy_structure(self, ensemble):
        """Member with the lowest calculate_potential (no topology, as the
        reference evaluates it, physics_engine.cpp:3672-3676)."""
        if len(ensemble) == 0:
            raise ValueError("ensemble empty")
        from .device import DeviceBatch
        systems = [(*particle_arrays(m), None) for m in ensemble]
        b = DeviceBatch(systems, precision=self.precision)
        tot = b.energy_terms()[:, 4].cpu().numpy()
        return list(ensemble[int(np.argmin(tot))])

    def num_threads(self):
        """Streaming multiprocessors available (the reference reports its
        OpenMP thread count)."""
        import torch
        if not torch.cuda.is_available():
            return 1
        return int(torch.cuda.get_device_properties(0).multi_processor_count)

    @staticmethod
    def device_name():
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("no CUDA device")
        return torch.cuda.get_device_name(0)

    # ---- Monte Carlo (engine methods defined in mc.py) ------------------------------
    def _next_seed(self):
        self._calls += 1
        return (self._seed * 0x9E3779B97F4A7C15 + self._calls) & ((1 << 64) - 1)

    def generate_ensemble(self, initial_state, topology, n_candidates, steps_per_cand, temperature=0.6,
                          max_angle=0.12):
        from .mc import generate_ensemble
        return generate_ensemble(self, initial_state, topology, n_candidates, steps_per_cand, temperature,
                                 max_angle)

    def run_landscape_trajectory(self, initial_state, topology, n_snapshots, steps_per_snapshot,
                                 temperature=0.6, max_angle=0.12):
        from .mc import run_landscape
        snaps, energies, _ = run_landscape(self, initial_state, topology, n_snapshots, steps_per_snapshot,
                                           temperature, max_angle)
        return snaps, energies

    def run_landscape_segment(self, initial_state, topology, n_snapshots, steps_per_snapshot,
                              temperature=0.6, max_angle=0.12):
        from .mc import run_landscape
        return run_landscape(self, initial_state, topology, n_snapshots, steps_per_snapshot, temperature,
                             max_angle)

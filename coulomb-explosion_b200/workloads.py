"""Workload definitions: the molecules and geometry distributions the engine is
measured and checked on, and a seeded numpy geometry sampler for host-side
inputs.

Molecules follow the reference's conventions: masses in amu converted to
electron masses at the boundary (include/coulomb/molecule.hpp:23-25,
units.hpp:11-14), integer charges, Coulomb constant 1 (atomic units).

  ch4          C + 4 H, all q = +1 (examples/generate_dataset.cpp:56-66);
               positions uniform in a 3.3-bohr ball, pairs >= 0.5 bohr
  h2o_stiff    O (q +3) + 2 H (q +1) in a 2.0-bohr ball, pairs >= 0.3 bohr
  c2h6_like    2 C (q +2) + 8 H (q +1), 4.0-bohr ball, pairs >= 0.5 bohr
  mixed        N ~ U{2..10}, species ~ U{H, C, N, O, S}, q ~ U{+1, +2, +3},
               radius 2.0 N^(1/3) bohr, pairs >= 0.5 bohr

Every atom is placed independently and uniformly in the ball; a geometry with
any pair closer than the minimum is redrawn whole. (The reference's
UniformSphereSampler instead redraws atom by atom, src/sampler.cpp:28-57; the
host C++ mirror of that sampler lives in host/src/host.cpp.)
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

AMU_TO_ME = 1822.888486209
SPECIES_AMU = {"H": 1.008, "C": 12.011, "N": 14.007, "O": 15.999, "S": 32.06}
MIXED_SPECIES = ("H", "C", "N", "O", "S")


@dataclass(frozen=True)
class Molecule:
    symbols: tuple
    charges: tuple
    radius: float
    min_sep: float

    @property
    def n(self) -> int:
        return len(self.symbols)

    @property
    def masses_me(self) -> np.ndarray:
        return np.array([SPECIES_AMU[s] for s in self.symbols]) * AMU_TO_ME

    @property
    def charge_array(self) -> np.ndarray:
        return np.array(self.charges, dtype=np.float64)


CH4 = Molecule(("C", "H", "H", "H", "H"), (1.0, 1.0, 1.0, 1.0, 1.0), 3.3, 0.5)
H2O_STIFF = Molecule(("O", "H", "H"), (3.0, 1.0, 1.0), 2.0, 0.3)
C2H6_LIKE = Molecule(("C", "C") + ("H",) * 8, (2.0, 2.0) + (1.0,) * 8, 4.0, 0.5)

# Tolerance points: (rtol, atol, pe_stop_fraction).
PRODUCTION = (1e-4, 1e-7, 1e-5)  # docs/decisions/0004-precision-policy.md:42-46
TIGHT = (1e-6, 1e-7, 1e-7)       # the <= 1e-5 relative-momentum-error point
REFERENCE_DEFAULT = (1e-8, 1e-16, 1e-9)  # driver.hpp:147, integrator.hpp:231-232


def _min_pair_ok(x: np.ndarray, dmin: float) -> np.ndarray:
    n = x.shape[1]
    if n < 2:
        return np.ones(x.shape[0], bool)
    d = x[:, :, None, :] - x[:, None, :, :]
    d2 = np.einsum("sijc,sijc->sij", d, d)
    iu = np.triu_indices(n, 1)
    return d2[:, iu[0], iu[1]].min(axis=1) >= dmin * dmin


def sample_ball(rng: np.random.Generator, S: int, n: int, radius: float, min_sep: float) -> np.ndarray:
    """S geometries of n atoms, each atom uniform in the ball (cube rejection),
    whole-geometry rejection on the minimum pair distance. float64 [S, n, 3]."""
    out = np.empty((S, n, 3))
    todo = np.arange(S)
    while todo.size:
        m = todo.size
        pts = np.empty((m, n, 3))
        need = np.ones((m, n), bool)
        while need.any():
            k = int(need.sum())
            cand = rng.uniform(-radius, radius, (k, 3))
            pts[need] = cand
            need[need] = (cand * cand).sum(1) > radius * radius
        ok = _min_pair_ok(pts, min_sep)
        out[todo[ok]] = pts[ok]
        todo = todo[~ok]
    return out


def sample_molecule(mol: Molecule, S: int, seed: int) -> np.ndarray:
    return sample_ball(np.random.default_rng(seed), S, mol.n, mol.radius, mol.min_sep)


def sample_mixed(S: int, seed: int, n_min: int = 2, n_max: int = 10):
    """Mixed 2..10-atom molecules. Returns (n_per [S] uint8, masses_me [S,10],
    charges [S,10], pos [S,10,3]); padding atoms have mass 1, charge 0, x = 0."""
    rng = np.random.default_rng(seed)
    n_per = rng.integers(n_min, n_max + 1, S).astype(np.uint8)
    sp = rng.integers(0, len(MIXED_SPECIES), (S, 10))
    amu = np.array([SPECIES_AMU[s] for s in MIXED_SPECIES])[sp]
    q = rng.integers(1, 4, (S, 10)).astype(np.float64)
    pos = np.zeros((S, 10, 3))
    for n in range(n_min, n_max + 1):
        idx = np.nonzero(n_per == n)[0]
        if idx.size:
            pos[idx, :n] = sample_ball(rng, idx.size, n, 2.0 * n ** (1.0 / 3.0), 0.5)
    mask = np.arange(10)[None, :] < n_per[:, None]
    masses = np.where(mask, amu * AMU_TO_ME, 1.0)
    charges = np.where(mask, q, 0.0)
    return n_per, masses, charges, pos

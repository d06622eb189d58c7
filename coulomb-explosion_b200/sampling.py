"""Counter-based (Philox4x32-10) geometry sampling through libce_gpu.so.

The host twins (ce_sample_*_host) need no GPU and produce the same bits as the
device kernels (ce_sample_*_device); see include/ce_sampler.h.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import CeBallSampler, CeMixedSampler, load_library
from .workloads import MIXED_SPECIES, SPECIES_AMU, Molecule


def ball_config(mol: Molecule, seed: int, max_attempts: int = 0) -> CeBallSampler:
    return CeBallSampler(int(seed), float(mol.radius), float(mol.min_sep), int(max_attempts))


def mixed_config(seed: int, n_min: int = 2, n_max: int = 10, radius_coeff: float = 2.0, min_sep: float = 0.5,
                 q_min: int = 1, q_max: int = 3, species=MIXED_SPECIES, max_attempts: int = 0) -> CeMixedSampler:
    amu = (C.c_double * 8)(*([SPECIES_AMU[s] for s in species] + [0.0] * (8 - len(species))))
    return CeMixedSampler(int(seed), n_min, n_max, float(radius_coeff), float(min_sep), int(max_attempts), q_min,
                          q_max, len(species), amu)


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def sample_ball_host(mol: Molecule, S: int, seed: int, first_sim: int = 0):
    """(pos float32 [S, n, 3], pos float64 [S, n, 3], flags uint8 [S])."""
    lib = load_library()
    pos = np.zeros((S, mol.n, 3), np.float32)
    pos64 = np.zeros((S, mol.n, 3), np.float64)
    flags = np.zeros(S, np.uint8)
    cfg = ball_config(mol, seed)
    rc = lib.ce_sample_ball_host(mol.n, int(first_sim), int(S), C.byref(cfg), _p(pos), _p(pos64), _p(flags))
    if rc != 0:
        raise RuntimeError(f"ce_sample_ball_host failed: {rc}")
    return pos, pos64, flags


def sample_mixed_host(S: int, seed: int, first_sim: int = 0, **kw):
    """(n_atoms [S], mass_me [S,10], charge [S,10], pos f32 [S,10,3], pos f64, flags)."""
    lib = load_library()
    n = np.zeros(S, np.uint8)
    m = np.zeros((S, 10))
    q = np.zeros((S, 10))
    pos = np.zeros((S, 10, 3), np.float32)
    pos64 = np.zeros((S, 10, 3))
    flags = np.zeros(S, np.uint8)
    cfg = mixed_config(seed, **kw)
    rc = lib.ce_sample_mixed_host(int(first_sim), int(S), C.byref(cfg), _p(n), _p(m), _p(q), _p(pos), _p(pos64),
                                  _p(flags))
    if rc != 0:
        raise RuntimeError(f"ce_sample_mixed_host failed: {rc}")
    return n, m, q, pos, pos64, flags


def philox(ctr, key) -> tuple:
    lib = load_library()
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib.ce_philox4x32_10(c, k, o)
    return tuple(int(v) for v in o)

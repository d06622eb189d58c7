"""Pin the restated FP64 scipy oracle (oracle/scipy_oracle.py) to the reference's own (CPU only).

The reference's Python oracle (python/reference/coulomb.py:80-109) is the ground
truth its accuracy studies compare against. Its outputs were recorded by
importing that module (tests/golden/make_golden.py) on the reference's three
oracle cases and on 48 sims each of the benchmark workloads. The restatement
calls the same scipy solve_ivp with its own right-hand side, so it differs only
by floating-point reassociation: 1e-12 relative is the bar, far below every
error it is used to measure (>= 1e-8).
"""
from __future__ import annotations

import json
import sys

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

sys.path.insert(0, str(ROOT / "oracle"))
import scipy_oracle as so  # noqa: E402

TOL = 1e-12


def test_reference_cases():
    doc = json.loads((GOLDEN / "reference_cases.json").read_text())
    assert doc["rk_rtol"] == so.RTOL and doc["rk_atol"] == so.ATOL
    for c in doc["cases"]:
        p = so.asymptotic_momenta(np.array(c["positions_init"]), np.array(c["masses"]), np.array(c["charges"]))
        ref = np.array(c["momenta_final"])
        assert np.abs(p - ref).max() <= TOL * np.abs(ref).max(), c["name"]


@pytest.mark.parametrize("tag", ["ch4", "h2o", "c2h6"])
def test_fixed_molecules(tag):
    d = np.load(GOLDEN / "scipy_ref.npz")
    pos = d[f"{tag}_pos"][:12]
    p = so.run_many(pos, d[f"{tag}_masses"], d[f"{tag}_charges"], processes=1)
    ref = d[f"{tag}_p"][:12]
    rel = np.linalg.norm((p - ref).reshape(len(p), -1), axis=1) / np.linalg.norm(ref.reshape(len(p), -1), axis=1)
    assert rel.max() <= TOL, rel.max()


def test_mixed_population_through_the_pool():
    """The spawn pool path: 48 mixed sims over 4 worker processes."""
    d = np.load(GOLDEN / "scipy_ref.npz")
    p = so.run_many(d["mixed_pos"], d["mixed_masses"], d["mixed_charges"], n_per=d["mixed_n"], processes=4)
    ref = d["mixed_p"]
    rel = np.linalg.norm((p - ref).reshape(len(p), -1), axis=1) / np.linalg.norm(ref.reshape(len(p), -1), axis=1)
    assert rel.max() <= TOL, rel.max()
    assert not p[np.arange(10)[None, :] >= d["mixed_n"][:, None]].any()  # rows zero past n

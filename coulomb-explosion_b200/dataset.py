"""Reader for the dataset format shared with the reference (fixed-width records
plus a .meta.json sidecar; examples/generate_dataset.cpp:10-19 and
examples/to_parquet.py:34-42 of the reference), as written by
bin/ce_generate_dataset and coulomb::DatasetWriter."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

AMU_TO_ME = 1822.888486209


def record_dtype(n_atoms: int) -> np.dtype:
    return np.dtype([("init_pos", "<f4", (n_atoms * 3,)), ("final_p", "<f4", (n_atoms * 3,)), ("steps", "<u4"),
                     ("converged", "u1")])


def read_dataset(path: str | Path):
    """(meta dict, records memmap) for a dataset file."""
    path = Path(path)
    meta = json.loads(Path(str(path) + ".meta.json").read_text())
    rec = np.memmap(path, dtype=record_dtype(int(meta["n_atoms"])), mode="r")
    return meta, rec


def sanity(meta: dict, rec, n: int | None = None) -> dict:
    """The physics checks of the reference's demo/sanity_check.py:58-139 on the
    first n records: KER vs initial Coulomb PE, total momentum, and the
    per-species energy partition against the equal-|p| prediction."""
    k = int(meta["n_atoms"])
    n = len(rec) if n is None else min(n, len(rec))
    masses_amu = np.asarray(meta["masses_amu"], float)
    masses = masses_amu * AMU_TO_ME
    q = np.asarray(meta["charges"], float)
    x = rec["init_pos"][:n].reshape(-1, k, 3).astype(float)
    p = rec["final_p"][:n].reshape(-1, k, 3).astype(float)
    ke_atom = (p ** 2).sum(axis=2) / (2.0 * masses)
    ker = ke_atom.sum(axis=1)
    iu = np.triu_indices(k, 1)
    r = np.linalg.norm(x[:, :, None, :] - x[:, None, :, :], axis=3)
    pe = (np.outer(q, q)[iu] / r[:, iu[0], iu[1]]).sum(axis=1)
    tot = np.linalg.norm(p.sum(axis=1), axis=1)
    typ = np.linalg.norm(p, axis=2).mean()
    groups: dict[str, list[int]] = {}
    for i, s in enumerate(meta["symbols"]):
        groups.setdefault(s, []).append(i)
    w = {s: len(idx) / masses_amu[idx[0]] for s, idx in groups.items()}
    wsum = sum(w.values())
    partition = {s: (float(ke_atom[:, idx].sum() / ke_atom.sum()), w[s] / wsum) for s, idx in groups.items()}
    return {"ker_vs_pe_max_rel": float(np.max(np.abs(ker - pe) / pe)),
            "momentum_ratio_mean": float((tot / typ).mean()),
            "partition": partition,
            "converged_frac": float(rec["converged"][:n].mean())}

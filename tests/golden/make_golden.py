#!/usr/bin/env python3
"""Generate the golden fixtures under tests/golden/ (run in the build container,
where the reference checkout and the reference engine built from it exist).

  reference_cases.json  the reference's three oracle cases (two_protons,
                        triangle_H3, pentatomic_BrClFCH): inputs read from the
                        reference's tests/reference/reference_cases.json, every
                        output recomputed here by importing the reference's own
                        Python oracle (python/reference/coulomb.py:23-109, scipy
                        solve_ivp RK45 to t = 1e10) and checked against the
                        committed reference values.
  ch4_ref.npz           256 seeded CH4 geometries and the reference scalar
                        engine's f32/f64 outputs (oracle/_ref, built from
                        src/*.cpp) at the production and tight tolerance points,
                        plus the scipy oracle's momenta for the first 24.
  mixed_ref.npz         128 mixed 2..10-atom molecules, reference f32/f64
                        engine outputs at the tight point.
  h2o_ref.npz           96 stiff H2O geometries, reference f32/f64 outputs.
  sampler_ref.npz       reference UniformSphereSampler draws (mt19937_64) for
                        the host C++ sampler mirror.
  scipy_ref.npz         the reference's scipy oracle (simulate_explosion) on 48
                        sims each of CH4, stiff H2O, the C2H6-like 10-atom
                        molecule and the mixed 2..10-atom population (Philox
                        geometries of the benchmark workloads), to pin the
                        restated scipy oracle (oracle/scipy_oracle.py).

Usage: python tests/golden/make_golden.py --reference <reference checkout> [--only scipy]
(or COULOMB_REFERENCE_DIR=<checkout>); needs oracle/_ref (`make -C oracle REF=<checkout>`).
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
REF: Path  # the reference checkout, from --reference or COULOMB_REFERENCE_DIR
sys.path.insert(0, str(ROOT / "tests"))
import oracle_lib as ol  # noqa: E402
from pkg_loader import load_submodule  # noqa: E402

wl = load_submodule("workloads")
sp = load_submodule("sampling")


def load_reference_oracle():
    spec = importlib.util.spec_from_file_location("ref_coulomb", REF / "python" / "reference" / "coulomb.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def potential_energy(x, q):
    u = 0.0
    for i in range(len(q)):
        for j in range(i + 1, len(q)):
            u += q[i] * q[j] / np.linalg.norm(x[i] - x[j])
    return float(u)


def make_reference_cases(co):
    src = json.loads((REF / "tests" / "reference" / "reference_cases.json").read_text())
    cases = []
    for c in src["cases"]:
        m = np.array(c["masses"], float)
        q = np.array(c["charges"], float)
        x0 = np.array(c["positions_init"], float)
        f0 = co.forces(x0, q)
        xf, vf = co.simulate_explosion(x0, np.zeros_like(x0), m, q)
        pf = m[:, None] * vf
        for key, mine in (("forces_init", f0), ("momenta_final", pf), ("positions_final", xf)):
            theirs = np.array(c[key])
            assert np.allclose(mine, theirs, rtol=1e-12, atol=1e-12), (c["name"], key)
        cases.append(dict(
            name=c["name"], symbols=c["symbols"], masses=m.tolist(), charges=q.tolist(),
            positions_init=x0.tolist(), forces_init=f0.tolist(),
            potential_energy_init=potential_energy(x0, q),
            kinetic_energy_final=float(0.5 * np.sum(np.sum(pf ** 2, 1) / m)),
            momenta_final=pf.tolist(),
        ))
    doc = dict(
        description=("Reference oracle cases: inputs from the reference's tests/reference/"
                     "reference_cases.json, outputs recomputed with its python/reference/coulomb.py "
                     "(scipy solve_ivp RK45, rtol 1e-8, atol 1e-16, to t = 1e10). Atomic units, "
                     "masses in electron masses. Generated by tests/golden/make_golden.py."),
        coulomb_constant=1.0, rk_rtol=co.RKRTOL, rk_atol=co.RKATOL, cases=cases,
    )
    (HERE / "reference_cases.json").write_text(json.dumps(doc, indent=1) + "\n")


def ref_outputs(pos, mass, q, points):
    out = {}
    for tag, (rtol, atol, pes) in points.items():
        for bits in (32, 64):
            r = ol.ref_run_batch(pos, mass, q, bits=bits, rtol=rtol, atol=atol, pe_stop=pes)
            out[f"p_{tag}_f{bits}"] = r["momenta"]
            out[f"steps_{tag}_f{bits}"] = r["steps"]
            out[f"status_{tag}_f{bits}"] = r["status"]
    return out


def make_scipy_ref(co):
    """48 sims per workload through the reference's simulate_explosion."""
    out = {}
    count = 48

    def run(pos, m, q, n_per=None):
        p = np.zeros(pos.shape)
        for s in range(pos.shape[0]):
            n = pos.shape[1] if n_per is None else int(n_per[s])
            ms = m[s] if m.ndim == 2 else m
            qs = q[s] if q.ndim == 2 else q
            _, vf = co.simulate_explosion(pos[s, :n], np.zeros((n, 3)), ms[:n], qs[:n])
            p[s, :n] = ms[:n, None] * vf
        return p

    for tag, mol in (("ch4", wl.CH4), ("h2o", wl.H2O_STIFF), ("c2h6", wl.C2H6_LIKE)):
        pos32, _, flags = sp.sample_ball_host(mol, count, seed=20261203)
        assert not flags.any()
        pos = pos32.astype(np.float64)
        out[f"{tag}_pos"], out[f"{tag}_masses"], out[f"{tag}_charges"] = pos, mol.masses_me, mol.charge_array
        out[f"{tag}_p"] = run(pos, mol.masses_me, mol.charge_array)
    n_per, m, q, pos32, _, flags = sp.sample_mixed_host(count, 20261203)
    assert not flags.any()
    pos = pos32.astype(np.float64)
    out.update(mixed_n=n_per, mixed_masses=m, mixed_charges=q, mixed_pos=pos)
    out["mixed_p"] = run(pos, m, q, n_per)
    np.savez_compressed(HERE / "scipy_ref.npz", **out)


def main():
    global REF
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("COULOMB_REFERENCE_DIR"),
                    help="the reference checkout (or COULOMB_REFERENCE_DIR)")
    ap.add_argument("--only", choices=["scipy"], default=None, help="regenerate one fixture only")
    args = ap.parse_args()
    if not args.reference:
        ap.error("give the reference checkout with --reference or COULOMB_REFERENCE_DIR")
    REF = Path(args.reference)
    co = load_reference_oracle()
    if args.only == "scipy":
        make_scipy_ref(co)
        print("scipy_ref.npz written to", HERE)
        return
    make_reference_cases(co)
    make_scipy_ref(co)
    points = {"prod": wl.PRODUCTION, "tight": wl.TIGHT}

    # CH4, 256 sims.
    mol = wl.CH4
    pos = wl.sample_molecule(mol, 256, seed=20261203)
    pos32 = pos.astype(np.float32).astype(np.float64)  # the engines narrow to float on load
    data = dict(pos=pos32, masses=mol.masses_me, charges=mol.charge_array)
    data.update(ref_outputs(pos32, mol.masses_me, mol.charge_array, points))
    n_sci = 24
    p_sci = np.zeros((n_sci, mol.n, 3))
    for s in range(n_sci):
        _, vf = co.simulate_explosion(pos32[s], np.zeros((mol.n, 3)), mol.masses_me, mol.charge_array)
        p_sci[s] = mol.masses_me[:, None] * vf
    data["p_scipy"] = p_sci
    np.savez_compressed(HERE / "ch4_ref.npz", **data)

    # Mixed 2..10, 128 sims: the reference engine takes one Molecule per run.
    n_per, mass, q, pos = wl.sample_mixed(128, seed=777)
    pos32 = pos.astype(np.float32).astype(np.float64)
    mixed = dict(n_per=n_per, masses=mass, charges=q, pos=pos32)
    for bits in (32, 64):
        p = np.zeros((128, 10, 3))
        st = np.zeros(128, np.uint32)
        for s in range(128):
            n = int(n_per[s])
            r = ol.ref_run_batch(pos32[s:s + 1, :n], mass[s, :n], q[s, :n], bits=bits, rtol=wl.TIGHT[0],
                                 atol=wl.TIGHT[1], pe_stop=wl.TIGHT[2], threads=1)
            p[s, :n] = r["momenta"][0]
            st[s] = r["steps"][0]
        mixed[f"p_tight_f{bits}"] = p
        mixed[f"steps_tight_f{bits}"] = st
    np.savez_compressed(HERE / "mixed_ref.npz", **mixed)

    # Stiff H2O, 96 sims.
    mol = wl.H2O_STIFF
    pos = wl.sample_molecule(mol, 96, seed=4242)
    pos32 = pos.astype(np.float32).astype(np.float64)
    data = dict(pos=pos32, masses=mol.masses_me, charges=mol.charge_array)
    data.update(ref_outputs(pos32, mol.masses_me, mol.charge_array, points))
    np.savez_compressed(HERE / "h2o_ref.npz", **data)

    # Reference sampler draws (mt19937_64, sequential per-atom redraw).
    samp = {}
    for seed, n, r, d in ((49188291, 5, 4.0, 0.25), (7, 10, 4.0, 0.5), (123, 3, 2.0, 0.3)):
        buf = np.zeros((16, n, 3))
        rc = ol.ref(64).ref_sample(r, d, 10000, seed, n, 16, ol._p(buf))
        assert rc == 0
        samp[f"pos_{seed}_{n}"] = buf
    np.savez_compressed(HERE / "sampler_ref.npz", **samp)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()

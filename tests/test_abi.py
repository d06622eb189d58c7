"""The C ABI library loads and exports every entry point include/*.h declares
(CPU only: no compute call is made)."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import pytest

from conftest import ROOT

HEADERS = sorted((ROOT / "include").glob("*.h"))
DECL = re.compile(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(ce_\w+)\s*\(", re.M)


def declared(header: Path) -> set[str]:
    text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
    text = "\n".join(line for line in text.splitlines() if not line.lstrip().startswith("#"))
    return set(DECL.findall(text))


def test_headers_declare_entry_points():
    names = set().union(*(declared(h) for h in HEADERS))
    assert {"ce_create", "ce_destroy", "ce_set_molecule", "ce_run", "ce_run_device", "ce_last_error"} <= names


def test_library_exports_every_declared_symbol(ce):
    lib = ce.load_library()
    missing = []
    for h in HEADERS:
        for name in sorted(declared(h)):
            if not hasattr(lib, name):
                missing.append(f"{h.name}:{name}")
    assert not missing, missing


def test_python_binding_covers_every_declared_symbol(ce):
    names = set().union(*(declared(h) for h in HEADERS))
    assert names <= set(ce._SIGNATURES), sorted(names - set(ce._SIGNATURES))


def test_default_config_is_reference_default(ce):
    lib = ce.load_library()
    cfg = ce.CeRunConfig()
    lib.ce_default_config(C.byref(cfg))
    # include/coulomb/driver.hpp:147-162, include/coulomb/integrator.hpp:231-232
    assert (cfg.rtol, cfg.atol, cfg.pe_stop_fraction, cfg.max_dt, cfg.max_steps, cfg.redistribute_energy) == (
        1e-8, 1e-16, 1e-9, 1e12, 1_000_000, 1)
    assert ce.RunConfig().to_c().rtol == cfg.rtol


def test_null_engine_is_rejected_without_a_gpu(ce):
    lib = ce.load_library()
    m = (C.c_double * 2)(1.0, 1.0)
    assert lib.ce_set_molecule(None, 2, m, m, 1.0) == ce.CE_ERR_INVALID
    assert lib.ce_run(None, 1, None, None, None) == ce.CE_ERR_INVALID
    assert lib.ce_last_error(None) == b"null engine"
    assert lib.ce_create(None, 0) == ce.CE_ERR_INVALID
    assert lib.ce_version().startswith(b"ce_gpu")


def test_create_reports_no_device_or_succeeds(ce):
    lib = ce.load_library()
    h = C.c_void_p()
    rc = lib.ce_create(C.byref(h), 0)
    assert rc in (ce.CE_OK, ce.CE_ERR_NO_DEVICE)
    if rc == ce.CE_OK:
        lib.ce_destroy(h)


def test_engine_fails_loudly_when_library_missing(ce, tmp_path):
    with pytest.raises(RuntimeError, match="not built"):
        ce.load_library(tmp_path / "libce_gpu.so")

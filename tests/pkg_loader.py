"""Import the in-tree package directory ``coulomb-explosion_b200/`` (its name is
not a Python identifier) as the module ``coulomb_explosion_b200``."""
from __future__ import annotations

import importlib
import importlib.util
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
PKG_DIR = ROOT / "coulomb-explosion_b200"
NAME = "coulomb_explosion_b200"


def load_package():
    if NAME in sys.modules:
        return sys.modules[NAME]
    spec = importlib.util.spec_from_file_location(NAME, PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[NAME] = mod
    spec.loader.exec_module(mod)
    return mod


def load_submodule(name: str):
    load_package()
    return importlib.import_module(f"{NAME}.{name}")

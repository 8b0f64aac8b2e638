"""The C-ABI library loads without a GPU and exports every function that
include/unichem.h declares (no compute call is made)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "unichem.h"


def declared():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_]\w*\s*\**\s*(uc_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_path():
    names = declared()
    for must in ("uc_init", "uc_rates", "uc_omega", "uc_props", "uc_cp_h", "uc_species_update",
                 "uc_temperature_from_h", "uc_sweep", "uc_destroy", "uc_species_update_noalloc"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from unicorn_b200.unichem import LIB_PATH
    if not LIB_PATH.exists():
        from unicorn_b200.build import build
        build()
    lib = ctypes.CDLL(str(LIB_PATH))
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_mirror_fails_loudly_without_library(tmp_path, monkeypatch):
    from unicorn_b200 import unichem
    monkeypatch.setattr(unichem, "_lib", None)
    with pytest.raises(unichem.UniChemError):
        unichem.load_library(tmp_path / "missing.so")

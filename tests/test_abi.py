"""The C-ABI library loads and exports every symbol the header declares (CPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "oxiblas_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(oxi_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("oxi_create", "oxi_destroy", "oxi_dgetrf", "oxi_dgetrs", "oxi_dgemm_update"):
        assert s in syms


def test_library_exports_every_declared_symbol(pkg):
    L = pkg.load()
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing


def test_status_strings_without_gpu(pkg):
    L = pkg.load()
    assert L.oxi_status_string(0) == b"ok"
    assert b"singular" in L.oxi_status_string(2)


def test_binding_declares_only_exported_symbols(pkg):
    L = pkg.load()
    for s in pkg.exported_symbols():
        assert hasattr(L, s), s

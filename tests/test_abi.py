"""The C-ABI library loads and exports every entry point declared in
include/disorder.h (no GPU needed: nothing is called)."""

import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    txt = open(os.path.join(ROOT, "include", "disorder.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(disorder_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_entry_points():
    names = declared()
    for n in ("disorder_encode", "disorder_decode", "disorder_encodedecode", "disorder_sinc_rigid_transform",
              "disorder_sinc_rigid_transform_gradient", "disorder_cg_solve", "disorder_lm_step",
              "disorder_compute_energy", "disorder_plan_create"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from disorder_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libdisorder.so not built")
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding declares exactly the header's entry points
    assert sorted(_lib.exported_symbols()) == declared()

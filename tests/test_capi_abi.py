"""The C-ABI library loads and exports every symbol that include/repulsor_b200.h declares."""
import os
import re
import subprocess

import numpy as np
import pytest

import repulsor_b200 as rpb
from repulsor_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "repulsor_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(rpb_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "rpb_mesh_create" in names and "rpb_tpm0_solve" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", _capi.LIB_PATH], check=True, capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (rpb_[a-z0-9_]+)", out))
    missing = [n for n in declared_symbols() if n not in exported]
    assert not missing, f"declared but not exported: {missing}"


def test_ctypes_signatures_cover_header():
    assert set(_capi.SIGNATURES) == set(declared_symbols())
    lib = _capi.load()
    for name in _capi.SIGNATURES:
        assert hasattr(lib, name)


def test_default_settings_are_reference_defaults():
    s = rpb.default_settings()
    assert s.split_threshold == 1
    assert s.far_field_separation == 0.5
    assert s.near_field_separation == 10.0
    assert s.max_refinement == 30


def test_invalid_arguments_are_rejected_without_device():
    V = np.zeros((3, 3))
    S = np.array([[0, 1, 2]], np.int32)
    with pytest.raises(rpb.RepulsorError):
        rpb.HostTree(V, np.array([[0, 1, 7]], np.int32))          # index out of range
    with pytest.raises(rpb.RepulsorError):
        rpb.HostTree(np.full((3, 3), np.nan), S)                  # non-finite coordinates
    with pytest.raises(rpb.RepulsorError):
        rpb.HostTree(V, S, split_threshold=2)                     # unsupported setting

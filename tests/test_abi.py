"""The C-ABI library loads and exports every symbol the header declares (no compute)."""

from __future__ import annotations

import ctypes
import re
import subprocess

import pytest

from pyticc_b200 import _build
from pyticc_b200 import _native as nat


def _declared_symbols() -> set[str]:
    text = nat.HEADER_PATH.read_text()
    return set(re.findall(r"^\s*(?:int|long long)\s+(ticc_\w+)\s*\(", text, flags=re.MULTILINE))


@pytest.fixture(scope="module")
def library():
    _build.build()
    return nat.load_library()


def test_header_declares_the_bound_entry_points():
    assert _declared_symbols() == set(nat.SIGNATURES)


def test_library_exports_every_declared_symbol(library):
    for name in _declared_symbols():
        assert isinstance(getattr(library, name), ctypes._CFuncPtr), name
    exported = subprocess.run(["nm", "-D", "--defined-only", str(nat.LIB_PATH)], capture_output=True, text=True, check=True).stdout
    for name in _declared_symbols():
        assert re.search(rf"\bT {name}\b", exported), name


def test_host_side_validation_needs_no_device(library):
    assert library.ticc_version() >= 10000
    out = ctypes.c_size_t(0)
    assert library.ticc_ldmd_workspace_size(0, 1, 1, 0, 0, ctypes.byref(out)) == nat.ERR_INVALID_ARGUMENT
    assert "n_channel=0" in nat.last_error()
    assert library.ticc_ldmd_workspace_size(16, 2, 3, 0, 0, ctypes.byref(out)) == nat.OK
    assert out.value > 0
    assert library.ticc_match_workspace_size(4, 1, 0, 9, ctypes.byref(out)) == nat.ERR_INVALID_ARGUMENT


def test_library_is_built_for_sm100a_only():
    assert any("compute_100a,code=sm_100a" in flag for flag in _build.NVCC_FLAGS)

"""CPU tests of the C-ABI boundary: the library builds and loads, and exports
every function include/radik.h declares.  No compute call is made here."""
from __future__ import annotations

import ctypes
import re

from conftest import ROOT, load_package


def _declared_functions():
    text = (ROOT / "include" / "radik.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(radik_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(radik):
    from radik_b200 import _lib
    L = _lib.load()
    declared = _declared_functions()
    assert len(declared) >= 15
    missing = [name for name in declared if not hasattr(L, name)]
    assert not missing, missing
    assert set(declared) == set(_lib.EXPORTS)


def test_status_strings_and_version(radik):
    from radik_b200 import _lib
    L = _lib.load()
    assert L.radik_version().decode().startswith("radik-b200")
    assert L.radik_status_string(0) == b"ok"
    assert L.radik_status_string(3) == b"workspace too small"
    assert L.radik_last_error() is not None


def test_argument_validation_without_device(radik):
    """Argument checks return before any device call."""
    from radik_b200 import _lib
    L = _lib.load()
    ws = ctypes.c_void_p()
    assert L.radik_ws_create(10, 1, 3, ctypes.byref(ws)) == 1
    assert b"4 or 8" in L.radik_last_error()
    assert L.radik_ws_create(-1, 1, 4, ctypes.byref(ws)) == 1
    assert L.radik_topk_radix_select(None, None, 4, None, None, None, None, 1, 1, 0, None) == 1


def test_package_mirrors_reference_exports():
    pkg = load_package()
    # src/RadiK.jl:19-22 exports topk_radix_select!, topk, topk!, RadiKWorkspace
    for name in ("topk_radix_select_", "topk", "topk_", "RadiKWorkspace", "RadiKError"):
        assert hasattr(pkg, name)

"""CPU checks of the C-ABI library: it builds, loads and exports every entry point
include/bem3d_b200.h declares (no device calls)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "bem3d_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bem_[a-z0-9_]+)\s*\(", text)))


def test_header_lists_expected_entry_points():
    syms = declared_symbols()
    for s in ("bem_ghmat8", "bem_solve", "bem_internal_points", "bem_reorganize", "bem_dgesv"):
        assert s in syms


def test_library_exports_all_declared_symbols():
    from bem3d_elastostatic_b200 import _lib

    L = _lib.load()
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing
    assert set(_lib.EXPORTS) == set(declared_symbols())


def test_library_is_sm100a():
    from bem3d_elastostatic_b200 import build

    path = build.build()
    assert os.path.getsize(path) > 0
    # the build pins sm_100a only
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)

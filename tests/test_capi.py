"""The C-ABI library loads and exports every entry point that
include/amigo_b200.h declares (CPU only; no compute calls)."""
import ctypes
import os
import re

from amigo_b200 import _lib

HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                   "include", "amigo_b200.h")


def declared():
    src = open(HDR).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\bint\s+(ab_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared()
    assert "ab_ldl_create" in names and "ab_ipm_max_step" in names
    assert len(names) >= 20


def test_library_exports_all_declared_symbols():
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared() if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared()) <= set(_lib.exported_symbols()) | {"ab_ldl_analyze"}
    _lib.lib()

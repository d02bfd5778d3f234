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


def test_autotune_arguments_without_a_gpu():
    """ab_ldl_autotune refuses an analysis-only handle (no device plan) and
    bad arguments before any CUDA call; ab_ldl_apply_tuning checks every
    field's range."""
    import numpy as np
    from amigo_b200 import linalg
    L = _lib.lib()
    n = 4
    rowp = np.array([0, 2, 4, 6, 8], np.int32)
    cols = np.array([0, 1, 0, 1, 2, 3, 2, 3], np.int32)
    h = ctypes.c_void_p()
    ip = ctypes.POINTER(ctypes.c_int)
    assert L.ab_ldl_analyze(n, rowp.ctypes.data_as(ip), cols.ctypes.data_as(ip), 1,
                            ctypes.byref(h)) == 0
    try:
        t = linalg.LdlTuning()
        assert L.ab_ldl_autotune(None, None, 1, None, ctypes.byref(t)) == -1
        assert L.ab_ldl_autotune(h, None, 0, None, ctypes.byref(t)) == -1
        assert L.ab_ldl_autotune(h, None, 1, None, ctypes.byref(t)) == -4
        good = linalg.LdlTuning(panel_mode=0, cl_min_rows=768, panel_cache_bytes=0,
                                cluster_entries=1 << 14, wide_entries=1 << 22,
                                solve_queue=1)
        assert L.ab_ldl_apply_tuning(h, ctypes.byref(good)) == 0
        assert L.ab_ldl_apply_tuning(h, None) == -1
        for field, bad in (("panel_mode", 4), ("cl_min_rows", 0),
                           ("panel_cache_bytes", 300 * 1024), ("cluster_entries", 0),
                           ("wide_entries", 0), ("solve_queue", 4)):
            b = linalg.LdlTuning.from_buffer_copy(good)
            setattr(b, field, bad)
            assert L.ab_ldl_apply_tuning(h, ctypes.byref(b)) == -1, field
    finally:
        L.ab_ldl_destroy(h)

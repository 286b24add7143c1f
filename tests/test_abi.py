"""The C-ABI library loads and exports every symbol include/*.h declares
(no compute calls: these run without a GPU)."""
import ctypes
import glob
import os
import re

from wavetrisk_hydrostatic_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(wt_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("wt_create", "wt_destroy", "wt_trend", "wt_rk4_step", "wt_grid_build"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_native.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_create_without_device_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        return
    lib = _native.lib()
    h = ctypes.c_void_p()
    desc = _native.wt_grid_desc()
    desc.levels = None
    rc = lib.wt_create(ctypes.byref(desc), ctypes.byref(h))
    assert rc == _native.WT_ERR_ARG


def test_tune_rejects_bad_arguments_without_a_device():
    """wt_tune checks its arguments before touching a handle or the device."""
    lib = _native.lib()
    assert lib.wt_tune(None, 1, -1) == _native.WT_ERR_ARG      # WT_TUNE_WAVELET_LAYERS out of range
    assert lib.wt_tune(None, 1, 65) == _native.WT_ERR_ARG
    assert lib.wt_tune(None, 2, 1) == _native.WT_ERR_ARG       # WT_TUNE_SKIP_INACTIVE needs a handle
    assert lib.wt_tune(None, 99, 0) == _native.WT_ERR_ARG      # unknown parameter

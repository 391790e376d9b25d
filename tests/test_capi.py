"""The C-ABI library loads and exports every entry point include/fluxos_gpu.h
declares (no compute calls: runs without a GPU)."""
import ctypes
import os
import re

import fluxos_cpp_b200 as fx

HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                   "fluxos_gpu.h")


def declared():
    text = open(HDR).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.findall(r"^\s*(?:[A-Za-z_][\w\s\*]*?)\b(fx_\w+)\s*\(", text, flags=re.M)


def test_every_declared_symbol_is_exported():
    names = declared()
    assert len(names) >= 20
    lib = ctypes.CDLL(fx.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(fx.EXPORTED)


def test_errors_without_a_context_are_reported():
    L = fx.lib()
    g, p = fx.FxGrid(1, 1, 2, 1, -9999.0, 0.0, 0.0), fx.FxParams()
    h = ctypes.c_void_p()
    assert L.fx_create(ctypes.byref(g), ctypes.byref(p), ctypes.byref(h)) == -1  # FX_ERR_ARG
    assert b"nrows" in L.fx_last_error(None)
    assert not h.value
    assert L.fx_load_modset(b"/nonexistent/modset.json", ctypes.byref(g), ctypes.byref(p), None, None,
                            None, None, None, None, None, None, None, None, None, None) == -3  # FX_ERR_IO

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


def test_footprint_counts_one_record_per_cell_and_step_in_flight():
    """fx_footprint is host arithmetic (no GPU): each step in flight adds one
    slot of per-step state per cell, a 32-byte record and a flag byte in FP32,
    a 48-byte record and a flag byte in FP64, plus the ADE's per-strip
    hand-over and counters and its unit table."""
    n = 1000
    ld = ((n + 2 + 1 + 31) // 32) * 32
    plane = ld * (n + 2)
    strips = (n + 29) // 30
    ade = 8 * strips * (n + 2) * 3 + 8 * strips + 16 * strips  # hand-over, counters, units (one solute)
    for precision, per_cell in (("fp32", 33), ("fp64", 49)):
        a = fx.footprint(n, n, nchem=1, precision=precision, steps_in_flight=8)
        b = fx.footprint(n, n, nchem=1, precision=precision, steps_in_flight=9)
        assert b - a == plane * per_cell + ade, (precision, b - a)
    # FP32 state holds less than FP64 at the same steps in flight
    assert fx.footprint(n, n, precision="fp32", steps_in_flight=31) < fx.footprint(n, n, precision="fp64",
                                                                                 steps_in_flight=31)

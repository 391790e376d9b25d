"""B200-native FLUXOS-OVERLAND time step: Python front-end of libfluxos_gpu.so.

The compute path is the in-tree CUDA library (``fluxos_cpp_b200/lib/
libfluxos_gpu.so``, built by :mod:`fluxos_cpp_b200.build`), reached through
its C ABI (``include/fluxos_gpu.h``). There is no CPU fallback: when the
library is missing or no GPU is present the calls raise.

Grids cross the boundary in the reference's GlobVar layout: numpy arrays of
shape ``(ncols + 2, nrows + 2)`` (C order), i.e. index ``[icol, irow]`` over
column-major ``(NROWS+2) x (NCOLS+2)`` storage with the ghost ring.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libfluxos_gpu.so")
EXE_PATH = os.path.join(HERE, "lib", "fluxos_gpu")
MAX_CHEM = 8
METEO_ROWS = 2000

FIELDS = ("z", "zb", "h", "qx", "qy", "twet", "h0", "fe_1", "fe_2", "fe_3", "fn_1", "fn_2", "fn_3",
          "conc")

# C header symbols, in declaration order (checked by tests/test_capi.py).
EXPORTED = ("fx_create", "fx_destroy", "fx_last_error", "fx_device_bytes", "fx_footprint", "fx_upload",
            "fx_download",
            "fx_upload_flags", "fx_download_flags", "fx_set_forcing", "fx_set_inflow", "fx_set_manning",
            "fx_set_melt_field", "fx_set_option", "fx_prepare", "fx_step", "fx_run_to_print",
            "fx_print_done", "fx_get_status", "fx_stream", "fx_time_steps", "fx_mass", "fx_autotune",
            "fx_batch_create",
            "fx_batch_destroy", "fx_batch_last_error", "fx_batch_add", "fx_batch_remove",
            "fx_batch_size", "fx_batch_step", "fx_batch_stream", "fx_batch_set_option",
            "fx_batch_autotune", "fx_adesolver_noalloc",
            "fx_initiate",
            "fx_load_modset", "fx_open_modset", "fx_write_results", "fx_write_results_async",
            "fx_results_wait", "fx_write_results_host", "fx_run")


class FluxosError(RuntimeError):
    """A libfluxos_gpu call returned an error code."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"libfluxos_gpu error {code}: {msg}")
        self.code = code


class FxGrid(C.Structure):
    _fields_ = [("nrows", C.c_int), ("ncols", C.c_int), ("dxy", C.c_int), ("nchem", C.c_int),
                ("nodata", C.c_double), ("xll", C.c_double), ("yll", C.c_double)]


class FxParams(C.Structure):
    _fields_ = [("hdry", C.c_double), ("ks", C.c_double), ("ntim", C.c_double),
                ("print_step", C.c_double), ("print_next", C.c_double), ("tim", C.c_double),
                ("h_min_print", C.c_double), ("ade", C.c_int), ("volrat_mode", C.c_int),
                ("d_coef", C.c_double * MAX_CHEM), ("steps_in_flight", C.c_int),
                ("precision", C.c_int), ("wintra", C.c_int), ("soil_release_rate", C.c_double)]


class FxStatus(C.Structure):
    _fields_ = [("tim", C.c_double), ("dtfl", C.c_double), ("print_next", C.c_double),
                ("hpall", C.c_double), ("steps", C.c_longlong), ("it", C.c_int),
                ("print_pending", C.c_int), ("finished", C.c_int), ("device_error", C.c_int),
                ("forcing_overrun", C.c_int), ("budget_melt", C.c_double), ("budget_out", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib: Optional[C.CDLL] = None


def lib() -> C.CDLL:
    """Load libfluxos_gpu.so (building it first if it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build as _build
        _build.build()
    L = C.CDLL(LIB_PATH)
    vp, dp, fp, cp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_float), C.c_char_p, C.c_int
    L.fx_create.argtypes = [C.POINTER(FxGrid), C.POINTER(FxParams), C.POINTER(vp)]
    L.fx_destroy.argtypes = [vp]
    L.fx_destroy.restype = None
    L.fx_last_error.argtypes = [vp]
    L.fx_last_error.restype = cp
    L.fx_device_bytes.argtypes = [vp, C.POINTER(C.c_longlong)]
    L.fx_footprint.argtypes = [C.POINTER(FxGrid), C.POINTER(FxParams), ip, C.POINTER(C.c_longlong)]
    L.fx_upload.argtypes = [vp, cp, dp]
    L.fx_download.argtypes = [vp, cp, dp]
    L.fx_upload_flags.argtypes = [vp, fp, fp]
    L.fx_download_flags.argtypes = [vp, fp, fp, fp]
    L.fx_set_forcing.argtypes = [vp, fp, ip]
    L.fx_set_inflow.argtypes = [vp, fp, ip, ip]
    L.fx_set_manning.argtypes = [vp, dp]
    L.fx_set_melt_field.argtypes = [vp, dp]
    L.fx_set_option.argtypes = [vp, cp, C.c_longlong]
    L.fx_prepare.argtypes = [vp]
    L.fx_step.argtypes = [vp, ip, C.POINTER(FxStatus)]
    L.fx_run_to_print.argtypes = [vp, C.POINTER(FxStatus)]
    L.fx_print_done.argtypes = [vp]
    L.fx_get_status.argtypes = [vp, C.POINTER(FxStatus)]
    L.fx_stream.argtypes = [vp]
    L.fx_stream.restype = vp
    L.fx_time_steps.argtypes = [vp, ip, dp, dp, dp]
    L.fx_mass.argtypes = [vp, dp, dp]
    L.fx_autotune.argtypes = [vp, ip, C.POINTER(ip)]
    L.fx_batch_set_option.argtypes = [vp, cp, C.c_longlong]
    L.fx_batch_autotune.argtypes = [vp, ip, C.POINTER(ip), C.POINTER(ip)]
    L.fx_adesolver_noalloc.argtypes = [vp, vp, vp, vp, vp, vp, ip, ip, ip, ip, C.c_double, C.c_double, vp]
    L.fx_batch_create.argtypes = [C.POINTER(vp)]
    L.fx_batch_destroy.argtypes = [vp]
    L.fx_batch_destroy.restype = None
    L.fx_batch_last_error.argtypes = [vp]
    L.fx_batch_last_error.restype = cp
    L.fx_batch_add.argtypes = [vp, vp]
    L.fx_batch_remove.argtypes = [vp, vp]
    L.fx_batch_size.argtypes = [vp]
    L.fx_batch_step.argtypes = [vp, ip, C.POINTER(FxStatus)]
    L.fx_batch_stream.argtypes = [vp]
    L.fx_batch_stream.restype = vp
    L.fx_initiate.argtypes = [vp, dp]
    L.fx_load_modset.argtypes = [cp, C.POINTER(FxGrid), C.POINTER(FxParams), dp, dp, dp, dp, dp, dp,
                                 dp, dp, fp, fp, fp, C.POINTER(ip)]
    L.fx_open_modset.argtypes = [cp, C.POINTER(vp)]
    L.fx_write_results.argtypes = [vp, cp]
    L.fx_write_results_async.argtypes = [vp, cp]
    L.fx_results_wait.argtypes = [vp]
    L.fx_write_results_host.argtypes = [cp, ip, ip, ip, C.c_double, C.c_double, C.c_double, dp, dp, dp,
                                        dp, dp, dp, dp, dp, dp, dp]
    L.fx_run.argtypes = [cp]
    _lib = L
    return L


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _check(rc: int, ctx=None) -> None:
    if rc != 0:
        msg = lib().fx_last_error(ctx)
        raise FluxosError(rc, msg.decode() if msg else "")


def load_modset(path: str) -> dict:
    """Host-only start-up (no GPU): the grid, parameters and initial state
    the reference builds from a modset (main.cpp:104-262)."""
    L = lib()
    g, p = FxGrid(), FxParams()
    nul = C.POINTER(C.c_double)()
    nulf = C.POINTER(C.c_float)()
    _check(L.fx_load_modset(path.encode(), C.byref(g), C.byref(p), nul, nul, nul, nul, nul, nul, nul,
                            nul, nulf, nulf, nulf, None))
    shape = (g.ncols + 2, g.nrows + 2)
    out = {k: np.zeros(shape) for k in ("zb", "z", "h", "qx", "qy", "twet", "conc", "soil_mass")}
    out["ldry"] = np.zeros(shape, dtype=np.float32)
    out["wall"] = np.zeros(shape, dtype=np.float32)
    out["meteo"] = np.zeros((3, METEO_ROWS), dtype=np.float32)
    hm = C.c_int(0)
    _check(L.fx_load_modset(path.encode(), C.byref(g), C.byref(p), _dptr(out["zb"]), _dptr(out["z"]),
                            _dptr(out["h"]), _dptr(out["qx"]), _dptr(out["qy"]), _dptr(out["twet"]),
                            _dptr(out["conc"]), _dptr(out["soil_mass"]), _fptr(out["ldry"]),
                            _fptr(out["wall"]), _fptr(out["meteo"]), C.byref(hm)))
    out["grid"] = {k: getattr(g, k) for k, _ in g._fields_}
    out["params"] = {k: getattr(p, k) for k, _ in p._fields_ if k != "d_coef"}
    out["params"]["d_coef"] = list(p.d_coef)
    out["has_meteo"] = hm.value
    return out


def write_results_host(path: str, nrows: int, ncols: int, dxy: int, xll: float, yll: float,
                       h_min_print: float, grids: dict) -> None:
    """write_results (write_results.cpp:30-101) on host grids; without a
    "soil_mass" grid that column is 0."""
    a = {k: np.ascontiguousarray(grids[k], dtype=np.float64) for k in
         ("z", "zb", "h", "qx", "qy", "conc", "fe_1", "fn_1", "twet")}
    soil_arr = np.ascontiguousarray(grids["soil_mass"], dtype=np.float64) if "soil_mass" in grids else None
    soil = _dptr(soil_arr) if soil_arr is not None else C.POINTER(C.c_double)()
    _check(lib().fx_write_results_host(path.encode(), nrows, ncols, dxy, xll, yll, h_min_print,
                                       _dptr(a["z"]), _dptr(a["zb"]), _dptr(a["h"]), _dptr(a["qx"]),
                                       _dptr(a["qy"]), _dptr(a["conc"]), soil, _dptr(a["fe_1"]),
                                       _dptr(a["fn_1"]), _dptr(a["twet"])))


def run(modset_path: str) -> None:
    """The whole program, like the reference's ``fluxos <modset.json>``."""
    _check(lib().fx_run(modset_path.encode()))


def footprint(nrows: int, ncols: int, *, nchem: int = 1, precision: str = "fp64",
              steps_in_flight: int = 0, extension_grids: int = 0) -> int:
    """Device bytes a Domain of this size would hold (fx_footprint)."""
    g = FxGrid(nrows, ncols, 1, nchem, -9999.0, 0.0, 0.0)
    p = FxParams()
    p.steps_in_flight = int(steps_in_flight)
    p.precision = 1 if precision == "fp32" else 0
    v = C.c_longlong(0)
    _check(lib().fx_footprint(C.byref(g), C.byref(p), int(extension_grids), C.byref(v)))
    return v.value


class Domain:
    """One FLUXOS-OVERLAND domain resident on the GPU (an fx_ctx)."""

    def __init__(self, nrows: int, ncols: int, dxy: int, *, nchem: int = 1, nodata: float = -9999.0,
                 xll: float = 0.0, yll: float = 0.0, hdry: float = 0.001, ks: Optional[float] = None,
                 ntim: float = 0.0, print_step: float = 600.0, print_next: Optional[float] = None,
                 tim: float = 0.0, h_min_print: float = 0.0, ade: bool = True, volrat_mode: int = 0,
                 d_coef: Sequence[float] = (0.01,), steps_in_flight: int = 0, precision: str = "fp64",
                 wintra: bool = False, soil_release_rate: float = 0.0, _handle=None):
        self.L = lib()
        self.nrows, self.ncols, self.dxy, self.nchem = nrows, ncols, dxy, nchem
        self.xll, self.yll, self.h_min_print = xll, yll, h_min_print
        if precision not in ("fp64", "fp32"):
            raise ValueError("precision must be 'fp64' or 'fp32'")
        self.precision = precision
        if _handle is not None:
            self.h = _handle
            return
        g = FxGrid(nrows, ncols, int(dxy), nchem, float(nodata), float(xll), float(yll))
        p = FxParams()
        p.hdry = hdry
        p.ks = hdry if ks is None else ks
        p.ntim = ntim
        p.print_step = print_step
        p.print_next = print_step if print_next is None else print_next
        p.tim = tim
        p.h_min_print = h_min_print
        p.ade = 1 if ade else 0
        p.volrat_mode = volrat_mode
        for k in range(MAX_CHEM):
            p.d_coef[k] = float(d_coef[k] if k < len(d_coef) else d_coef[-1])
        p.steps_in_flight = int(steps_in_flight)
        p.precision = 1 if precision == "fp32" else 0
        p.wintra = 1 if wintra else 0
        p.soil_release_rate = float(soil_release_rate)
        h = C.c_void_p()
        _check(self.L.fx_create(C.byref(g), C.byref(p), C.byref(h)))
        self.h = h

    @classmethod
    def from_modset(cls, path: str) -> "Domain":
        L = lib()
        h = C.c_void_p()
        _check(L.fx_open_modset(path.encode(), C.byref(h)))
        info = load_modset(path)
        g = info["grid"]
        d = cls(g["nrows"], g["ncols"], g["dxy"], nchem=g["nchem"], xll=g["xll"], yll=g["yll"],
                h_min_print=info["params"]["h_min_print"], _handle=h)
        return d

    @classmethod
    def from_modset_state(cls, path: str, *, steps_in_flight: int = 0, precision: str = "fp64") -> "Domain":
        """A context holding the start-up state of a modset (the state
        fx_open_modset builds, from the host loader), with the given steps in
        flight and precision; no output folder is created."""
        info = load_modset(path)
        g, p = info["grid"], info["params"]
        d = cls(g["nrows"], g["ncols"], g["dxy"], nchem=g["nchem"], nodata=g["nodata"], xll=g["xll"],
                yll=g["yll"], hdry=p["hdry"], ks=p["ks"], ntim=p["ntim"], print_step=p["print_step"],
                print_next=p["print_next"], tim=p["tim"], h_min_print=p["h_min_print"], ade=bool(p["ade"]),
                volrat_mode=p["volrat_mode"], d_coef=p["d_coef"][:g["nchem"]],
                steps_in_flight=steps_in_flight, precision=precision, wintra=bool(p["wintra"]),
                soil_release_rate=p["soil_release_rate"])
        for k in ("zb", "z", "h", "qx", "qy", "twet", "conc"):
            d.upload(k, info[k])
        if p["wintra"] or info["soil_mass"].any():
            d.upload("soil_mass", info["soil_mass"])
        d.upload_flags(info["ldry"], info["wall"])
        d.set_forcing(info["meteo"] if info["has_meteo"] else None)
        d.prepare()
        return d

    def close(self) -> None:
        if getattr(self, "h", None):
            self.L.fx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc: int) -> None:
        _check(rc, self.h)

    @property
    def shape(self):
        return (self.ncols + 2, self.nrows + 2)

    def upload(self, field: str, grid: np.ndarray) -> None:
        a = np.ascontiguousarray(grid, dtype=np.float64)
        assert a.shape == self.shape, (a.shape, self.shape)
        self._ck(self.L.fx_upload(self.h, field.encode(), _dptr(a)))

    def download(self, field: str, out: Optional[np.ndarray] = None) -> np.ndarray:
        a = np.empty(self.shape) if out is None else out
        self._ck(self.L.fx_download(self.h, field.encode(), _dptr(a)))
        return a

    def upload_flags(self, ldry: np.ndarray, wall: np.ndarray) -> None:
        a = np.ascontiguousarray(ldry, dtype=np.float32)
        b = np.ascontiguousarray(wall, dtype=np.float32)
        self._ck(self.L.fx_upload_flags(self.h, _fptr(a), _fptr(b)))

    def download_flags(self):
        a = np.empty(self.shape, dtype=np.float32)
        b = np.empty(self.shape, dtype=np.float32)
        c = np.empty(self.shape, dtype=np.float32)
        self._ck(self.L.fx_download_flags(self.h, _fptr(a), _fptr(b), _fptr(c)))
        return {"ldry": a, "ldry_prev": b, "wall": c}

    def set_forcing(self, table: Optional[np.ndarray]) -> None:
        if table is None:
            self._ck(self.L.fx_set_forcing(self.h, None, 0))
            return
        t = np.ascontiguousarray(table, dtype=np.float32)
        assert t.shape == (3, METEO_ROWS)
        self._ck(self.L.fx_set_forcing(self.h, _fptr(t), 1))

    def set_inflow(self, table: Optional[np.ndarray], irow: int = 0, icol: int = 0) -> None:
        """Point inflow: (3, 2000) float table (time, discharge m^3/s, conc), rows from 0."""
        if table is None:
            self._ck(self.L.fx_set_inflow(self.h, None, 0, 0))
            return
        t = np.ascontiguousarray(table, dtype=np.float32)
        assert t.shape == (3, METEO_ROWS)
        self._keep_inflow = t
        self._ck(self.L.fx_set_inflow(self.h, _fptr(t), int(irow), int(icol)))

    def set_manning(self, grid: Optional[np.ndarray]) -> None:
        self._keep_n = None if grid is None else np.ascontiguousarray(grid, dtype=np.float64)
        self._ck(self.L.fx_set_manning(self.h, None if grid is None else _dptr(self._keep_n)))

    def set_melt_field(self, grid: Optional[np.ndarray]) -> None:
        self._keep_m = None if grid is None else np.ascontiguousarray(grid, dtype=np.float64)
        self._ck(self.L.fx_set_melt_field(self.h, None if grid is None else _dptr(self._keep_m)))

    def set_option(self, name: str, value: int) -> None:
        self._ck(self.L.fx_set_option(self.h, name.encode(), int(value)))

    def initiate(self, zb_raw: np.ndarray) -> None:
        a = np.ascontiguousarray(zb_raw, dtype=np.float64)
        self._ck(self.L.fx_initiate(self.h, _dptr(a)))

    def prepare(self) -> None:
        self._ck(self.L.fx_prepare(self.h))

    def step(self, n: int = 1) -> dict:
        st = FxStatus()
        self._ck(self.L.fx_step(self.h, int(n), C.byref(st)))
        return st.as_dict()

    def run_to_print(self) -> dict:
        st = FxStatus()
        self._ck(self.L.fx_run_to_print(self.h, C.byref(st)))
        return st.as_dict()

    def print_done(self) -> None:
        self._ck(self.L.fx_print_done(self.h))

    def status(self) -> dict:
        st = FxStatus()
        self._ck(self.L.fx_get_status(self.h, C.byref(st)))
        return st.as_dict()

    def stream(self) -> int:
        return int(self.L.fx_stream(self.h) or 0)

    def device_bytes(self) -> int:
        v = C.c_longlong(0)
        self._ck(self.L.fx_device_bytes(self.h, C.byref(v)))
        return v.value

    def time_steps(self, n: int):
        t, a, b = C.c_double(), C.c_double(), C.c_double()
        self._ck(self.L.fx_time_steps(self.h, int(n), C.byref(t), C.byref(a), C.byref(b)))
        return t.value, a.value, b.value

    def autotune(self, trial_steps: int = 16) -> int:
        """Pick the fastest tile shape on this domain (runs real steps)."""
        r = C.c_int(0)
        self._ck(self.L.fx_autotune(self.h, int(trial_steps), C.byref(r)))
        return r.value

    def mass(self):
        """(stored water [m^3], array of stored solute masses), FP64 sums on the device."""
        w = C.c_double()
        m = np.zeros(MAX_CHEM)
        self._ck(self.L.fx_mass(self.h, C.byref(w), _dptr(m)))
        return w.value, m[: self.nchem].copy()

    def write_results(self, path: Optional[str] = None, wait: bool = True) -> None:
        """The Results file of the current state (write_results.cpp:30-101),
        by default <OUTPUT_FOLDER>/<print_next>.txt. With wait=False the rows
        are compacted on the device and the file is written by a host thread
        while the domain keeps stepping; results_wait() collects the outcome."""
        p = path.encode() if path else None
        if wait:
            self._ck(self.L.fx_write_results(self.h, p))
        else:
            self._ck(self.L.fx_write_results_async(self.h, p))

    def results_wait(self) -> None:
        self._ck(self.L.fx_results_wait(self.h))


class Batch:
    """Several domains advanced together by the same launches (fx_batch)."""

    def __init__(self):
        self.L = lib()
        h = C.c_void_p()
        _check(self.L.fx_batch_create(C.byref(h)))
        self.h = h
        self.members = []

    def close(self) -> None:
        if getattr(self, "h", None):
            self.L.fx_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, d: "Domain") -> None:
        _check(self.L.fx_batch_add(self.h, d.h))
        self.members.append(d)

    def remove(self, d: "Domain") -> None:
        _check(self.L.fx_batch_remove(self.h, d.h))
        self.members.remove(d)

    def step(self, n: int) -> list:
        arr = (FxStatus * max(1, len(self.members)))()
        _check(self.L.fx_batch_step(self.h, int(n), arr))
        return [arr[i].as_dict() for i in range(len(self.members))]

    def stream(self) -> int:
        return int(self.L.fx_batch_stream(self.h) or 0)

    def set_option(self, name: str, value: int) -> None:
        _check(self.L.fx_batch_set_option(self.h, name.encode(), int(value)))

    def autotune(self, trial_steps: int = 8):
        """(tile_rows, steps_in_flight) picked for this batch (runs real steps)."""
        r, k = C.c_int(0), C.c_int(0)
        _check(self.L.fx_batch_autotune(self.h, int(trial_steps), C.byref(r), C.byref(k)))
        return r.value, k.value

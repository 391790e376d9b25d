"""ctypes front-ends for the two CPU checkers of the FLUXOS step.

TEST INFRASTRUCTURE ONLY (tests/, __graft_entry__.smoke(), bench.py's CPU legs).

* :class:`OracleRun` drives the project's C restatement
  (``oracle/libfluxos_oracle.so``);
* :class:`RefRun` drives the FLUXOS reference sources compiled here
  (``oracle/_ref/libfluxos_ref.so``, or ``libfluxos_ref_closed.so`` for the
  "closed" edge mode), built only where the reference tree exists.

Both expose the same calls, so a test can run them side by side. Grids come
back as numpy views of shape ``(ncols + 2, nrows + 2)``: index ``[icol, irow]``
over the column-major Armadillo layout of the reference's GlobVar.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libfluxos_oracle.so")
REF_SO = {0: os.path.join(HERE, "_ref", "libfluxos_ref.so"),
          1: os.path.join(HERE, "_ref", "libfluxos_ref_closed.so")}
REF_BIN = os.path.join(HERE, "_ref", "fluxos_ref")

DGRIDS = ("z", "zb", "h", "qx", "qy", "us", "ks", "fe_1", "fe_2", "fe_3", "fn_1", "fn_2", "fn_3",
          "twet", "h0", "dh", "dqx", "dqy", "qxf", "qyf", "soil_mass", "conc")
FGRIDS = ("ldry", "ldry_prev", "wall")
METEO_ROWS = 2000

_libs = {}


def _load(path: str) -> C.CDLL:
    if path not in _libs:
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (run oracle/Makefile)")
        lib = C.CDLL(path)
        _libs[path] = lib
    return _libs[path]


def oracle_lib() -> C.CDLL:
    lib = _load(ORACLE_SO)
    vp, dp, fp, cp = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_float), C.c_char_p
    lib.ox_create.restype = vp
    lib.ox_create.argtypes = [C.c_int, C.c_int, C.c_int]
    lib.ox_destroy.argtypes = [vp]
    lib.ox_grid.restype = dp
    lib.ox_grid.argtypes = [vp, cp]
    lib.ox_fgrid.restype = fp
    lib.ox_fgrid.argtypes = [vp, cp]
    lib.ox_scalar.restype = C.c_double
    lib.ox_scalar.argtypes = [vp, cp]
    lib.ox_set_scalar.argtypes = [vp, cp, C.c_double]
    lib.ox_set_manning.argtypes = [vp, dp]
    lib.ox_set_melt_field.argtypes = [vp, dp]
    lib.ox_read_dem.argtypes = [cp, C.c_int, C.c_int, dp]
    lib.ox_read_dem.restype = C.c_int
    lib.ox_geo_prepare.argtypes = [vp, dp, C.c_double]
    lib.ox_initiation_zero.argtypes = [vp]
    for n in ("ox_courant", "ox_hydrodynamics", "ox_manning", "ox_print_done"):
        getattr(lib, n).argtypes = [vp]
    for n in ("ox_add_meteo", "ox_add_inflow", "ox_step", "ox_running", "ox_print_due"):
        getattr(lib, n).argtypes = [vp]
        getattr(lib, n).restype = C.c_int
    lib.ox_adesolver.argtypes = [vp, C.c_int, C.c_int]
    lib.ox_weir_term.argtypes = [C.c_double, C.c_double]
    lib.ox_weir_term.restype = C.c_double
    return lib


def ref_available(mode: int = 0) -> bool:
    return os.path.exists(REF_SO[mode])


def ref_lib(mode: int = 0) -> C.CDLL:
    lib = _load(REF_SO[mode])
    vp, dp, fp, cp = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_float), C.c_char_p
    lib.fxr_open.restype = vp
    lib.fxr_open.argtypes = [cp]
    lib.fxr_close.argtypes = [vp]
    lib.fxr_main.argtypes = [cp]
    lib.fxr_main.restype = C.c_int
    lib.fxr_grid.restype = dp
    lib.fxr_grid.argtypes = [vp, cp]
    lib.fxr_fgrid.restype = fp
    lib.fxr_fgrid.argtypes = [vp, cp]
    lib.fxr_scalar.restype = C.c_double
    lib.fxr_scalar.argtypes = [vp, cp]
    lib.fxr_set_scalar.argtypes = [vp, cp, C.c_double]
    for n in ("fxr_courant", "fxr_hydrodynamics"):
        getattr(lib, n).argtypes = [vp]
    for n in ("fxr_add_meteo", "fxr_add_inflow", "fxr_step", "fxr_running", "fxr_maybe_print"):
        getattr(lib, n).argtypes = [vp]
        getattr(lib, n).restype = C.c_int
    lib.fxr_adesolver.argtypes = [vp, C.c_int, C.c_int]
    return lib


def read_meteo_table(path: str) -> np.ndarray:
    """The 2000x3 float forcing table as read_meteo fills it
    (read_functions.cpp:256-272): CSV tokens parsed as double, stored as
    float, data row k (1-based after the header) into table row k."""
    tab = np.zeros((3, METEO_ROWS), dtype=np.float32)  # [col, row] = column-major fmat
    with open(path) as f:
        lines = f.read().split("\n")
    rows = []
    for ln in lines:
        if ln == "":
            break
        vals = []
        for tok in ln.split(","):
            try:
                vals.append(float(tok))
            except ValueError:
                vals.append(0.0)
        rows.append(vals)
    for a in range(1, len(rows)):
        for c in range(3):
            tab[c, a] = np.float32(rows[a][c] if c < len(rows[a]) else 0.0)
    return tab


def read_inflow_table(path: str) -> np.ndarray:
    """The 2000x3 float point-inflow table as read_inflow fills it
    (read_functions.cpp:303-316): like the forcing table, but data row k
    (1-based after the header) into table row k - 1."""
    tab = read_meteo_table(path)
    out = np.zeros_like(tab)
    out[:, :-1] = tab[:, 1:]
    return out


class _Run:
    nrows: int
    ncols: int

    def grid(self, name: str) -> np.ndarray:
        raise NotImplementedError

    def interior(self, name: str) -> np.ndarray:
        return self.grid(name)[1:-1, 1:-1]

    def snapshot(self, names=DGRIDS + FGRIDS) -> dict:
        return {n: self.grid(n).copy() for n in names}

    def apply_wet_start(self, h: np.ndarray, qx: Optional[np.ndarray] = None,
                        qy: Optional[np.ndarray] = None, conc: Optional[list] = None) -> None:
        """Overwrite the interior state after start-up: z = zb + h, ldry = 0
        where h > 0 (as a restart file would, initiate.cpp:133-156)."""
        zb = self.interior("zb")
        self.interior("h")[...] = h.T
        self.interior("z")[...] = zb + h.T
        if qx is not None:
            self.interior("qx")[...] = qx.T
        if qy is not None:
            self.interior("qy")[...] = qy.T
        if conc is not None:
            for k, c in enumerate(conc):
                self.interior("conc" if k == 0 else f"conc{k}")[...] = c.T
        self.interior("ldry")[...] = np.where(h.T > 0, 0.0, 1.0).astype(np.float32)


class OracleRun(_Run):
    """The C restatement, started from a scenario's files like main.cpp:104-262."""

    def __init__(self, modset_dir: str, sc, volrat_mode: int = 0):
        self.lib = oracle_lib()
        self.nrows, self.ncols = sc.nrows, sc.ncols
        self.s = self.lib.ox_create(sc.nrows, sc.ncols, sc.nchem)
        L, s = self.lib, self.s
        L.ox_set_scalar(s, b"dxy", float(sc.dxy))
        L.ox_set_scalar(s, b"nodata", float(sc.nodata))
        L.ox_set_scalar(s, b"print_step", float(sc.print_step))
        L.ox_set_scalar(s, b"ade", 1.0 if sc.ade else 0.0)
        L.ox_set_scalar(s, b"volrat_mode", float(volrat_mode))
        L.ox_set_scalar(s, b"wintra", 1.0 if (sc.wintra and sc.ade) else 0.0)  # main.cpp:209-213
        L.ox_set_scalar(s, b"soil_release_rate", float(sc.soil_release_rate))
        if sc.d_coefs:
            for k, d in enumerate(sc.d_coefs):
                L.ox_set_scalar(s, f"D_coef{k}".encode(), float(d))
        else:
            L.ox_set_scalar(s, b"D_coef", float(sc.d_coef))
        zb_raw = np.zeros((sc.ncols + 2, sc.nrows + 2), dtype=np.float64)
        rc = L.ox_read_dem(os.path.join(modset_dir, "dem.asc").encode(), sc.nrows, sc.ncols,
                           zb_raw.ctypes.data_as(C.POINTER(C.c_double)))
        if rc:
            raise IOError("DEM not readable")
        self._zb_raw = zb_raw
        L.ox_geo_prepare(s, zb_raw.ctypes.data_as(C.POINTER(C.c_double)), float(np.float64(sc.ks)))
        L.ox_initiation_zero(s)
        tab = read_meteo_table(os.path.join(modset_dir, "meteo.csv"))
        self.fgrid("meteo")[...] = tab
        L.ox_set_scalar(s, b"has_meteo", 1.0)
        n_data = self._meteo_rows(os.path.join(modset_dir, "meteo.csv"))
        last_t = float(tab[0, n_data]) if n_data > 0 else 0.0
        ntim = int(np.float32(last_t))
        if sc.inflow is not None:  # read_inflow, read_geo's discharge cell (read_functions.cpp:228-231)
            from fluxos_cpp_b200 import scenarios as _S
            itab = read_inflow_table(os.path.join(modset_dir, "inflow.csv"))
            self.fgrid("inflow")[...] = itab
            L.ox_set_scalar(s, b"has_inflow", 1.0)
            irow, icol = _S.inflow_cell(sc)
            L.ox_set_scalar(s, b"inflow_nrow", float(irow))
            L.ox_set_scalar(s, b"inflow_ncol", float(icol))
            n_in = self._meteo_rows(os.path.join(modset_dir, "inflow.csv"))
            ntim = max(ntim, int(np.float32(itab[0, n_in - 1])) if n_in > 0 else 0)
        L.ox_set_scalar(s, b"ntim", float(ntim))  # main.cpp:181-192
        L.ox_set_scalar(s, b"print_next", float(sc.print_step))
        self._keep = []
        if sc.manning is not None:
            m = np.zeros((sc.ncols + 2, sc.nrows + 2))
            m[1:-1, 1:-1] = sc.manning.T
            self._keep.append(m)
            L.ox_set_manning(s, m.ctypes.data_as(C.POINTER(C.c_double)))
        if sc.melt_mult is not None:
            m = np.ones((sc.ncols + 2, sc.nrows + 2))
            m[1:-1, 1:-1] = sc.melt_mult.T
            self._keep.append(m)
            L.ox_set_melt_field(s, m.ctypes.data_as(C.POINTER(C.c_double)))

    @staticmethod
    def _meteo_rows(path: str) -> int:
        n = 0
        with open(path) as f:
            for ln in f.read().split("\n"):
                if ln == "":
                    break
                n += 1
        return n - 1

    def __del__(self):
        try:
            self.lib.ox_destroy(self.s)
        except Exception:
            pass

    def grid(self, name: str) -> np.ndarray:
        p = self.lib.ox_grid(self.s, name.encode())
        if not p:
            if name in FGRIDS:
                return self.fgrid(name)
            raise KeyError(name)
        return np.ctypeslib.as_array(p, shape=(self.ncols + 2, self.nrows + 2))

    def fgrid(self, name: str) -> np.ndarray:
        p = self.lib.ox_fgrid(self.s, name.encode())
        if not p:
            raise KeyError(name)
        if name in ("meteo", "inflow"):
            return np.ctypeslib.as_array(p, shape=(3, METEO_ROWS))
        return np.ctypeslib.as_array(p, shape=(self.ncols + 2, self.nrows + 2))

    def scalar(self, name: str) -> float:
        return self.lib.ox_scalar(self.s, name.encode())

    def set_scalar(self, name: str, v: float) -> None:
        self.lib.ox_set_scalar(self.s, name.encode(), float(v))

    def courant(self):
        self.lib.ox_courant(self.s)

    def add_meteo(self):
        return self.lib.ox_add_meteo(self.s)

    def hydrodynamics(self):
        self.lib.ox_hydrodynamics(self.s)

    def adesolver(self, it: int, ichem: int = 0):
        self.lib.ox_adesolver(self.s, it, ichem)

    def step(self) -> int:
        return self.lib.ox_step(self.s)

    def running(self) -> bool:
        return bool(self.lib.ox_running(self.s))

    def print_due(self) -> bool:
        return bool(self.lib.ox_print_due(self.s))

    def print_done(self) -> None:
        self.lib.ox_print_done(self.s)


class RefRun(_Run):
    """The reference sources, started by the harness (main.cpp:104-262)."""

    def __init__(self, modset_path: str, sc, volrat_mode: int = 0):
        self.lib = ref_lib(volrat_mode)
        self.nrows, self.ncols = sc.nrows, sc.ncols
        self.h = self.lib.fxr_open(modset_path.encode())
        if not self.h:
            raise IOError("reference start-up failed")

    def __del__(self):
        try:
            self.lib.fxr_close(self.h)
        except Exception:
            pass

    def grid(self, name: str) -> np.ndarray:
        if name in FGRIDS:
            return self.fgrid(name)
        p = self.lib.fxr_grid(self.h, name.encode())
        if not p:
            raise KeyError(name)
        return np.ctypeslib.as_array(p, shape=(self.ncols + 2, self.nrows + 2))

    def fgrid(self, name: str) -> np.ndarray:
        p = self.lib.fxr_fgrid(self.h, name.encode())
        if not p:
            raise KeyError(name)
        if name in ("meteo", "inflow"):
            return np.ctypeslib.as_array(p, shape=(3, METEO_ROWS))
        return np.ctypeslib.as_array(p, shape=(self.ncols + 2, self.nrows + 2))

    def scalar(self, name: str) -> float:
        return self.lib.fxr_scalar(self.h, name.encode())

    def set_scalar(self, name: str, v: float) -> None:
        self.lib.fxr_set_scalar(self.h, name.encode(), float(v))

    def courant(self):
        self.lib.fxr_courant(self.h)

    def add_meteo(self):
        return self.lib.fxr_add_meteo(self.h)

    def hydrodynamics(self):
        self.lib.fxr_hydrodynamics(self.h)

    def adesolver(self, it: int, ichem: int = 0):
        self.lib.fxr_adesolver(self.h, it, ichem)

    def step(self) -> int:
        return self.lib.fxr_step(self.h)

    def running(self) -> bool:
        return bool(self.lib.fxr_running(self.h))

    def print_due(self) -> bool:
        return self.scalar("tim") >= self.scalar("print_next")

    def print_done(self) -> None:
        self.set_scalar("print_next", self.scalar("print_next") + self.scalar("print_step"))


def max_ulp_diff(a: np.ndarray, b: np.ndarray) -> float:
    """Largest relative difference |a-b| / max(|a|,|b|,tiny), NaN-aware."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    both_nan = np.isnan(a) & np.isnan(b)
    d = np.abs(a - b)
    s = np.maximum(np.maximum(np.abs(a), np.abs(b)), 1e-300)
    r = np.where(both_nan, 0.0, d / s)
    r = np.where((a == b), 0.0, r)
    return float(np.nanmax(r)) if r.size else 0.0

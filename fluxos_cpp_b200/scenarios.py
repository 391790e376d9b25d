"""Seeded synthetic FLUXOS-OVERLAND scenarios and their input files.

A scenario is written in the reference's own input formats, so the same files
drive the reference program and this package:

* ``modset.json``: the master file read by ``read_modset``
  (reference ``src/fluxos/read_functions.cpp:26-110``);
* ``dem.asc``: ESRI ASCII grid read by ``get_domain_size`` and ``read_geo``
  (``common.cpp:110-161``, ``read_functions.cpp:112-235``). The first data
  line is grid row ``irow = NROWS`` (``read_functions.cpp:145-163``);
* ``meteo.csv``: header plus ``time [s], rate [mm/day], concentration`` rows
  read by ``read_meteo`` (``read_functions.cpp:237-282``);
* ``inflow.csv`` (only with a point inflow): header plus ``time [s],
  discharge [m^3/s], concentration`` rows read by ``read_inflow``
  (``read_functions.cpp:284-326``), entering the cell of the modset's
  ``INFLOW_FILE.DISCHARGE_LOCATION``.

The reference picks the first forcing row whose time exceeds the clock
(``common.cpp:195-200``) and sets the run length from the last row's time
(``read_functions.cpp:280``, ``main.cpp:192``). The writer therefore appends a
guard row far in the future with rate 0, followed by a final row at the
horizon: the clock never runs off the end of the table, and the run still
stops at the horizon.

Grids in this module are numpy arrays of shape ``(nrows, ncols)`` indexed
``[irow - 1, icol - 1]``. The synthetic fields replace the public datasets
the configurations name (none is available offline); they follow the stated
shapes, sizes and value ranges.
"""
from __future__ import annotations

import json
import math
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

GUARD_TIME = 1.0e9  # exactly representable as float32


@dataclass
class Scenario:
    """One overland-flow run: terrain, forcing, physics switches and output."""

    name: str
    dem: np.ndarray  # (nrows, ncols) bed elevation [m], NODATA or 0 -> wall
    dxy: int = 2  # integer cell size [m] (GlobVar.h:76)
    xll: float = 0.0
    yll: float = 0.0
    nodata: int = -9999
    meteo: Sequence[Tuple[float, float, float]] = ((0.0, 20.0, 1.0),)
    horizon: float = 21600.0  # [s]; sets the reference's ntim
    print_step: int = 600
    ks: float = 0.001  # ROUGNESS_HEIGHT, also the dry threshold hdry
    ade: bool = True
    d_coef: float = 0.01
    h_min_print: float = 0.0
    # Extensions (no reference counterpart); None = parity mode.
    manning: Optional[np.ndarray] = None
    melt_mult: Optional[np.ndarray] = None
    d_coefs: Optional[List[float]] = None  # one D per solute (>= 1 solutes)
    # Optional point inflow (INFLOW_FILE): rows (t [s], discharge [m^3/s],
    # concentration) and the discharge location (X, Y) in the DEM's
    # coordinates, integers as the reference stores them (GlobVar.h:100).
    inflow: Optional[Sequence[Tuple[float, float, float]]] = None
    inflow_xy: Optional[Tuple[int, int]] = None
    # WINTRA soil release (EXTERNAL_MODULES.WINTRA, SOIL_RELEASE_RATE [1/hour])
    # and the soil mass per cell it releases (interior array; the reference
    # only fills it from a restart file, initiate.cpp:93-152).
    wintra: bool = False
    soil_release_rate: float = 0.0
    init_soil: Optional[np.ndarray] = None
    # Optional wet start (interior arrays, same shape as dem).
    init_h: Optional[np.ndarray] = None
    init_qx: Optional[np.ndarray] = None
    init_qy: Optional[np.ndarray] = None
    init_conc: Optional[List[np.ndarray]] = None
    extra: dict = field(default_factory=dict)

    @property
    def nrows(self) -> int:
        return int(self.dem.shape[0])

    @property
    def ncols(self) -> int:
        return int(self.dem.shape[1])

    @property
    def nchem(self) -> int:
        return len(self.d_coefs) if self.d_coefs else 1

    def write(self, folder: str) -> str:
        """Write modset.json, dem.asc and meteo.csv; return the modset path."""
        os.makedirs(folder, exist_ok=True)
        dem_path = os.path.join(folder, "dem.asc")
        met_path = os.path.join(folder, "meteo.csv")
        out_dir = os.path.join(folder, "Results")
        write_esri_ascii(dem_path, self.dem, self.dxy, self.xll, self.yll, self.nodata)
        write_meteo(met_path, self.meteo, self.horizon)
        inflow_path = os.path.join(folder, "inflow.csv")
        if self.inflow is not None:
            write_meteo(inflow_path, self.inflow, self.horizon)
        modset = {
            "COMMNET": f"synthetic scenario {self.name}",
            "DEM_FILE": dem_path,
            "SIM_DATETIME_START": "2020JAN01 00:00:00",
            "RESTART": False,
            "METEO_FILE": met_path,
            "OUTPUT": {
                "OUTPUT_FOLDER": out_dir,
                "PRINT_STEP": int(self.print_step),
                "H_MIN_TO_PRINT": self.h_min_print,
            },
            "ROUGNESS_HEIGHT": self.ks,
            "SOIL_RELEASE_RATE": float(self.soil_release_rate),
            "SOIL_CONC_BACKGROUND": 0.0,
            "EXTERNAL_MODULES": {
                "ADE_TRANSPORT": {"STATUS": bool(self.ade), "D_COEF": self.d_coef},
                "OPENWQ": {"STATUS": False, "MASTERFILE_DIR": ""},
                "WINTRA": {"STATUS": bool(self.wintra), "SWE_STD": 0.0, "SWE_MAX": 0.0},
            },
        }
        if self.inflow is not None:
            x, y = self.inflow_xy
            modset["INFLOW_FILE"] = {"FILENAME": inflow_path,
                                     "DISCHARGE_LOCATION": {"X_COORDINATE": int(x), "Y_COORDINATE": int(y)}}
        path = os.path.join(folder, "modset.json")
        with open(path, "w") as f:
            f.write("// FLUXOS master file (comments allowed, main.cpp:106-109)\n")
            json.dump(modset, f, indent=2)
        return path


def write_esri_ascii(path: str, dem: np.ndarray, dxy: int, xll: float, yll: float,
                     nodata: int) -> None:
    """ESRI ASCII grid; data line k (0-based) holds grid row irow = NROWS - k."""
    nr, nc = dem.shape
    with open(path, "w") as f:
        f.write(f"NCOLS {nc}\nNROWS {nr}\nXLLCORNER {xll!r}\nYLLCORNER {yll!r}\n")
        f.write(f"CELLSIZE {int(dxy)}\nNODATA_VALUE {int(nodata)}\n")
        vals = np.asarray(dem, dtype=np.float64)[::-1]
        for row in vals:
            f.write(" ".join("%.6f" % v for v in row))
            f.write("\n")


def write_meteo(path: str, rows: Sequence[Tuple[float, float, float]], horizon: float) -> None:
    """Forcing CSV with the guard row and the horizon row described above."""
    with open(path, "w") as f:
        f.write("t [s],rate [mm/day],conc [mg/l]\n")
        for t, r, c in rows:
            f.write("%r,%r,%r\n" % (float(t), float(r), float(c)))
        f.write("%r,0.0,0.0\n" % GUARD_TIME)
        f.write("%r,0.0,0.0\n" % float(horizon))


def box3(a: np.ndarray) -> np.ndarray:
    """3x3 box filter with edge replication."""
    p = np.pad(a, 1, mode="edge")
    out = np.zeros_like(a)
    for di in range(3):
        for dj in range(3):
            out += p[di:di + a.shape[0], dj:dj + a.shape[1]]
    return out / 9.0


def plane_dem(nrows: int, ncols: int, dxy: int = 2, slope: float = 0.01, sigma: float = 0.05,
              seed: int = 0, base: float = 100.0) -> np.ndarray:
    """Plane falling towards irow = NROWS (the outflow edge) plus smoothed
    i.i.d. Gaussian bumps; the small-domain configuration's terrain."""
    rng = np.random.default_rng(seed)
    irow = np.arange(1, nrows + 1, dtype=np.float64)[:, None]
    plane = base + slope * (nrows - irow) * dxy + np.zeros((1, ncols))
    bumps = box3(rng.normal(0.0, sigma, size=(nrows, ncols)))
    return (plane + bumps).astype(np.float32)


def spectral_field(n_rows: int, n_cols: int, beta: float, rng: np.random.Generator) -> np.ndarray:
    """Gaussian random field with power spectrum P(k) ~ k^-beta (zero mean)."""
    kx = np.fft.fftfreq(n_rows)[:, None]
    ky = np.fft.rfftfreq(n_cols)[None, :]
    k = np.sqrt(kx * kx + ky * ky)
    k[0, 0] = 1.0
    amp = k ** (-beta / 2.0)
    amp[0, 0] = 0.0
    spec = amp * (rng.normal(size=k.shape) + 1j * rng.normal(size=k.shape))
    f = np.fft.irfft2(spec, s=(n_rows, n_cols))
    return f - f.mean()


def fractal_dem(nrows: int, ncols: int, dxy: int, seed: int, relief: float = 3.0,
                n_depressions: int = 200, base: float = 100.0) -> np.ndarray:
    """Spectral fractal (P(k) ~ k^-3) rescaled to 0..relief m above base, with
    cosine-tapered circular depressions (radius log-uniform 5-40 m, depth
    U(0.2, 1.0) m); the large-domain and ensemble configurations' terrain."""
    rng = np.random.default_rng(seed)
    f = spectral_field(nrows, ncols, 3.0, rng)
    f = (f - f.min()) / max(f.max() - f.min(), 1e-12) * relief
    dem = base + f
    yy = (np.arange(nrows) + 0.5) * dxy
    xx = (np.arange(ncols) + 0.5) * dxy
    for _ in range(n_depressions):
        r = math.exp(rng.uniform(math.log(5.0), math.log(40.0)))
        d = rng.uniform(0.2, 1.0)
        cy = rng.uniform(0, nrows * dxy)
        cx = rng.uniform(0, ncols * dxy)
        i0, i1 = max(0, int((cy - r) / dxy) - 1), min(nrows, int((cy + r) / dxy) + 2)
        j0, j1 = max(0, int((cx - r) / dxy) - 1), min(ncols, int((cx + r) / dxy) + 2)
        if i0 >= i1 or j0 >= j1:
            continue
        dy = yy[i0:i1, None] - cy
        dx = xx[None, j0:j1] - cx
        rr = np.sqrt(dy * dy + dx * dx)
        taper = np.where(rr < r, 0.5 * (1.0 + np.cos(np.pi * rr / r)), 0.0)
        dem[i0:i1, j0:j1] -= d * taper
    return dem.astype(np.float32)


def smooth_field(nrows: int, ncols: int, seed: int, lo: float, hi: float,
                 corr_cells: float = 64.0) -> np.ndarray:
    """Smooth random field (Gaussian-filtered noise) rescaled to [lo, hi]."""
    rng = np.random.default_rng(seed)
    noise = rng.normal(size=(nrows, ncols))
    kx = np.fft.fftfreq(nrows)[:, None]
    ky = np.fft.rfftfreq(ncols)[None, :]
    g = np.exp(-0.5 * (kx * kx + ky * ky) * (2 * np.pi * corr_cells / 2.0) ** 2)
    f = np.fft.irfft2(np.fft.rfft2(noise) * g, s=(nrows, ncols))
    f = (f - f.min()) / max(f.max() - f.min(), 1e-12)
    return lo + (hi - lo) * f


def plane_scenario(nrows: int = 200, ncols: int = 200, seed: int = 0) -> Scenario:
    """The small CPU-runnable configuration: 200x200 cells of 2 m, a plane
    sloping 0.01 with smoothed bumps, 20 mm/day snowmelt for 6 h carrying
    1 mg/L of solute, D = 0.01 m^2/s, output every 600 s. ROUGNESS_HEIGHT
    (the dry threshold) is 1 mm so 6 h of melt (5 mm) can wet the terrain."""
    return Scenario(name=f"plane{nrows}x{ncols}", dem=plane_dem(nrows, ncols, seed=seed), dxy=2,
                    meteo=((0.0, 20.0, 1.0), (21600.0, 20.0, 1.0)), horizon=21600.0,
                    print_step=600, ks=0.001, ade=True, d_coef=0.01)


def fractal_scenario(n: int, dxy: int = 2, seed: int = 1, melt_seed: int = 2,
                     extensions: bool = True, horizon: float = 86400.0) -> Scenario:
    """The large-domain configuration (n x n cells of dxy m, fractal terrain
    with depressions). With ``extensions`` it also carries a smooth melt
    field of 5-40 mm/day and Manning n ~ U[0.03, 0.15]; without, the melt is
    the field's mean, uniform in space."""
    dem = fractal_dem(n, n, dxy, seed)
    melt = smooth_field(n, n, melt_seed, 5.0, 40.0)
    mean_rate = float(melt.mean())
    sc = Scenario(name=f"fractal{n}", dem=dem, dxy=dxy,
                  meteo=((0.0, mean_rate, 1.0), (horizon, mean_rate, 1.0)), horizon=horizon,
                  print_step=3600, ks=0.001, ade=True, d_coef=0.01)
    if extensions:
        rng = np.random.default_rng(seed + 1000)
        sc.melt_mult = (melt / mean_rate).astype(np.float64)
        sc.manning = rng.uniform(0.03, 0.15, size=(n, n))
    return sc


def wet_start(sc: Scenario, depth: float = 0.05, seed: int = 7, fill_depressions: bool = True
              ) -> Scenario:
    """Give a scenario a wet initial state: a uniform film of ``depth`` plus,
    optionally, water ponded up to a smoothed level so depressions hold more."""
    rng = np.random.default_rng(seed)
    dem = sc.dem.astype(np.float64)
    h = np.full(dem.shape, depth)
    if fill_depressions:
        level = box3(box3(dem))
        h += np.maximum(level - dem, 0.0)
    h *= rng.uniform(0.8, 1.2, size=h.shape)
    sc.init_h = h
    sc.init_qx = np.zeros_like(h)
    sc.init_qy = np.zeros_like(h)
    sc.init_conc = [np.where(h > 2 * depth, 1.0, 0.0) for _ in range(sc.nchem)]
    return sc


def dambreak_scenario(n: int = 2048, dxy: int = 1, radius: float = 300.0, depth: float = 2.0,
                      base: float = 10.0, manning: float = 0.02, horizon: float = 600.0) -> Scenario:
    """Circular dam break on a flat bed: ``depth`` m of water inside ``radius``
    m of the centre, dry outside, uniform Manning n, no melt, two solutes
    (unit concentration inside the dam, D = 0.1 and 1.0 m^2/s). The bed sits
    at ``base`` m because a DEM value of 0 marks a wall cell."""
    dem = np.full((n, n), base, dtype=np.float32)
    c = (np.arange(n) + 0.5) * dxy - 0.5 * n * dxy
    rr = np.sqrt(c[:, None] ** 2 + c[None, :] ** 2)
    inside = rr < radius
    sc = Scenario(name=f"dambreak{n}", dem=dem, dxy=dxy, meteo=((0.0, 0.0, 0.0),), horizon=horizon,
                  print_step=int(horizon), ks=0.001, ade=True, d_coef=0.1, d_coefs=[0.1, 1.0])
    sc.manning = np.full((n, n), manning)
    sc.init_h = np.where(inside, depth, 0.0)
    sc.init_qx = np.zeros((n, n))
    sc.init_qy = np.zeros((n, n))
    sc.init_conc = [inside.astype(np.float64), inside.astype(np.float64)]
    sc.extra["radius"] = radius
    return sc


def forcing_table(sc: Scenario) -> np.ndarray:
    """The forcing table as read_meteo fills GlobVar::meteo (3 x 2000 float,
    rows from 1), with the guard and horizon rows of write_meteo."""
    tab = np.zeros((3, 2000), dtype=np.float32)
    rows = list(sc.meteo) + [(GUARD_TIME, 0.0, 0.0), (sc.horizon, 0.0, 0.0)]
    for a, (t, r, c) in enumerate(rows, start=1):
        tab[:, a] = (t, r, c)
    return tab


def inflow_table(sc: Scenario) -> np.ndarray:
    """The point-inflow table as read_inflow fills GlobVar::inflow (3 x 2000
    float, data from row 0, read_functions.cpp:307-313), with the guard and
    horizon rows of write_meteo."""
    tab = np.zeros((3, 2000), dtype=np.float32)
    rows = list(sc.inflow) + [(GUARD_TIME, 0.0, 0.0), (sc.horizon, 0.0, 0.0)]
    for a, (t, r, c) in enumerate(rows):
        tab[:, a] = (t, r, c)
    return tab


def inflow_cell(sc: Scenario) -> Tuple[int, int]:
    """(irow, icol) of the discharge location as read_geo computes it
    (read_functions.cpp:228-231): round(coordinate - corner) / dxy, stored in
    an unsigned long."""
    x, y = sc.inflow_xy
    irow = int(math.floor(round(float(int(y)) - float(sc.yll)) / float(sc.dxy)))
    icol = int(math.floor(round(float(int(x)) - float(sc.xll)) / float(sc.dxy)))
    return irow, icol


def full_grid(sc: Scenario, interior: np.ndarray, fill: float = 0.0) -> np.ndarray:
    """An interior (nrows, ncols) array as a GlobVar grid (ncols+2, nrows+2)."""
    g = np.full((sc.ncols + 2, sc.nrows + 2), fill)
    g[1:-1, 1:-1] = np.asarray(interior, dtype=np.float64).T
    return g


def make_domain(sc: Scenario, *, precision: str = "fp64", steps_in_flight: int = 8):
    """A GPU domain of the scenario without its files: the reference's
    initiation of the DEM (fx_initiate), the forcing, the extension grids and
    the scenario's wet start, if any."""
    import fluxos_cpp_b200 as fx
    d = fx.Domain(sc.nrows, sc.ncols, sc.dxy, nchem=sc.nchem, nodata=float(sc.nodata), hdry=sc.ks,
                  ntim=sc.horizon, print_step=sc.print_step, print_next=sc.print_step, ade=sc.ade,
                  h_min_print=float(sc.h_min_print),
                  d_coef=list(sc.d_coefs) if sc.d_coefs else [sc.d_coef],
                  steps_in_flight=steps_in_flight, precision=precision, wintra=sc.wintra,
                  soil_release_rate=sc.soil_release_rate)
    d.initiate(full_grid(sc, sc.dem.astype(np.float64)))
    d.set_forcing(forcing_table(sc))
    if sc.inflow is not None:
        d.set_inflow(inflow_table(sc), *inflow_cell(sc))
    if sc.melt_mult is not None:
        d.set_melt_field(full_grid(sc, sc.melt_mult, 1.0))
    if sc.manning is not None:
        d.set_manning(full_grid(sc, sc.manning, 0.0))
    if sc.init_h is not None:
        zb = d.download("zb")
        h = full_grid(sc, sc.init_h)
        d.upload("z", zb + h)
        d.upload("h", h)
        if sc.init_qx is not None:
            d.upload("qx", full_grid(sc, sc.init_qx))
        if sc.init_qy is not None:
            d.upload("qy", full_grid(sc, sc.init_qy))
        for k, c in enumerate(sc.init_conc or []):
            d.upload("conc" if k == 0 else f"conc{k}", full_grid(sc, c))
        fl = d.download_flags()
        ld = full_grid(sc, np.where(sc.init_h > sc.ks, 0.0, 1.0))
        d.upload_flags(ld, fl["wall"])
    if sc.init_soil is not None:
        d.upload("soil_mass", full_grid(sc, sc.init_soil))
    d.prepare()
    return d


def ensemble_scenarios(count: int = 64, seed: int = 3, n_min: int = 256, n_max: int = 2048,
                       dxy: int = 2, horizon: float = 21600.0, wet: bool = True) -> List[Scenario]:
    """The batched-ensemble configuration: `count` square grids with sizes
    log-uniform in [n_min, n_max] (seeded), each with its own fractal DEM as
    in the large-domain configuration, a uniform melt rate U[5, 50] mm/day,
    Manning n U[0.03, 0.15] per cell, one solute, a 6 h horizon and (with
    `wet`) the wet start of wet_start."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(n_min), math.log(n_max), size=count)).round().astype(int)
    rates = rng.uniform(5.0, 50.0, size=count)
    seeds = rng.integers(0, 2**31 - 1, size=count)
    out = []
    for i in range(count):
        n, s = int(sizes[i]), int(seeds[i])
        sc = Scenario(name=f"ens{i}_{n}", dem=fractal_dem(n, n, dxy, s), dxy=dxy,
                      meteo=((0.0, float(rates[i]), 1.0), (horizon, float(rates[i]), 1.0)),
                      horizon=horizon, print_step=3600, ks=0.001, ade=True, d_coef=0.01)
        sc.manning = np.random.default_rng(s + 1).uniform(0.03, 0.15, size=(n, n))
        if wet:
            wet_start(sc, depth=0.005, seed=s + 2)
        out.append(sc)
    return out

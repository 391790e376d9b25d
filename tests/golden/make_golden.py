"""Regenerate the golden fixtures in this folder from the FLUXOS reference.

Run from the repository root where the reference tree is mounted:

    make -C oracle all REF=<FLUXOS_cpp tree> && python tests/golden/make_golden.py [case ...]

Each case is a small seeded scenario. Its input files are written exactly as
the reference reads them, and the reference sources compiled in
oracle/_ref/ are stepped through the harness (oracle/ref_harness.cpp). State
snapshots are saved at the listed step counts. Two cases also keep the
Results/<t>.txt files that the whole reference program (oracle/_ref/fluxos_ref)
writes. The fixtures hold the input text, so tests need neither the reference
nor this script.

The case ``c1_plane200`` is the small CPU configuration run in full by the
reference program: 200 x 200 cells of 2 m, a plane sloping 0.01 with smoothed
Gaussian bumps (seed 0), dry start, 20 mm/day of melt at 1 mg/L for 6 h,
D = 0.01 m^2/s, output every 600 s (36 Results files). Its 124 MB of text is
kept as digests (tests/results_digest.py: SHA-256, row set, wet-cell count,
column sums, sample rows) plus every value of the files at 10,200 s and
21,600 s, and the SHA-256 of the input files, which
scenarios.plane_scenario() regenerates.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from fluxos_cpp_b200 import scenarios as S  # noqa: E402
import pyoracle as P  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
SNAP_GRIDS = ("z", "h", "qx", "qy", "conc", "fe_1", "fe_2", "fe_3", "fn_1", "fn_2", "fn_3",
              "twet", "h0", "ldry", "ldry_prev", "zb", "wall", "ks", "soil_mass")


def case_plane_walls() -> dict:
    sc = S.plane_scenario(24, 20, seed=0)
    sc.horizon = 6000.0
    sc.meteo = ((0.0, 40.0, 1.0), (6000.0, 40.0, 1.0))
    sc.dem[3:6, 4] = -9999.0
    sc.dem[10, 2:9] = 0.0
    return dict(sc=sc, wet=None, steps=(1, 100, 1000, 5000), mode=0, results=True)


def _patch(nr, nc, seed):
    rng = np.random.default_rng(seed)
    h = np.where(rng.random((nr, nc)) < 0.6, rng.uniform(0, 0.05, (nr, nc)), 0.0)
    qx = rng.normal(0, 0.002, (nr, nc)) * (h > 0)
    qy = rng.normal(0, 0.002, (nr, nc)) * (h > 0)
    c = rng.uniform(0, 2, (nr, nc)) * (h > 0)
    return dict(h=h, qx=qx, qy=qy, conc=[c])


def case_patchwork(mode: int) -> dict:
    sc = S.plane_scenario(24, 20, seed=1)
    sc.horizon = 3000.0
    sc.dem[6, 3:7] = -9999.0
    return dict(sc=sc, wet=_patch(24, 20, 3), steps=(1, 10, 100, 300), mode=mode, results=False)


def case_dambreak() -> dict:
    nr, nc = 32, 28
    dem = np.full((nr, nc), 100.0, dtype=np.float32)
    sc = S.Scenario(name="dambreak", dem=dem, dxy=1, meteo=((0.0, 0.0, 0.0), (600.0, 0.0, 0.0)),
                    horizon=600.0, print_step=60, ks=0.001, ade=True, d_coef=0.1)
    yy, xx = np.mgrid[0:nr, 0:nc]
    r = np.hypot(yy - nr / 2 + 0.5, xx - nc / 2 + 0.5)
    h = np.where(r < 8.0, 0.5, 0.0)
    return dict(sc=sc, wet=dict(h=h, qx=np.zeros_like(h), qy=np.zeros_like(h),
                                conc=[np.where(r < 8.0, 1.0, 0.0)]),
                steps=(1, 20, 200), mode=0, results=False)


def case_inflow() -> dict:
    """A point inflow (INFLOW_FILE) on a dry plane under melt: three discharge
    rows with their own concentrations, then none."""
    sc = S.plane_scenario(24, 20, seed=2)
    sc.horizon = 4000.0
    sc.meteo = ((0.0, 20.0, 1.0), (4000.0, 20.0, 1.0))
    sc.inflow = ((0.0, 0.02, 5.0), (300.0, 0.05, 2.0), (900.0, 0.01, 0.5), (1500.0, 0.0, 0.0))
    sc.inflow_xy = (24, 32)  # icol 12, irow 16 at dxy 2
    sc.dem[8, 3:9] = -9999.0
    return dict(sc=sc, wet=None, steps=(1, 10, 200, 2000), mode=0, results=True)


def case_wintra() -> dict:
    """The WINTRA soil release (EXTERNAL_MODULES.WINTRA) on a wet patchwork
    under melt, with a seeded soil mass per cell (what a restart file's
    soil_mass column would hold)."""
    sc = S.plane_scenario(24, 20, seed=4)
    sc.horizon = 3000.0
    sc.wintra = True
    sc.soil_release_rate = 0.8
    sc.dem[5, 2:6] = -9999.0
    rng = np.random.default_rng(11)
    soil = rng.uniform(0.0, 50.0, (24, 20)) * (rng.random((24, 20)) < 0.7)
    return dict(sc=sc, wet=_patch(24, 20, 5), soil=soil, steps=(1, 10, 100, 400), mode=0, results=False)


def case_inflow_wintra() -> dict:
    """Point inflow, melt and the WINTRA soil release in the same steps, on a
    wet patchwork with walls (the inflow's dilution and the soil release
    both change the inflow cell's concentration)."""
    sc = S.plane_scenario(24, 20, seed=5)
    sc.horizon = 3000.0
    sc.wintra = True
    sc.soil_release_rate = 1.0
    sc.inflow = ((0.0, 0.01, 3.0), (100.0, 0.03, 0.5), (250.0, 0.0, 0.0))
    sc.inflow_xy = (20, 24)  # icol 10, irow 12 at dxy 2
    sc.dem[3, 5:9] = -9999.0
    rng = np.random.default_rng(13)
    soil = rng.uniform(0.0, 30.0, (24, 20))
    return dict(sc=sc, wet=_patch(24, 20, 7), soil=soil, steps=(1, 10, 100, 400), mode=0, results=False)


CASES = {
    "plane_walls": case_plane_walls,
    "patchwork_weir": lambda: case_patchwork(0),
    "patchwork_closed": lambda: case_patchwork(1),
    "dambreak": case_dambreak,
    "inflow": case_inflow,
    "wintra": case_wintra,
    "inflow_wintra": case_inflow_wintra,
}


def build_case(name: str, spec: dict) -> None:
    sc, mode = spec["sc"], spec["mode"]
    work = tempfile.mkdtemp(prefix=f"golden_{name}_")
    modset = sc.write(work)
    out = {}
    with open(os.path.join(work, "dem.asc")) as f:
        out["dem_asc"] = np.array(f.read())
    with open(os.path.join(work, "meteo.csv")) as f:
        out["meteo_csv"] = np.array(f.read())
    meta = dict(name=name, nrows=sc.nrows, ncols=sc.ncols, dxy=sc.dxy, nodata=sc.nodata,
                print_step=sc.print_step, ks=sc.ks, ade=sc.ade, d_coef=sc.d_coef,
                h_min_print=sc.h_min_print, volrat_mode=mode, steps=list(spec["steps"]),
                wet=spec["wet"] is not None, wintra=bool(sc.wintra),
                soil_release_rate=float(sc.soil_release_rate))
    if sc.inflow is not None:
        with open(os.path.join(work, "inflow.csv")) as f:
            out["inflow_csv"] = np.array(f.read())
        meta["inflow"] = [list(r) for r in sc.inflow]
        meta["inflow_xy"] = list(sc.inflow_xy)
    ref = P.RefRun(modset, sc, mode)
    if spec["wet"] is not None:
        w = spec["wet"]
        ref.apply_wet_start(w["h"], w["qx"], w["qy"], w["conc"])
        for k in ("h", "qx", "qy"):
            out[f"wet_{k}"] = w[k]
        out["wet_conc0"] = w["conc"][0]
    if spec.get("soil") is not None:
        ref.interior("soil_mass")[...] = spec["soil"].T
        out["soil0"] = spec["soil"]
    done = 0
    scal = {}
    for target in spec["steps"]:
        while done < target:
            ref.step()
            if ref.print_due():
                ref.print_done()
            done += 1
        for g in SNAP_GRIDS:
            out[f"s{target}_{g}"] = ref.grid(g).copy()
        scal[str(target)] = {k: ref.scalar(k) for k in ("tim", "dtfl", "it", "hpall", "print_next")}
    meta["scalars"] = scal
    if spec["results"]:
        work2 = tempfile.mkdtemp(prefix=f"golden_{name}_main_")
        modset2 = sc.write(work2)
        r = subprocess.run([P.REF_BIN, modset2], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(r.stderr)
        res = os.path.join(work2, "Results")
        files = sorted(os.listdir(res), key=lambda s: int(s.split(".")[0]))
        meta["results"] = files
        for fn in files:
            with open(os.path.join(res, fn)) as f:
                out[f"results_{fn}"] = np.array(f.read())
    out["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(name, "snapshots", spec["steps"], "results" if spec["results"] else "")


C1_FULL = ("10200.txt", "21600.txt")


def build_c1() -> None:
    """The small CPU configuration through the whole reference program."""
    import hashlib
    sys.path.insert(0, os.path.dirname(HERE))
    import results_digest as RD
    sc = S.plane_scenario()
    work = tempfile.mkdtemp(prefix="golden_c1_")
    modset = sc.write(work)
    r = subprocess.run([P.REF_BIN, modset], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stderr)
    res = os.path.join(work, "Results")
    files = sorted(os.listdir(res), key=lambda s: int(s.split(".")[0]))
    meta = dict(name="c1_plane200", nrows=sc.nrows, ncols=sc.ncols, dxy=sc.dxy, ks=sc.ks,
                horizon=sc.horizon, print_step=sc.print_step, results=files, full=list(C1_FULL),
                inputs={})
    for fn in ("dem.asc", "meteo.csv"):
        with open(os.path.join(work, fn), "rb") as f:
            meta["inputs"][fn] = hashlib.sha256(f.read()).hexdigest()
    out = {}
    meta["digest"] = {}
    for k, fn in enumerate(files):
        with open(os.path.join(res, fn)) as f:
            text = f.read()
        dg = RD.digest(text, sc.nrows, sc.ncols, seed=k, hdry=sc.ks)
        meta["digest"][fn] = {"sha256": dg["sha256"], "header": dg["header"], "rows": dg["rows"],
                              "wet": dg["wet"]}
        t = fn.split(".")[0]
        out[f"mask_{t}"] = dg["mask"]
        out[f"sums_{t}"] = dg["sums"]
        out[f"samples_{t}"] = dg["samples"]
        if fn in C1_FULL:
            out[f"full_{t}"] = RD.full_columns(text)
    out["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(os.path.join(HERE, "c1_plane200.npz"), **out)
    print("c1_plane200", len(files), "Results files")


def main() -> None:
    if not P.ref_available(0):
        sys.exit("oracle/_ref is not built: run `make -C oracle all REF=<FLUXOS_cpp tree>`")
    only = set(sys.argv[1:])
    for name, fn in CASES.items():
        if not only or name in only:
            build_case(name, fn())
    if not only or "c1_plane200" in only:
        build_c1()


if __name__ == "__main__":
    main()

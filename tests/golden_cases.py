"""Loader for the golden fixtures in tests/golden/ (see make_golden.py)."""
import json
import os

import numpy as np

from fluxos_cpp_b200 import scenarios as S

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ("plane_walls", "patchwork_weir", "patchwork_closed", "dambreak", "inflow", "wintra", "inflow_wintra")


def load(name: str):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    meta = json.loads(str(z["meta"]))
    return z, meta


def materialise(name: str, folder: str):
    """Write the case's input files into `folder`; return (scenario, z, meta, modset path)."""
    z, meta = load(name)
    os.makedirs(folder, exist_ok=True)
    with open(os.path.join(folder, "dem.asc"), "w") as f:
        f.write(str(z["dem_asc"]))
    with open(os.path.join(folder, "meteo.csv"), "w") as f:
        f.write(str(z["meteo_csv"]))
    sc = S.Scenario(name=name, dem=np.zeros((meta["nrows"], meta["ncols"]), dtype=np.float32),
                    dxy=meta["dxy"], nodata=meta["nodata"], print_step=meta["print_step"],
                    ks=meta["ks"], ade=meta["ade"], d_coef=meta["d_coef"],
                    h_min_print=meta["h_min_print"], wintra=meta.get("wintra", False),
                    soil_release_rate=meta.get("soil_release_rate", 0.0))
    modset = {
        "DEM_FILE": os.path.join(folder, "dem.asc"), "SIM_DATETIME_START": "2020JAN01 00:00:00",
        "RESTART": False, "METEO_FILE": os.path.join(folder, "meteo.csv"),
        "OUTPUT": {"OUTPUT_FOLDER": os.path.join(folder, "Results"),
                   "PRINT_STEP": meta["print_step"], "H_MIN_TO_PRINT": meta["h_min_print"]},
        "ROUGNESS_HEIGHT": meta["ks"], "SOIL_RELEASE_RATE": sc.soil_release_rate,
        "SOIL_CONC_BACKGROUND": 0.0,
        "EXTERNAL_MODULES": {"ADE_TRANSPORT": {"STATUS": meta["ade"], "D_COEF": meta["d_coef"]},
                             "OPENWQ": {"STATUS": False, "MASTERFILE_DIR": ""},
                             "WINTRA": {"STATUS": sc.wintra, "SWE_STD": 0.0, "SWE_MAX": 0.0}},
    }
    if "inflow_csv" in z.files:
        with open(os.path.join(folder, "inflow.csv"), "w") as f:
            f.write(str(z["inflow_csv"]))
        sc.inflow = [tuple(r) for r in meta["inflow"]]
        sc.inflow_xy = tuple(meta["inflow_xy"])
        modset["INFLOW_FILE"] = {"FILENAME": os.path.join(folder, "inflow.csv"),
                                 "DISCHARGE_LOCATION": {"X_COORDINATE": sc.inflow_xy[0],
                                                        "Y_COORDINATE": sc.inflow_xy[1]}}
    mp = os.path.join(folder, "modset.json")
    with open(mp, "w") as f:
        f.write("/* golden case */\n")
        json.dump(modset, f, indent=1)
    return sc, z, meta, mp


def wet_arrays(z):
    return dict(h=z["wet_h"], qx=z["wet_qx"], qy=z["wet_qy"], conc=[z["wet_conc0"]])


def apply_start(run, z, meta) -> None:
    """The case's wet start and seeded soil mass on an oracle run."""
    if meta["wet"]:
        w = wet_arrays(z)
        run.apply_wet_start(w["h"], w["qx"], w["qy"], w["conc"])
    if "soil0" in z.files:
        run.interior("soil_mass")[...] = z["soil0"].T

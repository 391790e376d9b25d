"""The product's host C++ file surface (modset / DEM / forcing readers,
initiation, restart, Results writer) against the oracle, without a GPU."""
import json
import os

import numpy as np
import pytest

import fluxos_cpp_b200 as fx
import golden_cases as G
import pyoracle as P
from fluxos_cpp_b200 import scenarios as S


@pytest.mark.parametrize("case", G.CASES)
def test_load_modset_matches_oracle_startup(case, tmp_path):
    sc, z, meta, mp = G.materialise(case, str(tmp_path))
    st = fx.load_modset(mp)
    ora = P.OracleRun(str(tmp_path), sc, 0)
    for k in ("zb", "z", "h", "qx", "qy", "twet", "conc"):
        assert np.array_equal(st[k], ora.grid(k)), k
    assert np.array_equal(st["ldry"], ora.grid("ldry"))
    assert np.array_equal(st["wall"], ora.grid("wall"))
    assert np.array_equal(st["meteo"], ora.fgrid("meteo"))
    p = st["params"]
    assert p["hdry"] == ora.scalar("hdry")
    assert p["ntim"] == ora.scalar("ntim")
    assert p["print_next"] == ora.scalar("print_next")
    assert st["grid"]["dxy"] == sc.dxy and st["grid"]["nodata"] == sc.nodata
    # the golden bed (zb) and walls were produced by the reference's readers
    first = meta["steps"][0]
    assert np.array_equal(st["zb"], z[f"s{first}_zb"])
    assert np.array_equal(st["wall"], z[f"s{first}_wall"])


def test_modset_comments_and_truncations(tmp_path):
    sc = S.plane_scenario(6, 5)
    mp = sc.write(str(tmp_path))
    text = open(mp).read()
    text = text.replace('"PRINT_STEP": 600,', '/* block */ "PRINT_STEP": 600.9, // trailing')
    text = text.replace('"H_MIN_TO_PRINT": 0.0', '"H_MIN_TO_PRINT": 0.005')
    open(mp, "w").write(text)
    st = fx.load_modset(mp)
    assert st["params"]["print_step"] == 600.0  # unsigned long (GlobVar.h:102)
    assert st["params"]["h_min_print"] == 0.0   # 0.005 -> 0
    assert st["params"]["hdry"] == 0.001


def test_missing_forcing_is_an_error(tmp_path):
    sc = S.plane_scenario(6, 5)
    mp = sc.write(str(tmp_path))
    m = json.loads(open(mp).read().split("\n", 1)[1])
    del m["METEO_FILE"]
    open(mp, "w").write(json.dumps(m))
    with pytest.raises(fx.FluxosError) as e:
        fx.load_modset(mp)
    assert "METEO_FILE or INFLOW_FILE" in str(e.value)


def _inflow_modset(tmp_path, xy, meteo=True, horizon=3000.0):
    sc = S.plane_scenario(12, 10)
    sc.horizon = horizon
    sc.inflow = ((0.0, 0.01, 1.0), (1200.0, 0.0, 0.0))
    sc.inflow_xy = xy
    mp = sc.write(str(tmp_path))
    if not meteo:
        m = json.loads(open(mp).read().split("\n", 1)[1])
        del m["METEO_FILE"]
        open(mp, "w").write(json.dumps(m))
    return sc, mp


def test_inflow_only_modset_takes_ntim_from_the_inflow_file(tmp_path):
    """INFLOW_FILE alone is enough (read_functions.cpp:74-95); ntim is the
    inflow file's last time as read_inflow returns it (main.cpp:184-192)."""
    sc, mp = _inflow_modset(tmp_path, (4, 6), meteo=False, horizon=2500.5)
    st = fx.load_modset(mp)
    assert st["has_meteo"] == 0
    assert st["params"]["ntim"] == 2500.0
    assert not st["meteo"].any()
    if P.ref_available(0):
        ref = P.RefRun(mp, sc, 0)
        assert ref.scalar("ntim") == st["params"]["ntim"]
        assert ref.scalar("has_inflow") == 1.0
        assert (ref.scalar("inflow_nrow"), ref.scalar("inflow_ncol")) == S.inflow_cell(sc) == (3, 2)


@pytest.mark.parametrize("xy", [(0, 0), (4, 60), (40, 6), (4, 1)])
def test_inflow_location_off_the_interior_is_an_error(xy, tmp_path):
    """Both coordinates 0 leave the reference's cell unset, and a cell off
    the DEM's interior would be indexed outside the grid: both refused."""
    _, mp = _inflow_modset(tmp_path, xy)
    with pytest.raises(fx.FluxosError) as e:
        fx.load_modset(mp)
    assert "DISCHARGE_LOCATION" in str(e.value)


def test_restart_reads_newest_results_file(tmp_path):
    sc = S.plane_scenario(8, 7)
    mp = sc.write(str(tmp_path))
    m = json.loads(open(mp).read().split("\n", 1)[1])
    m["RESTART"] = True
    m["SOIL_CONC_BACKGROUND"] = 3.5
    open(mp, "w").write(json.dumps(m))
    res = os.path.join(str(tmp_path), "Results")
    os.makedirs(res)
    st0 = fx.load_modset(mp)  # no file yet: zero state, print_next = 0 + 600
    assert st0["params"]["print_next"] == 600.0
    assert not st0["soil_mass"].any()  # initiate.cpp:177 without a file
    zb = st0["zb"]
    rows = ["h"] + [",".join(["3", "4", "0", "0", repr(float(zb[4, 3]) + 0.25), "0.25", "0", "0", "0.5", "-0.5",
                              "0", "2.0", "4.25", "0", "0", "7.5"])]
    open(os.path.join(res, "1200.txt"), "w").write("\n".join(rows) + "\n")
    open(os.path.join(res, "600.txt"), "w").write("h\n")
    st = fx.load_modset(mp)
    assert st["params"]["print_next"] == 1800.0
    assert st["z"][4, 3] == zb[4, 3] + 0.25 and st["h"][4, 3] == 0.25
    assert st["qx"][4, 3] == 0.5 and st["qy"][4, 3] == -0.5
    assert st["conc"][4, 3] == 2.0 and st["twet"][4, 3] == 7.5
    assert st["ldry"][4, 3] == 0.0 and st["ldry"][4, 4] == 1.0
    # soil mass: the file's column 12, SOIL_CONC_BACKGROUND on the other
    # interior cells (initiate.cpp:93-107,152), 0 on the ghost ring
    soil = st["soil_mass"]
    assert soil[4, 3] == 4.25 and soil[1, 1] == 3.5 and soil[0, 0] == 0.0
    assert np.all(soil[1:-1, 1:-1][np.abs(zb[1:-1, 1:-1]) != 99999] > 0)


def test_wintra_settings_are_read(tmp_path):
    """SOIL_RELEASE_RATE and EXTERNAL_MODULES.WINTRA.STATUS (read_functions.cpp:46,65);
    WINTRA is switched off without the ADE module (main.cpp:209-213)."""
    sc = S.plane_scenario(6, 5)
    sc.wintra, sc.soil_release_rate = True, 0.25
    st = fx.load_modset(sc.write(str(tmp_path / "a")))
    assert st["params"]["wintra"] == 1 and st["params"]["soil_release_rate"] == 0.25
    sc.ade = False
    st = fx.load_modset(sc.write(str(tmp_path / "b")))
    assert st["params"]["wintra"] == 0


def test_results_writer_soil_mass_column(tmp_path):
    sc = S.plane_scenario(5, 4)
    grids = {k: np.zeros((6, 7)) for k in ("z", "h", "qx", "qy", "conc", "fe_1", "fn_1", "twet")}
    grids["zb"] = np.full((6, 7), 10.0)
    grids["h"][2, 3] = 0.5
    grids["z"] = grids["zb"] + grids["h"]
    grids["soil_mass"] = np.zeros((6, 7))
    grids["soil_mass"][2, 3] = 12.125
    fn = str(tmp_path / "600.txt")
    fx.write_results_host(fn, 5, 4, 2, 0.0, 0.0, 0.0, grids)
    rows = open(fn).read().strip().split("\n")
    assert len(rows) == 2
    v = [float(x) for x in rows[1].split(",")]
    assert (v[0], v[1], v[12]) == (3.0, 2.0, 12.125)


def test_results_writer_empty_domain_writes_one_zero_row(tmp_path):
    n = (5 + 2) * (4 + 2)
    zeros = np.zeros((6, 7))
    grids = {k: zeros for k in ("z", "zb", "h", "qx", "qy", "conc", "fe_1", "fn_1", "twet")}
    fn = str(tmp_path / "0.txt")
    fx.write_results_host(fn, 5, 4, 2, 0.0, 0.0, 0.0, grids)
    lines = open(fn).read().splitlines()
    assert len(lines) == 2 and lines[1] == ",".join(["0"] * 16)
    assert n == 42

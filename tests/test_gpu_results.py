"""The Results files written from the device (fx_write_results and
fx_write_results_async: rows compacted on the GPU, formatted on host
threads) against the host writer on downloaded grids, which itself matches
the reference program's files byte for byte (test_oracle_golden.py)."""
import os

import numpy as np
import pytest

import fluxos_cpp_b200 as fx
from fluxos_cpp_b200 import scenarios as S

pytestmark = pytest.mark.gpu

GRIDS = ("z", "zb", "h", "qx", "qy", "conc", "soil_mass", "fe_1", "fn_1", "twet")


def _host_file(d, path):
    g = {k: d.download(k) for k in GRIDS}
    fx.write_results_host(path, d.nrows, d.ncols, d.dxy, d.xll, d.yll, d.h_min_print, g)
    with open(path) as f:
        return f.read()


def _domain(precision, n=150, seed=3, h_min_print=0.0):
    sc = S.fractal_scenario(n, dxy=2, seed=seed, melt_seed=seed + 1, extensions=True)
    S.wet_start(sc, depth=0.005, seed=seed + 2)
    sc.wintra, sc.soil_release_rate = True, 0.5
    sc.init_soil = np.random.default_rng(seed).uniform(0.0, 10.0, (n, n))
    sc.h_min_print = h_min_print
    return S.make_domain(sc, precision=precision, steps_in_flight=8)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_device_rows_match_host_writer(precision, tmp_path):
    d = _domain(precision)
    for n in (0, 17, 40):
        d.step(n)
        a, b = str(tmp_path / f"dev{n}.txt"), str(tmp_path / f"host{n}.txt")
        d.write_results(a)
        with open(a) as f:
            got = f.read()
        want = _host_file(d, b)
        assert got == want, (precision, n)
        assert got.count("\n") > 1000
    d.close()


def test_threshold_zero_bed_and_empty_selection(tmp_path):
    """H_MIN_TO_PRINT drops shallow cells, zb == 0 cells are never printed,
    and a selection with no cell writes one row of zeros."""
    sc = S.dambreak_scenario(96, dxy=1, radius=20.0, depth=2.0, horizon=60.0)
    sc.h_min_print = 1
    d = S.make_domain(sc, precision="fp64")
    zb = d.download("zb")
    zb[40:44, 40:50] = 0.0
    d.upload("zb", zb)
    d.prepare()
    d.step(5)
    a = str(tmp_path / "a.txt")
    d.write_results(a)
    got = open(a).read()
    assert got == _host_file(d, str(tmp_path / "b.txt"))
    rows = got.strip().split("\n")[1:]
    assert 0 < len(rows) < 96 * 96
    assert all(float(r.split(",")[5]) > 1.0 for r in rows)
    d.close()
    dry = fx.Domain(20, 30, 2, ntim=100.0)
    dry.initiate(np.full((32, 22), 50.0))
    dry.write_results(a)
    assert open(a).read().split("\n")[1] == ",".join(["0"] * 16)
    dry.close()


def test_async_files_are_the_state_when_started(tmp_path):
    """Files started with wait=False hold the state at the call, while the
    domain keeps stepping; three files in flight reuse the two buffers."""
    d = _domain("fp32", n=200, seed=5)
    want = []
    for k in range(3):
        d.step(13)
        want.append(_host_file(d, str(tmp_path / f"host{k}.txt")))
        d.write_results(str(tmp_path / f"dev{k}.txt"), wait=False)
    d.step(20)
    d.results_wait()
    for k in range(3):
        with open(tmp_path / f"dev{k}.txt") as f:
            assert f.read() == want[k], k
    with pytest.raises(fx.FluxosError):
        d.write_results(str(tmp_path / "missing_dir" / "x.txt"), wait=False)
        d.results_wait()
    d.close()


def test_program_writes_while_stepping(tmp_path):
    """fluxos_gpu's loop (fx_run) starts each file and steps on; every file
    is complete when the run returns."""
    sc = S.plane_scenario(40, 30, seed=2)
    sc.horizon = 3000.0
    sc.meteo = ((0.0, 200.0, 1.0), (3000.0, 200.0, 1.0))
    mp = sc.write(str(tmp_path))
    fx.run(mp)
    files = sorted(os.listdir(tmp_path / "Results"), key=lambda s: int(s.split(".")[0]))
    assert files[:5] == [f"{t}.txt" for t in range(600, 3001, 600)]
    for fn in files:
        lines = open(tmp_path / "Results" / fn).read().split("\n")
        assert lines[-1] == "" and len(lines) > 3

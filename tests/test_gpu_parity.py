"""The CUDA path (through the C ABI) against the oracle: per-cell relative
error <= 1e-10 on every state grid (h, z, qx, qy, conc and the face fluxes),
identical wet/dry flags and clock, after the stated step counts.

The tolerance is 1e-10 relative per cell, floored at 1e-6 of the field's
largest magnitude. Arithmetic is FP64 in the same order as the reference, so
most runs are bit-identical; the edge weir's pow(h, 1.5) is evaluated
correctly rounded on the GPU where glibc's pow is off by one unit in the last
place for about 1e-3 of arguments."""
import numpy as np
import pytest

import fluxos_cpp_b200 as fx
import golden_cases as G
import gpu_pairs as GP
import pyoracle as P
from fluxos_cpp_b200 import scenarios as S

pytestmark = pytest.mark.gpu


def _pair_from_case(case, tmp_path, store_all=True):
    sc, z, meta, _ = G.materialise(case, str(tmp_path))
    ora = P.OracleRun(str(tmp_path), sc, meta["volrat_mode"])
    G.apply_start(ora, z, meta)
    d = GP.domain_from_oracle(ora, sc, meta["volrat_mode"], store_all)
    return sc, z, meta, ora, d


@pytest.mark.parametrize("case", G.CASES)
def test_golden_cases_step_parity(case, tmp_path):
    sc, z, meta, ora, d = _pair_from_case(case, tmp_path)
    done = 0
    for target in meta["steps"]:
        GP.advance_oracle(ora, target - done)
        GP.advance_domain(d, target - done)
        done = target
        res, bad = GP.compare(ora, d, sc)
        assert not bad, (case, target, bad)
        # and the GPU state against the reference's own snapshot
        h_ref = z[f"s{target}_h"][1:-1, 1:-1]
        assert GP.rel_err(h_ref, d.download("h")[1:-1, 1:-1], 1e-6 * np.abs(h_ref).max()) <= 1e-10
    d.close()


def _random_scenario(nr, nc, seed, walls=True):
    sc = S.plane_scenario(nr, nc, seed=seed)
    sc.horizon = 1e5
    if walls:
        rng = np.random.default_rng(seed)
        for _ in range(max(1, nr * nc // 400)):
            i, j = rng.integers(1, nr - 1), rng.integers(1, nc - 1)
            sc.dem[i, j] = -9999.0 if rng.random() < 0.5 else 0.0
    return sc


@pytest.mark.parametrize("nr,nc,seed,mode", [(97, 75, 11, 0), (64, 130, 12, 1), (150, 33, 13, 0)])
def test_random_patchwork_parity(nr, nc, seed, mode, tmp_path):
    """Ragged sizes (not multiples of the tile or strip), walls, wet/dry
    patchwork, both edge modes: 400 steps."""
    sc = _random_scenario(nr, nc, seed)
    sc.write(str(tmp_path))
    ora = P.OracleRun(str(tmp_path), sc, mode)
    rng = np.random.default_rng(seed + 1)
    h = np.where(rng.random((nr, nc)) < 0.7, rng.uniform(0, 0.05, (nr, nc)), 0.0)
    qx = rng.normal(0, 0.002, (nr, nc)) * (h > 0)
    qy = rng.normal(0, 0.002, (nr, nc)) * (h > 0)
    c = rng.uniform(0, 2, (nr, nc)) * (h > 0)
    ora.apply_wet_start(h, qx, qy, [c])
    d = GP.domain_from_oracle(ora, sc, mode)
    for n in (1, 10, 100, 289):
        GP.advance_oracle(ora, n)
        GP.advance_domain(d, n)
        res, bad = GP.compare(ora, d, sc)
        assert not bad, (n, bad)
    d.close()


@pytest.mark.parametrize("tile_rows", [8, 16])
def test_many_waves_of_tiles_parity(tile_rows, tmp_path):
    """A grid with far more tiles than the GPU holds at once (a 1,000 x 700
    grid is 33 x 117 tiles of 31 x 7 cells): tiles that start after their
    neighbours have finished must still read the neighbours' state from
    before the step. 40 steps against the oracle."""
    nr, nc, seed = 1000, 700, 17
    sc = _random_scenario(nr, nc, seed)
    sc.write(str(tmp_path))
    ora = P.OracleRun(str(tmp_path), sc, 0)
    rng = np.random.default_rng(seed + 1)
    h = np.where(rng.random((nr, nc)) < 0.8, rng.uniform(0, 0.2, (nr, nc)), 0.0)
    qx = rng.normal(0, 0.01, (nr, nc)) * (h > 0)
    qy = rng.normal(0, 0.01, (nr, nc)) * (h > 0)
    ora.apply_wet_start(h, qx, qy, [np.where(h > 0.1, 1.0, 0.0)])
    d = GP.domain_from_oracle(ora, sc, 0)
    d.set_option("tile_rows", tile_rows)
    for n in (3, 37):
        GP.advance_oracle(ora, n)
        GP.advance_domain(d, n)
        res, bad = GP.compare(ora, d, sc)
        assert not bad, (n, bad)
    d.close()


def test_flux_store_skipping_changes_nothing(tmp_path):
    """Skipping the fe_2/fe_3/fn_2/fn_3 stores of cells that end a step wet
    gives the same state as storing every flux."""
    nr, nc = 70, 61
    sc = _random_scenario(nr, nc, 21)
    sc.write(str(tmp_path))
    ora = P.OracleRun(str(tmp_path), sc, 0)
    rng = np.random.default_rng(5)
    h = np.where(rng.random((nr, nc)) < 0.5, rng.uniform(0, 0.03, (nr, nc)), 0.0)
    ora.apply_wet_start(h, None, None, [h * 10])
    a = GP.domain_from_oracle(ora, sc, 0, store_all=True)
    b = GP.domain_from_oracle(ora, sc, 0, store_all=False)
    GP.advance_domain(a, 300)
    GP.advance_domain(b, 300)
    for k in ("z", "h", "qx", "qy", "conc", "fe_1", "fn_1", "twet", "h0"):
        assert np.array_equal(a.download(k), b.download(k)), k
    assert np.array_equal(a.download_flags()["ldry"], b.download_flags()["ldry"])


@pytest.mark.parametrize("in_flight", [1, 3, 8])
def test_dry_start_melt_transition(in_flight, tmp_path):
    """Initially dry domain: Courant-only steps of a whole print interval,
    melt until the dry threshold is passed, then the solver switches on
    (the add_meteo ldry quirk and the it == 1 ADE skip are on this path).
    Outputs fall inside batches of ADE steps in flight, for several batch
    sizes."""
    sc = S.plane_scenario(48, 40, seed=3)
    sc.meteo = ((0.0, 80.0, 1.0), (3000.0, 80.0, 1.0))
    sc.horizon = 3000.0
    sc.write(str(tmp_path))
    ora = P.OracleRun(str(tmp_path), sc, 0)
    d = GP.domain_from_oracle(ora, sc, 0, steps_in_flight=in_flight)
    for n in (1, 2, 3, 50, 400, 2000):
        GP.advance_oracle(ora, n)
        GP.advance_domain(d, n)
        res, bad = GP.compare(ora, d, sc)
        assert not bad, (n, bad)
    d.close()


def test_extensions_multi_solute_manning_melt_field(tmp_path):
    """Two solutes with their own D, per-cell Manning n and a melt field
    (extensions; the oracle is the project's FP64 restatement)."""
    nr, nc = 60, 52
    sc = _random_scenario(nr, nc, 31, walls=False)
    sc.d_coefs = [0.1, 1.0]
    rng = np.random.default_rng(9)
    sc.manning = rng.uniform(0.03, 0.15, (nr, nc))
    sc.melt_mult = rng.uniform(0.25, 2.0, (nr, nc))
    sc.write(str(tmp_path))
    ora = P.OracleRun(str(tmp_path), sc, 0)
    h = rng.uniform(0.0, 0.04, (nr, nc))
    ora.apply_wet_start(h, None, None, [np.where(h > 0.02, 1.0, 0.0), np.where(h > 0.01, 2.0, 0.0)])
    d = GP.domain_from_oracle(ora, sc, 0)
    for n in (1, 20, 200):
        GP.advance_oracle(ora, n)
        GP.advance_domain(d, n)
        res, bad = GP.compare(ora, d, sc, rtol=1e-9)
        assert not bad, (n, bad)
    d.close()


@pytest.mark.parametrize("tma,in_flight,cell", [(1, 8, (90, 70)), (0, 1, (90, 70)), (1, 31, (1, 1)),
                                                (0, 3, (150, 130))])
def test_point_inflow_parity(tma, in_flight, cell, tmp_path):
    """Point inflow (INFLOW_FILE, add_inflow) on a wet patchwork large enough
    for the TMA-staged kernel. A row applies until its own time (the first
    row later than the clock, common.cpp:306-312), so the discharge starts at
    40 s, changes rate and concentration at 80 s and stops at 150 s; the
    inflow cell sits inside the grid or in a corner."""
    nr, nc = 150, 130
    sc = _random_scenario(nr, nc, 41)
    irow, icol = cell
    plain = S.plane_scenario(nr, nc, seed=41).dem
    sc.dem[nr - irow, icol - 1] = plain[nr - irow, icol - 1]  # not a wall
    sc.inflow = ((0.0, 0.05, 4.0), (40.0, 0.0, 0.0), (80.0, 0.02, 1.0), (150.0, 0.08, 0.0))
    sc.inflow_xy = (icol * sc.dxy, irow * sc.dxy)
    sc.write(str(tmp_path))
    ora = P.OracleRun(str(tmp_path), sc, 0)
    assert S.inflow_cell(sc) == cell
    rng = np.random.default_rng(5)
    h = np.where(rng.random((nr, nc)) < 0.5, rng.uniform(0, 0.03, (nr, nc)), 0.0)
    ora.apply_wet_start(h, None, None, [np.where(h > 0.01, 1.0, 0.0)])
    d = GP.domain_from_oracle(ora, sc, 0, steps_in_flight=in_flight)
    d.set_option("tma", tma)
    for n in (1, 20, 150, 400, 500):
        GP.advance_oracle(ora, n)
        GP.advance_domain(d, n)
        res, bad = GP.compare(ora, d, sc)
        assert not bad, (n, bad)
    assert ora.scalar("tim") > 150.0  # every discharge row was used
    d.close()


@pytest.mark.parametrize("in_flight,nchem", [(8, 1), (31, 2), (1, 3)])
def test_wintra_soil_release_parity(in_flight, nchem, tmp_path):
    """The WINTRA soil release fused into the ADE sweep's store, with several
    steps in flight and one or more solutes (each solute's sweep replays the
    reference's per-solute sequence on its own copy of the soil mass)."""
    nr, nc = 150, 130
    sc = _random_scenario(nr, nc, 51)
    sc.wintra, sc.soil_release_rate = True, 2.0
    if nchem > 1:
        sc.d_coefs = [0.01 * (k + 1) for k in range(nchem)]
    sc.write(str(tmp_path))
    ora = P.OracleRun(str(tmp_path), sc, 0)
    rng = np.random.default_rng(8)
    h = np.where(rng.random((nr, nc)) < 0.6, rng.uniform(0, 0.03, (nr, nc)), 0.0)
    ora.apply_wet_start(h, None, None, [np.where(h > 0.01, 1.0 + k, 0.0) for k in range(nchem)])
    ora.interior("soil_mass")[...] = (rng.uniform(0, 100.0, (nr, nc)) * (rng.random((nr, nc)) < 0.8)).T
    d = GP.domain_from_oracle(ora, sc, 0, steps_in_flight=in_flight)
    soil0 = ora.grid("soil_mass").sum()
    for n in (1, 20, 150, 300):
        GP.advance_oracle(ora, n)
        GP.advance_domain(d, n)
        res, bad = GP.compare(ora, d, sc)
        assert not bad, (n, bad)
    assert ora.grid("soil_mass").sum() < 0.999 * soil0  # the release happened
    d.close()


def test_bounded_wait_timeout_reports_device_error(tmp_path):
    """Failure detection without a fault: with the ADE dependency waits held
    unsatisfied (option fail_ade_waits), the waits run out, the step returns
    FX_ERR_DEVICE with the status flag set, the context refuses to step on,
    and a new context on the same device runs normally."""
    sc = _random_scenario(120, 90, 61)
    sc.write(str(tmp_path))
    ora = P.OracleRun(str(tmp_path), sc, 0)
    h = np.random.default_rng(2).uniform(0, 0.02, (120, 90))
    ora.apply_wet_start(h, None, None, [np.where(h > 0.01, 1.0, 0.0)])
    d = GP.domain_from_oracle(ora, sc, 0, steps_in_flight=8)
    d.set_option("fail_ade_waits", 1)
    with pytest.raises(fx.FluxosError) as e:
        d.step(8)
    assert e.value.code == -5 and "bounded wait" in str(e.value)
    assert d.status()["device_error"] != 0
    with pytest.raises(fx.FluxosError):
        d.step(1)
    d.close()
    d2 = GP.domain_from_oracle(ora, sc, 0, steps_in_flight=8)
    GP.advance_oracle(ora, 20)
    GP.advance_domain(d2, 20)
    res, bad = GP.compare(ora, d2, sc)
    assert not bad, bad
    d2.close()

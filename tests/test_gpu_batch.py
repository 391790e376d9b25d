"""Batches of domains (fx_batch): uneven grid sizes, own forcing, own edge
mode and own output schedule per member, advanced by shared launches.

Each member must match its oracle within 1e-10 per cell (as in
test_gpu_parity.py) and be bit-identical to the same domain stepped alone."""
import numpy as np
import pytest

import fluxos_cpp_b200 as fx
import gpu_pairs as GP
import pyoracle as P
from fluxos_cpp_b200 import scenarios as S

pytestmark = pytest.mark.gpu


def _member(tmp, nr, nc, seed, mode, rate, d_coef):
    sc = S.plane_scenario(nr, nc, seed=seed)
    sc.meteo = ((0.0, rate, 1.0), (1e5, rate, 1.0))
    sc.horizon = 1e5
    sc.print_step = 300 + 10 * seed
    sc.d_coef = d_coef
    sc.dem[nr // 3, 2:nc // 2] = -9999.0
    sc.write(tmp)
    ora = P.OracleRun(tmp, sc, mode)
    rng = np.random.default_rng(seed)
    h = np.where(rng.random((nr, nc)) < 0.75, rng.uniform(0, 0.05, (nr, nc)), 0.0)
    ora.apply_wet_start(h, None, None, [np.where(h > 0.02, 1.0, 0.0)])
    return sc, ora


def _run_batch(b, n):
    """n steps of every member, acknowledging outputs as they fall due."""
    start = [m.status()["steps"] for m in b.members]
    while True:
        for m in b.members:
            if m.status()["print_pending"]:
                m.print_done()
        left = [n - (m.status()["steps"] - s0) for m, s0 in zip(b.members, start)]
        if max(left) <= 0:
            return
        b.step(min(l for l in left if l > 0))


def test_batch_members_match_oracle_and_standalone(tmp_path):
    specs = [(40, 33, 1, 0, 30.0, 0.01), (97, 75, 2, 1, 60.0, 0.1), (64, 130, 3, 0, 10.0, 1.0)]
    members, alone = [], []
    for i, sp in enumerate(specs):
        d = tmp_path / f"m{i}"
        d.mkdir()
        sc, ora = _member(str(d), *sp)
        members.append((sc, ora, GP.domain_from_oracle(ora, sc, sp[3], steps_in_flight=4)))
        alone.append(GP.domain_from_oracle(ora, sc, sp[3], steps_in_flight=4))
    b = fx.Batch()
    for _, _, dom in members:
        b.add(dom)
    for n in (1, 37, 250):
        _run_batch(b, n)
        for (sc, ora, dom), solo in zip(members, alone):
            GP.advance_oracle(ora, n)
            GP.advance_domain(solo, n)
            res, bad = GP.compare(ora, dom, sc)
            assert not bad, (sc.nrows, n, bad)
            for k in ("z", "h", "qx", "qy", "conc", "fe_1", "fn_1", "twet"):
                assert np.array_equal(dom.download(k), solo.download(k)), (sc.nrows, n, k)
    b.close()


def test_batch_admits_and_retires_between_steps(tmp_path):
    d1, d2 = tmp_path / "a", tmp_path / "b"
    d1.mkdir()
    d2.mkdir()
    sc1, o1 = _member(str(d1), 50, 44, 5, 0, 20.0, 0.01)
    sc2, o2 = _member(str(d2), 31, 90, 6, 0, 40.0, 0.01)
    m1 = GP.domain_from_oracle(o1, sc1, 0)
    m2 = GP.domain_from_oracle(o2, sc2, 0)
    b = fx.Batch()
    b.add(m1)
    _run_batch(b, 20)
    GP.advance_oracle(o1, 20)
    b.add(m2)  # admitted mid-run
    _run_batch(b, 30)
    GP.advance_oracle(o1, 30)
    GP.advance_oracle(o2, 30)
    b.remove(m1)  # retired
    _run_batch(b, 10)
    GP.advance_oracle(o2, 10)
    for sc, o, m in ((sc1, o1, m1), (sc2, o2, m2)):
        res, bad = GP.compare(o, m, sc)
        assert not bad, bad
    b.close()


def _fractal_wet(n, seed):
    sc = S.fractal_scenario(n, dxy=2, seed=seed, melt_seed=seed + 1, extensions=True)
    S.wet_start(sc, depth=0.005, seed=seed + 2)
    return sc


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_tile_shapes_staging_and_autotuner_keep_results(precision):
    sc = _fractal_wet(150, 11)
    ref = S.make_domain(sc, precision=precision, steps_in_flight=4)
    ref.step(40)
    want = {k: ref.download(k) for k in ("z", "h", "qx", "qy", "conc")}
    for r, tma in ((4, 1), (16, 1), (8, 0), (16, 0)):
        d = S.make_domain(sc, precision=precision, steps_in_flight=4)
        d.set_option("tile_rows", r)
        d.set_option("tma", tma)  # TMA-staged persistent kernel or one block per tile
        d.step(40)
        for k, v in want.items():
            assert np.array_equal(d.download(k), v), (r, tma, k)
        d.close()
    d = S.make_domain(sc, precision=precision, steps_in_flight=4)
    assert d.autotune(4) in (4, 8, 16)  # 3 shapes x 2 runs x 4 real steps
    assert d.status()["steps"] == 24
    d.step(40 - d.status()["steps"])
    assert d.status()["steps"] == 40
    for k, v in want.items():
        assert np.array_equal(d.download(k), v), ("autotuned", k)


def test_batch_autotuner_keeps_results():
    scs = [_fractal_wet(n, 20 + i) for i, n in enumerate((48, 96, 130))]
    b = fx.Batch()
    members = [S.make_domain(sc, precision="fp32", steps_in_flight=8) for sc in scs]
    for m in members:
        b.add(m)
    rows, k = b.autotune(4)
    assert rows in (4, 8, 16) and 1 <= k <= 8
    b.step(10)
    for sc, m in zip(scs, members):
        solo = S.make_domain(sc, precision="fp32", steps_in_flight=8)
        solo.step(m.status()["steps"])
        for key in ("z", "h", "qx", "conc"):
            assert np.array_equal(m.download(key), solo.download(key)), key
    b.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batch_staged_kernel_matches_per_tile_kernel_and_alone(precision):
    """The persistent TMA-staged batch kernel (blocks walking ranges of the
    packed tile table, each domain staged through its own tensor maps) and
    the one-block-per-tile batch kernel give identical states, equal to each
    domain stepped alone; one member is dry (no solver step, so no stage)
    while the others are wet."""
    scs = [_fractal_wet(n, 40 + i) for i, n in enumerate((61, 150, 96))]
    dry = S.plane_scenario(64, 70, seed=9)
    dry.horizon, dry.meteo = 1e5, ((0.0, 0.0, 0.0), (1e5, 0.0, 0.0))  # stays dry
    scs.append(dry)
    keys = ("z", "h", "qx", "qy", "conc", "fe_1", "fn_1", "twet")
    out = {}
    for tma in (1, 0):
        b = fx.Batch()
        b.set_option("tma", tma)
        b.set_option("tile_rows", 8)
        ms = [S.make_domain(sc, precision=precision, steps_in_flight=8) for sc in scs]
        for m in ms:
            b.add(m)
        _run_batch(b, 25)
        out[tma] = [{k: m.download(k) for k in keys} for m in ms]
        out[f"st{tma}"] = [m.status() for m in ms]
        b.close()
        for m in ms:
            m.close()
    assert out["st1"][-1]["hpall"] == 0  # the dry member has not run the solver
    for i, sc in enumerate(scs):
        solo = S.make_domain(sc, precision=precision, steps_in_flight=8)
        GP.advance_domain(solo, out["st1"][i]["steps"])
        for k in keys:
            assert np.array_equal(out[1][i][k], out[0][i][k]), (i, k)
            assert np.array_equal(out[1][i][k], solo.download(k)), (i, k)
        solo.close()

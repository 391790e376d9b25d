"""fx_adesolver_noalloc: the allocation-free ADE sweep.

It serves callers that cannot call cudaMalloc: a host model whose device
memory all comes from its own pool or arena, or a job under a fixed memory
cap. The tests call it through the C ABI on device arrays they allocate
themselves, as such a caller would, and check it
* against the ADE sweep that fx_step runs on a context, on two calls in a row
  (each starting from the concentration the previous call left);
* against the oracle's restatement of ADEsolver_calc on the pre-sweep state
  of steps that carried melt (the solute diluted by add_meteo before the
  sweep), on two calls in a row;
* at the edge of its static scratch: a grid of 100 strips whose scratch is
  within one column of the 8 MiB array, and a tall grid with more strips than
  the sweep has resident warps (strips handed out in turn), against the
  oracle;
* and that it refuses the same 100-strip grid one column wider (this check
  touches no device and also runs without a GPU).

This file is named to be collected last; it passes alone and after the other
tests (the entry point's scratch is a static device array shared by calls,
which keeps the last call's contents)."""
import ctypes as C
import re

import numpy as np
import pytest

import fluxos_cpp_b200 as fx
import gpu_pairs as GP
import pyoracle as P
from fluxos_cpp_b200 import scenarios as S

ROFF = 1  # row offset of the device layout (include/fluxos_gpu.h)
ROWS = 30  # rows per strip of the sweep
SCRATCH = 8 << 20  # bytes of the static array


def _flag_bytes(ldry, ldry_prev, wall):
    return ((ldry == 1.0).astype(np.uint8) | ((ldry_prev == 1.0).astype(np.uint8) << 1) |
            ((wall == 1.0).astype(np.uint8) << 2))


def _ld(nr):
    return ((nr + 3 + 31) // 32) * 32


def _device(torch, host_grid, ld, dtype):
    """Copy a GlobVar-layout host grid ([icol, irow]) into a fresh device
    array with leading dimension ld and the library's one-row offset."""
    mc, mr = host_grid.shape
    t = torch.zeros((mc, ld), dtype=dtype, device="cuda")
    t[:, ROFF:ROFF + mr] = torch.from_numpy(np.ascontiguousarray(host_grid)).to("cuda")
    return t


def _call(L, torch, conc, dev, flags, nr, nc, ld, dxy, dtfl, d_coef):
    stream = torch.cuda.current_stream().cuda_stream
    return L.fx_adesolver_noalloc(
        C.c_void_p(conc.data_ptr()), C.c_void_p(dev["h"].data_ptr()), C.c_void_p(dev["h0"].data_ptr()),
        C.c_void_p(flags.data_ptr()), C.c_void_p(dev["fe_1"].data_ptr()), C.c_void_p(dev["fn_1"].data_ptr()),
        nr, nc, ld, dxy, C.c_double(dtfl), C.c_double(d_coef), C.c_void_p(stream))


def _call_presweep(L, torch, g, nr, nc, dxy, dtfl, d_coef):
    """Upload a pre-sweep state (host grids in GlobVar layout) and sweep it;
    returns the swept concentration as a host grid."""
    ld = _ld(nr)
    conc = _device(torch, g["conc"], ld, torch.float64)
    dev = {k: _device(torch, g[k], ld, torch.float64) for k in ("h", "h0", "fe_1", "fn_1")}
    flags = _device(torch, _flag_bytes(g["ldry"], g["ldry_prev"], g["wall"]), ld, torch.uint8)
    rc = _call(L, torch, conc, dev, flags, nr, nc, ld, dxy, dtfl, d_coef)
    assert rc == 0, L.fx_last_error(None)
    return conc[:, ROFF:ROFF + nr + 2].cpu().numpy()


def _check(want, got):
    scale = 1e-6 * max(float(np.abs(want).max()), 1e-300)
    err = GP.rel_err(want[1:-1, 1:-1], got[1:-1, 1:-1], scale)
    assert err <= 1e-10, err


def _pair(tmp_path):
    """Two domains with the same wet start and no forcing (so no dilution):
    A without the ADE module, B with it. Their hydrodynamics are identical;
    after each step A holds the pre-sweep state of B's step."""
    nr, nc = 77, 64
    sc = S.plane_scenario(nr, nc, seed=8)
    sc.dem[20, 10:30] = -9999.0
    sc.write(str(tmp_path))
    ora = P.OracleRun(str(tmp_path), sc, 0)
    rng = np.random.default_rng(8)
    h = np.where(rng.random((nr, nc)) < 0.8, rng.uniform(0, 0.05, (nr, nc)), 0.0)
    ora.apply_wet_start(h, None, None, [rng.uniform(0, 2, (nr, nc)) * (h > 0)])
    doms = []
    for ade in (False, True):
        sc.ade = ade
        d = GP.domain_from_oracle(ora, sc, 0)
        d.set_forcing(None)
        d.prepare()
        doms.append(d)
    sc.ade = True
    return sc, doms[0], doms[1]


@pytest.mark.gpu
def test_noalloc_sweep_matches_step(tmp_path):
    import torch
    L = fx.lib()
    sc, A, B = _pair(tmp_path)
    nr, nc = sc.nrows, sc.ncols
    ld = _ld(nr)
    conc = None
    for call in range(2):
        # step 1: it = 1, the sweep is skipped in both; step 2 and 3: B sweeps
        if call == 0:
            A.step(1)
            B.step(1)
        A.step(1)
        B.step(1)
        sa, sb = A.status(), B.status()
        assert sa["it"] == sb["it"] >= 2 and sa["dtfl"] == sb["dtfl"]
        if conc is None:
            conc = _device(torch, A.download("conc"), ld, torch.float64)
        dev = {k: _device(torch, A.download(k), ld, torch.float64) for k in ("h", "h0", "fe_1", "fn_1")}
        fl = A.download_flags()
        flags = _device(torch, _flag_bytes(fl["ldry"], fl["ldry_prev"], fl["wall"]), ld, torch.uint8)
        rc = _call(L, torch, conc, dev, flags, nr, nc, ld, sc.dxy, sa["dtfl"], sc.d_coef)
        assert rc == 0, L.fx_last_error(None)
        _check(B.download("conc"), conc[:, ROFF:ROFF + nr + 2].cpu().numpy())
        # the next call starts from the swept concentration, as B does
    A.close()
    B.close()


def _oracle_presweep_with_melt(ora):
    """One step of the oracle (main.cpp:300-398 order) up to the sweep:
    Courant dt, clock, add_meteo (melt and the solute's dilution), the
    hydrodynamic update. Returns the pre-sweep grids and the step's it and
    dtfl; the oracle is left just before its ADE call. The melt must have
    diluted the solute."""
    ora.courant()
    ora.set_scalar("tim", ora.scalar("tim") + ora.scalar("dtfl"))
    before = ora.grid("conc").copy()
    assert ora.add_meteo() == 0
    assert not np.array_equal(before, ora.grid("conc"))
    assert ora.scalar("hpall") != 0
    ora.set_scalar("it", ora.scalar("it") + 1)
    ora.hydrodynamics()
    g = {k: ora.grid(k).copy() for k in ("conc", "h", "h0", "fe_1", "fn_1", "ldry", "ldry_prev", "wall")}
    return g, int(ora.scalar("it")), ora.scalar("dtfl")


@pytest.mark.gpu
def test_noalloc_sweep_matches_oracle_after_melt(tmp_path):
    """Pre-sweep states of two consecutive steps with melt (20 mm/day at
    2 mg/L: the concentration is diluted before each sweep), swept by two
    calls in a row and compared with the oracle's ADEsolver_calc."""
    import torch
    L = fx.lib()
    nr, nc = 95, 80
    sc = S.plane_scenario(nr, nc, seed=9)
    sc.meteo = ((0.0, 20.0, 2.0), (sc.horizon, 20.0, 2.0))
    sc.dem[30, 5:40] = -9999.0
    sc.write(str(tmp_path))
    ora = P.OracleRun(str(tmp_path), sc, 0)
    rng = np.random.default_rng(9)
    h = np.where(rng.random((nr, nc)) < 0.75, rng.uniform(0, 0.04, (nr, nc)), 0.0)
    ora.apply_wet_start(h, rng.normal(0, 0.001, (nr, nc)) * (h > 0), None,
                        [rng.uniform(0, 2, (nr, nc)) * (h > 0)])
    ora.step()  # it = 1: no sweep (ADEsolver_calc.cpp:45)
    for call in range(2):
        g, it, dtfl = _oracle_presweep_with_melt(ora)
        assert it >= 2
        got = _call_presweep(L, torch, g, nr, nc, sc.dxy, dtfl, sc.d_coef)
        ora.adesolver(it, 0)
        _check(ora.grid("conc"), got)


class _OracleState:
    """A bare oracle state (no input files) holding a given pre-sweep state."""

    def __init__(self, nr, nc, dxy, d_coef, dtfl, hdry=0.001):
        self.lib = P.oracle_lib()
        self.nr, self.nc = nr, nc
        self.s = self.lib.ox_create(nr, nc, 1)
        for k, v in (("dxy", dxy), ("D_coef", d_coef), ("dtfl", dtfl), ("hdry", hdry)):
            self.lib.ox_set_scalar(self.s, k.encode(), float(v))

    def grid(self, name):
        fl = name in P.FGRIDS
        p = (self.lib.ox_fgrid if fl else self.lib.ox_grid)(self.s, name.encode())
        return np.ctypeslib.as_array(p, shape=(self.nc + 2, self.nr + 2))

    def close(self):
        self.lib.ox_destroy(self.s)


def _random_presweep(nr, nc, seed, hdry=0.001):
    """A seeded pre-sweep state in GlobVar layout: mostly wet cells with
    depths above hdry, dry cells at or below it, some cells that changed
    between wet and dry in the step, face fluxes of both signs; ghost cells
    keep a thin depth, zero concentration and ldry 0 as the reference's
    start-up leaves them."""
    rng = np.random.default_rng(seed)
    shp = (nc + 2, nr + 2)
    wet = rng.random(shp) < 0.85
    h = np.where(wet, rng.uniform(0.002, 0.05, shp), rng.uniform(0.0, hdry, shp))
    g = {"h": h, "h0": h * rng.uniform(0.8, 1.2, shp),
         "fe_1": rng.normal(0, 0.002, shp), "fn_1": rng.normal(0, 0.002, shp),
         "conc": rng.uniform(0, 2, shp) * (rng.random(shp) < 0.9)}
    ldry = (~wet).astype(np.float32)
    prev = np.where(rng.random(shp) < 0.05, 1.0 - ldry, ldry).astype(np.float32)
    for a in (ldry, prev, g["conc"]):
        a[0, :] = a[-1, :] = 0
        a[:, 0] = a[:, -1] = 0
    g["ldry"], g["ldry_prev"] = ldry, prev
    g["wall"] = np.zeros(shp, dtype=np.float32)
    return g


def _oracle_sweep(g, nr, nc, dxy, d_coef, dtfl):
    o = _OracleState(nr, nc, dxy, d_coef, dtfl)
    for k, v in g.items():
        o.grid(k)[...] = v
    P.oracle_lib().ox_adesolver(o.s, 2, 0)
    out = o.grid("conc").copy()
    o.close()
    return out


def _needed_bytes(L, nr, nc):
    """The scratch the entry point reports for a grid that does not fit
    (fake pointers: the size is refused before any device access)."""
    p = C.c_void_p(256)
    ld = _ld(nr)
    rc = L.fx_adesolver_noalloc(p, p, p, p, p, p, nr, nc, ld, 2, C.c_double(0.1), C.c_double(0.01), None)
    assert rc == -1  # FX_ERR_ARG
    msg = L.fx_last_error(None).decode()
    assert "static array" in msg
    return int(re.search(r"needs (\d+) bytes", msg).group(1))


def _r256(n):
    return (n + 255) // 256 * 256


def _fixed_bytes(L):
    """The size-independent part of the scratch (control block, descriptor),
    from the bytes the entry point reports for a grid far over the limit."""
    nr, nc = 9000, 9000
    ns = (nr + ROWS - 1) // ROWS
    return _needed_bytes(L, nr, nc) - _r256(16 * ns) - _r256(8 * ns) - ns * (nc + 2) * 24


def _widest_fitting(L, nr):
    ns = (nr + ROWS - 1) // ROWS
    room = SCRATCH - _fixed_bytes(L) - _r256(16 * ns) - _r256(8 * ns)
    return room // (24 * ns) - 2


@pytest.mark.gpu
def test_noalloc_at_the_scratch_limit_matches_oracle():
    """100 strips whose hand-over scratch fills the 8 MiB array to within
    one column; the next wider grid is refused. Two calls in a row (the
    second on another state) check that the shared scratch starts clean."""
    import torch
    L = fx.lib()
    nr = 3000
    nc = _widest_fitting(L, nr)
    assert 3400 < nc < 3500
    assert _needed_bytes(L, nr, nc + 1) > SCRATCH
    for seed in (21, 22):
        g = _random_presweep(nr, nc, seed)
        dtfl = 0.5
        got = _call_presweep(L, torch, g, nr, nc, 2, dtfl, 0.01)
        _check(_oracle_sweep(g, nr, nc, 2, 0.01, dtfl), got)


@pytest.mark.gpu
def test_noalloc_more_strips_than_resident_warps_matches_oracle():
    """2,000 strips of a tall grid: more units than the sweep's resident
    warps (148 SMs x 3 blocks x 4 warps), so warps take strips in turn."""
    import torch
    L = fx.lib()
    nr, nc = 60000, 3
    g = _random_presweep(nr, nc, 23)
    got = _call_presweep(L, torch, g, nr, nc, 1, 0.25, 0.1)
    _check(_oracle_sweep(g, nr, nc, 1, 0.1, 0.25), got)


def test_noalloc_rejects_grids_beyond_the_static_scratch():
    L = fx.lib()
    assert _needed_bytes(L, 8192, 8192) > SCRATCH
    nr = 3000
    assert _needed_bytes(L, nr, _widest_fitting(L, nr) + 1) > SCRATCH

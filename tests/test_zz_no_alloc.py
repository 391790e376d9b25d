"""fx_adesolver_noalloc: the allocation-free ADE sweep, called through the C
ABI on device arrays this test allocates itself (as a caller with its own
memory pool would), checked against the ADE sweep that fx_step runs on a
context, on two calls in a row.

This file is named to be collected last; it passes alone and after the other
tests (the entry point's scratch is a static device array shared by calls)."""
import ctypes as C

import numpy as np
import pytest

import fluxos_cpp_b200 as fx
import gpu_pairs as GP
import pyoracle as P
from fluxos_cpp_b200 import scenarios as S

pytestmark = pytest.mark.gpu

ROFF = 1  # row offset of the device layout (include/fluxos_gpu.h)


def _flag_bytes(fl):
    return ((fl["ldry"] == 1.0).astype(np.uint8) | ((fl["ldry_prev"] == 1.0).astype(np.uint8) << 1) |
            ((fl["wall"] == 1.0).astype(np.uint8) << 2))


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


def _device(torch, host_grid, ld, dtype):
    """Copy a GlobVar-layout host grid into a fresh device array with leading
    dimension ld and the library's one-row offset."""
    mc, mr = host_grid.shape
    t = torch.zeros((mc, ld), dtype=dtype, device="cuda")
    t[:, ROFF:ROFF + mr] = torch.from_numpy(np.ascontiguousarray(host_grid)).to("cuda")
    return t


def test_noalloc_sweep_matches_step(tmp_path):
    import torch
    L = fx.lib()
    sc, A, B = _pair(tmp_path)
    nr, nc = sc.nrows, sc.ncols
    ld = ((nr + 3 + 31) // 32) * 32
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
        flags = _device(torch, _flag_bytes(A.download_flags()), ld, torch.uint8)
        stream = torch.cuda.current_stream().cuda_stream
        rc = L.fx_adesolver_noalloc(
            C.c_void_p(conc.data_ptr()), C.c_void_p(dev["h"].data_ptr()), C.c_void_p(dev["h0"].data_ptr()),
            C.c_void_p(flags.data_ptr()), C.c_void_p(dev["fe_1"].data_ptr()),
            C.c_void_p(dev["fn_1"].data_ptr()), nr, nc, ld, sc.dxy, C.c_double(sa["dtfl"]),
            C.c_double(sc.d_coef), C.c_void_p(stream))
        assert rc == 0, L.fx_last_error(None)
        got = conc[:, ROFF:ROFF + nr + 2].cpu().numpy()
        want = B.download("conc")
        scale = 1e-6 * float(np.abs(want).max())
        assert GP.rel_err(want[1:-1, 1:-1], got[1:-1, 1:-1], scale) <= 1e-10, call
        # the next call starts from the swept concentration, as B does
    A.close()
    B.close()


def test_noalloc_rejects_grids_beyond_the_static_scratch():
    L = fx.lib()
    big = 8192  # 274 strips x 8194 columns x 24 bytes > 8 MiB
    p = C.c_void_p(16)
    rc = L.fx_adesolver_noalloc(p, p, p, p, p, p, big, big, big + 32, 2, C.c_double(0.1), C.c_double(0.01),
                                None)
    assert rc == -1
    assert b"static array" in L.fx_last_error(None)

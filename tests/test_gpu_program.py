"""The drop-in surface on the GPU: `fluxos_gpu <modset.json>` (and the
library's fx_open_modset / fx_run_to_print / fx_write_results behind it)
against the Results files the reference program wrote for the same inputs
(tests/golden/plane_walls.npz and inflow.npz, frozen from the reference).

Every file must list the same cells in the same order with the same
integer and coordinate columns; state columns agree within 1e-10 relative
per value (floored at 1e-6 of the column's largest magnitude)."""
import os
import subprocess

import numpy as np
import pytest

import fluxos_cpp_b200 as fx
import golden_cases as G

pytestmark = pytest.mark.gpu


def _parse(text):
    lines = text.strip().split("\n")
    return lines[0], np.array([[float(v) for v in ln.split(",")] for ln in lines[1:]])


def _compare_results(folder, z, meta):
    got_files = sorted(os.listdir(folder), key=lambda s: int(s.split(".")[0]))
    assert got_files == meta["results"]
    for fn in got_files:
        hdr_ref, ref = _parse(str(z[f"results_{fn}"]))
        with open(os.path.join(folder, fn)) as f:
            hdr, got = _parse(f.read())
        assert hdr == hdr_ref
        assert got.shape == ref.shape, (fn, got.shape, ref.shape)
        assert np.array_equal(got[:, :4], ref[:, :4]), fn
        for col in range(4, 16):
            a, b = ref[:, col], got[:, col]
            scale = max(float(np.abs(a).max()), 1e-300) * 1e-6
            err = np.abs(a - b) / np.maximum(np.maximum(np.abs(a), np.abs(b)), scale)
            assert float(err.max()) <= 1e-10, (fn, col, float(err.max()))


@pytest.mark.parametrize("case", ["plane_walls", "inflow"])
def test_program_matches_reference_results(case, tmp_path):
    sc, z, meta, mp = G.materialise(case, str(tmp_path))
    r = subprocess.run([fx.EXE_PATH, mp], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    _compare_results(os.path.join(str(tmp_path), "Results"), z, meta)


def test_library_run_matches_reference_results(tmp_path):
    sc, z, meta, mp = G.materialise("plane_walls", str(tmp_path))
    fx.run(mp)
    _compare_results(os.path.join(str(tmp_path), "Results"), z, meta)


def test_open_modset_state_matches_host_loader(tmp_path):
    sc, z, meta, mp = G.materialise("patchwork_weir", str(tmp_path))
    d = fx.Domain.from_modset(mp)
    st = fx.load_modset(mp)
    for k in ("zb", "z", "h", "qx", "qy", "conc"):
        assert np.array_equal(d.download(k), st[k]), k
    fl = d.download_flags()
    assert np.array_equal(fl["ldry"], st["ldry"]) and np.array_equal(fl["wall"], st["wall"])
    d.close()

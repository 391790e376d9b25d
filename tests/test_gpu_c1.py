"""The small CPU configuration end to end on the GPU, FP64: the drop-in
program `fluxos_gpu <modset.json>` on the 200 x 200 plane with bumps, dry
start, 6 h of melt (46,113 iterations of main.cpp:271-470, 36 Results
files), against the reference program's files frozen in
tests/golden/c1_plane200.npz.

Every file must exist with the same name, header, row set and order and the
same number of wet cells (h > ROUGNESS_HEIGHT); its text is either identical
to the reference's (SHA-256) or its state columns agree within 1e-10
relative per value on 256 sample rows and within 1e-10 of the column's sum of
magnitudes on three column sums. The files at 10,200 s and 21,600 s are
compared value by value (1e-10 relative, floored at 1e-6 of the column's
largest magnitude)."""
import os
import subprocess
import time

import pytest

import c1_case as C1
import fluxos_cpp_b200 as fx
import results_digest as RD

pytestmark = pytest.mark.gpu


def test_c1_program_matches_reference_results(tmp_path):
    z, meta = C1.load()
    sc, mp = C1.write_inputs(str(tmp_path))
    t0 = time.perf_counter()
    r = subprocess.run([fx.EXE_PATH, mp], capture_output=True, text=True, timeout=900)
    wall = time.perf_counter() - t0
    assert r.returncode == 0, r.stderr[-2000:]
    res = os.path.join(str(tmp_path), "Results")
    files = sorted(os.listdir(res), key=lambda s: int(s.split(".")[0]))
    assert files == meta["results"]
    identical, worst = 0, 0.0
    for fn in files:
        with open(os.path.join(res, fn)) as f:
            text = f.read()
        out = RD.compare(text, C1.digest_of(z, meta, fn), sc.nrows, sc.ncols, sc.ks)
        identical += out["identical"]
        worst = max(worst, out["worst"])
        if fn in meta["full"]:
            worst = max(worst, RD.compare_full(text, z[f"full_{fn.split('.')[0]}"]))
    print(f"c1: {len(files)} files, {identical} byte-identical to the reference's, worst relative "
          f"difference {worst:.3g}, program wall time {wall:.2f} s")

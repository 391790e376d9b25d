"""The per-step fields (h, h0, fe_1, fn_1) live in one record per cell and
slot plane. Uploading one writes its component into the current slot and
into every slot's ghost ring; downloading reads the current slot. Both
precisions must return what was uploaded (FP32: rounded once to float),
each field unchanged by uploads of the others."""
import numpy as np
import pytest

import fluxos_cpp_b200 as fx

pytestmark = pytest.mark.gpu

FIELDS = ("h", "h0", "fe_1", "fn_1")


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_record_fields_round_trip(precision):
    rng = np.random.default_rng(7)
    d = fx.Domain(70, 45, 2, hdry=0.001, ntim=100.0, precision=precision, steps_in_flight=5)
    grids = {k: rng.uniform(-1.0, 1.0, d.shape) for k in FIELDS}
    for k in FIELDS:
        d.upload(k, grids[k])
    for k in FIELDS:
        want = grids[k] if precision == "fp64" else grids[k].astype(np.float32).astype(np.float64)
        assert np.array_equal(d.download(k), want), k
    # a second upload of one field leaves the others as they were
    grids["h0"] = rng.uniform(-1.0, 1.0, d.shape)
    d.upload("h0", grids["h0"])
    for k in FIELDS:
        want = grids[k] if precision == "fp64" else grids[k].astype(np.float32).astype(np.float64)
        assert np.array_equal(d.download(k), want), k
    d.close()

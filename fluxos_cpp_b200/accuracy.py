"""Error of a run against the FP64 path, and the water balance of a run.

Used by the FP32 tests and by bench.py. Depth and discharge errors compare
interior cells of two domains holding the same scenario at the same step:

* relative L1 error  sum|a - b| / sum|b|;
* L-infinity error   max|a - b| (absolute) and that divided by max|b|;
* discharge is |q| = sqrt(qx^2 + qy^2).

The relative mass-balance error of one run is
|W(t) - W(0) - (melt in - out)| / W(t), with W the stored water (FP64 sum on
the device, fx_mass) and the two budget terms the run's FP64 accumulators
(fx_status budget_melt, budget_out).
"""
from __future__ import annotations

import numpy as np


def _interior(g: np.ndarray) -> np.ndarray:
    return np.asarray(g, dtype=np.float64)[1:-1, 1:-1]


def _pair_errors(a: np.ndarray, b: np.ndarray) -> dict:
    d = np.abs(a - b)
    sb = float(np.abs(b).sum())
    mb = float(np.abs(b).max()) if b.size else 0.0
    return {"l1_rel": float(d.sum()) / sb if sb > 0 else float(d.sum()),
            "linf_abs": float(d.max()) if d.size else 0.0,
            "linf_rel": (float(d.max()) / mb) if mb > 0 else 0.0}


def state_errors(test, ref, hdry: float = 1e-3) -> dict:
    """Depth, discharge and solute errors of domain `test` against `ref`."""
    ht, hr = _interior(test.download("h")), _interior(ref.download("h"))
    qt = np.hypot(_interior(test.download("qx")), _interior(test.download("qy")))
    qr = np.hypot(_interior(ref.download("qx")), _interior(ref.download("qy")))
    out = {"depth": _pair_errors(ht, hr), "discharge": _pair_errors(qt, qr)}
    wt, wr = ht > hdry, hr > hdry
    out["wet_cells"] = {"test": int(wt.sum()), "ref": int(wr.sum()), "differ": int((wt != wr).sum())}
    conc = []
    for k in range(ref.nchem):
        nm = "conc" if k == 0 else f"conc{k}"
        conc.append(_pair_errors(_interior(test.download(nm)) * ht, _interior(ref.download(nm)) * hr))
    out["solute_mass_density"] = conc
    return out


def water_balance(d, w0: float) -> dict:
    """Stored water now, the budget since creation, and the relative error."""
    w, _ = d.mass()
    st = d.status()
    resid = (w - w0) - (st["budget_melt"] - st["budget_out"])
    return {"stored": w, "stored0": w0, "melt_in": st["budget_melt"], "out": st["budget_out"],
            "residual": resid, "rel_err": abs(resid) / w if w > 0 else abs(resid)}

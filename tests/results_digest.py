"""Compact digests of Results/<t>.txt files (write_results.cpp:30-101), so a
long run's outputs can be frozen as a small fixture and compared later.

A digest keeps, per file:
* the SHA-256 of the whole text (equal text: every value identical);
* the header line and the row count;
* which cells are listed, as a bit mask over the interior in file order
  (icol outer, irow inner), which fixes the row set and its order;
* per state column, the sum, the sum of magnitudes and a sum weighted by a
  fixed function of the cell (so a value moved to another cell shows);
* 256 seeded sample rows, every column at full precision;
* the number of listed cells deeper than the dry threshold (wet cells).
Whole files, when wanted, are kept as arrays of the varying columns.

Columns (16): irow, icol, X, Y, z, h, ux, uy, qx*dxy, qy*dxy, us, conc,
soil_mass, fe_1, fn_1, twet. ux, uy and us are always 0 in this version of
the reference (never computed), so they are checked to be 0.
"""
from __future__ import annotations

import hashlib

import numpy as np

STATE_COLS = (4, 5, 8, 9, 11, 12, 13, 14, 15)
ZERO_COLS = (6, 7, 10)
SAMPLES = 256


def parse(text: str):
    lines = text.rstrip("\n").split("\n")
    body = "\n".join(lines[1:])
    if not body:
        return lines[0], np.zeros((0, 16))
    a = np.array(body.replace("\n", ",").split(","), dtype=np.float64).reshape(-1, 16)
    return lines[0], a


def cell_weights(irow: np.ndarray, icol: np.ndarray) -> np.ndarray:
    """A fixed weight in [-0.5, 0.5) per cell, independent of row order."""
    k = (irow.astype(np.int64) * 7919 + icol.astype(np.int64) * 104729) % 1009
    return k / 1009.0 - 0.5


def digest(text: str, nrows: int, ncols: int, seed: int, hdry: float) -> dict:
    hdr, a = parse(text)
    irow, icol = a[:, 0].astype(np.int64), a[:, 1].astype(np.int64)
    mask = np.zeros((ncols, nrows), dtype=bool)  # [icol - 1, irow - 1]: file order when raveled
    mask[icol - 1, irow - 1] = True
    w = cell_weights(irow, icol)
    sums = np.array([[a[:, c].sum(), np.abs(a[:, c]).sum(), (w * a[:, c]).sum(), np.abs(a[:, c]).max(initial=0.0)]
                     for c in STATE_COLS])
    rng = np.random.default_rng(seed)
    pick = np.sort(rng.choice(len(a), size=min(SAMPLES, len(a)), replace=False)) if len(a) else np.zeros(0, int)
    return {"sha256": hashlib.sha256(text.encode()).hexdigest(), "header": hdr, "rows": int(len(a)),
            "wet": int((a[:, 5] > hdry).sum()), "mask": np.packbits(mask.ravel()), "sums": sums,
            "samples": a[pick]}


def full_columns(text: str) -> np.ndarray:
    """The listed cells' irow, icol and state columns of one file."""
    _, a = parse(text)
    return a[:, (0, 1) + STATE_COLS]


def rel_err_floored(a: np.ndarray, b: np.ndarray, scale: float) -> float:
    """Largest |a-b| / max(|a|, |b|, scale) (0 when equal)."""
    if np.array_equal(a, b):
        return 0.0
    d = np.abs(a - b)
    return float((d / np.maximum(np.maximum(np.abs(a), np.abs(b)), scale)).max())


def compare(text: str, ref: dict, nrows: int, ncols: int, hdry: float, rtol: float = 1e-10) -> dict:
    """Check a Results file against a digest: the same header, row count and
    row set, the same number of wet cells; zero ux, uy, us; per state column
    the sums within rtol of the sum of magnitudes (plus the per-value floor
    of 1e-6 of the column's largest magnitude); the sample rows within rtol
    per value (same floor). Returns {"identical": bool, "worst": float};
    raises AssertionError on a failed check."""
    hdr, a = parse(text)
    if hashlib.sha256(text.encode()).hexdigest() == ref["sha256"]:
        return {"identical": True, "worst": 0.0}
    assert hdr == ref["header"], "header differs"
    assert len(a) == ref["rows"], ("row count", len(a), ref["rows"])
    assert int((a[:, 5] > hdry).sum()) == ref["wet"], "wet cell count differs"
    irow, icol = a[:, 0].astype(np.int64), a[:, 1].astype(np.int64)
    mask = np.zeros((ncols, nrows), dtype=bool)
    mask[icol - 1, irow - 1] = True
    assert np.array_equal(np.packbits(mask.ravel()), ref["mask"]), "row set differs"
    order = np.lexsort((irow, icol))
    assert np.array_equal(order, np.arange(len(a))), "rows out of file order"
    for c in ZERO_COLS:
        assert not np.any(a[:, c]), ("column must be 0", c)
    w = cell_weights(irow, icol)
    worst = 0.0
    n = max(len(a), 1)
    for j, c in enumerate(STATE_COLS):
        s_ref, abs_ref, w_ref, mx_ref = ref["sums"][j]
        tol = rtol * abs_ref + rtol * 1e-6 * mx_ref * n + 1e-300
        for got, want in ((a[:, c].sum(), s_ref), (np.abs(a[:, c]).sum(), abs_ref), ((w * a[:, c]).sum(), w_ref)):
            err = abs(got - want)
            assert err <= tol, ("column sum", c, float(got), float(want))
            worst = max(worst, err / max(abs_ref, 1e-300))
    smp = ref["samples"]
    key = {(int(r[0]), int(r[1])): i for i, r in enumerate(a[:, :2])}
    rows = a[[key[(int(r[0]), int(r[1]))] for r in smp]] if len(smp) else np.zeros((0, 16))
    assert np.array_equal(rows[:, :4], smp[:, :4]), "sample cells differ"
    for c in STATE_COLS:
        scale = max(float(ref["sums"][STATE_COLS.index(c)][3]), 1e-300) * 1e-6
        e = rel_err_floored(smp[:, c], rows[:, c], scale)
        assert e <= rtol, ("sample values", c, e)
        worst = max(worst, e)
    return {"identical": False, "worst": worst}


def compare_full(text: str, ref_cols: np.ndarray, rtol: float = 1e-10) -> float:
    """Every listed value of a file against the frozen columns; returns the
    largest relative error (floored at 1e-6 of each column's largest
    magnitude)."""
    got = full_columns(text)
    assert got.shape == ref_cols.shape, (got.shape, ref_cols.shape)
    assert np.array_equal(got[:, :2], ref_cols[:, :2]), "row set differs"
    worst = 0.0
    for j in range(2, got.shape[1]):
        scale = max(float(np.abs(ref_cols[:, j]).max(initial=0.0)), 1e-300) * 1e-6
        worst = max(worst, rel_err_floored(ref_cols[:, j], got[:, j], scale))
    assert worst <= rtol, worst
    return worst

"""The Results-file digests (tests/results_digest.py) on the CPU: a file
passes against its own digest, planted mistakes in a copy are caught, and
the config-1 fixture's inputs are regenerated byte for byte."""
import numpy as np
import pytest

import c1_case as C1
import golden_cases as G
import results_digest as RD


def _case_text():
    z, meta = G.load("plane_walls")
    fn = meta["results"][-1]
    return str(z[f"results_{fn}"]), meta


def test_digest_accepts_its_own_file():
    text, meta = _case_text()
    dg = RD.digest(text, meta["nrows"], meta["ncols"], seed=0, hdry=meta["ks"])
    assert RD.compare(text, dg, meta["nrows"], meta["ncols"], meta["ks"])["identical"]


def _replace_value(text, row, col, fmt):
    lines = text.split("\n")
    vals = lines[row].split(",")
    vals[col] = fmt(float(vals[col]))
    lines[row] = ",".join(vals)
    return "\n".join(lines)


@pytest.mark.parametrize("col", [4, 5, 11, 15])
def test_digest_catches_a_changed_value(col):
    text, meta = _case_text()
    dg = RD.digest(text, meta["nrows"], meta["ncols"], seed=0, hdry=meta["ks"])
    nlines = len(text.rstrip("\n").split("\n"))
    for row in (1, nlines // 2, nlines - 1):
        bad = _replace_value(text, row, col, lambda v: repr(v * (1 + 1e-7) + 1e-9))
        with pytest.raises(AssertionError):
            RD.compare(bad, dg, meta["nrows"], meta["ncols"], meta["ks"])
    # a rounding in the last printed digit stays within 1e-10
    ok = _replace_value(text, 1, col, lambda v: repr(float(np.nextafter(v, np.inf))))
    assert not RD.compare(ok, dg, meta["nrows"], meta["ncols"], meta["ks"])["identical"]


def test_digest_catches_a_missing_or_moved_row():
    text, meta = _case_text()
    dg = RD.digest(text, meta["nrows"], meta["ncols"], seed=0, hdry=meta["ks"])
    lines = text.rstrip("\n").split("\n")
    with pytest.raises(AssertionError):
        RD.compare("\n".join(lines[:-1]) + "\n", dg, meta["nrows"], meta["ncols"], meta["ks"])
    swapped = lines[:]
    swapped[1], swapped[2] = swapped[2], swapped[1]
    with pytest.raises(AssertionError):
        RD.compare("\n".join(swapped) + "\n", dg, meta["nrows"], meta["ncols"], meta["ks"])


def test_c1_inputs_regenerate(tmp_path):
    z, meta = C1.load()
    C1.write_inputs(str(tmp_path))
    assert len(meta["results"]) == 36
    assert meta["results"][-1] == "21600.txt"
    assert set(meta["full"]) <= set(meta["results"])

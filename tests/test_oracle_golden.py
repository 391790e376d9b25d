"""The oracle (C restatement) against the golden fixtures frozen from the
FLUXOS reference: every state grid bit for bit at every snapshot, and the
Results/<t>.txt files byte for byte through the product's writer."""
import os

import numpy as np
import pytest

import golden_cases as G
import pyoracle as P

SNAP = ("z", "h", "qx", "qy", "conc", "fe_1", "fe_2", "fe_3", "fn_1", "fn_2", "fn_3", "twet", "h0",
        "ldry", "ldry_prev", "zb", "wall", "ks", "soil_mass")


@pytest.mark.parametrize("case", G.CASES)
def test_oracle_matches_reference_snapshots(case, tmp_path):
    sc, z, meta, _ = G.materialise(case, str(tmp_path))
    ora = P.OracleRun(str(tmp_path), sc, meta["volrat_mode"])
    G.apply_start(ora, z, meta)
    done = 0
    for target in meta["steps"]:
        while done < target:
            ora.step()
            if ora.print_due():
                ora.print_done()
            done += 1
        for g in SNAP:
            ref = z[f"s{target}_{g}"]
            got = ora.grid(g)
            assert np.array_equal(ref, got, equal_nan=True), (case, target, g, P.max_ulp_diff(ref, got))
        sc_ref = meta["scalars"][str(target)]
        for k in ("tim", "dtfl", "it", "hpall", "print_next"):
            assert ora.scalar(k) == sc_ref[k], (case, target, k)


@pytest.mark.parametrize("case", ["plane_walls", "inflow"])
def test_results_files_match_reference_program(case, tmp_path):
    """Step the oracle through a case and write every output with the
    product's host writer; compare with the reference program's files."""
    from fluxos_cpp_b200 import write_results_host
    sc, z, meta, _ = G.materialise(case, str(tmp_path))
    ora = P.OracleRun(str(tmp_path), sc, 0)
    files = meta["results"]
    out = tmp_path / "out"
    out.mkdir()
    written = []
    while ora.running():
        ora.step()
        if ora.print_due():
            pn = int(round(ora.scalar("print_next")))
            fn = str(out / f"{pn}.txt")
            grids = {k: ora.grid(k) for k in ("z", "zb", "h", "qx", "qy", "conc", "soil_mass", "fe_1", "fn_1",
                                              "twet")}
            write_results_host(fn, sc.nrows, sc.ncols, sc.dxy, sc.xll, sc.yll, meta["h_min_print"], grids)
            written.append(f"{pn}.txt")
            ora.print_done()
    assert written == files
    for f in files:
        with open(out / f) as fh:
            assert fh.read() == str(z[f"results_{f}"]), f

"""Build an oracle run and a GPU domain from the same start-up state, step
them side by side, and compare. Used by the gpu tests and by smoke()."""
import numpy as np

import fluxos_cpp_b200 as fx
import pyoracle as P

STATE = ("z", "h", "qx", "qy", "twet", "h0", "fe_1", "fe_2", "fe_3", "fn_1", "fn_2", "fn_3")


def domain_from_oracle(ora, sc, volrat_mode=0, store_all=True, steps_in_flight=0):
    nchem = sc.nchem
    d = fx.Domain(sc.nrows, sc.ncols, sc.dxy, nchem=nchem, nodata=float(sc.nodata),
                  hdry=ora.scalar("hdry"), ntim=ora.scalar("ntim"), print_step=sc.print_step,
                  print_next=ora.scalar("print_next"), tim=ora.scalar("tim"), ade=sc.ade,
                  volrat_mode=volrat_mode,
                  d_coef=list(sc.d_coefs) if sc.d_coefs else [sc.d_coef],
                  steps_in_flight=steps_in_flight, wintra=bool(ora.scalar("wintra")),
                  soil_release_rate=ora.scalar("soil_release_rate"))
    for k in ("zb",) + STATE:
        d.upload(k, ora.grid(k))
    for k in range(nchem):
        nm = "conc" if k == 0 else f"conc{k}"
        d.upload(nm, ora.grid(nm))
    d.upload_flags(ora.grid("ldry"), ora.grid("wall"))
    if ora.grid("soil_mass").any():
        d.upload("soil_mass", ora.grid("soil_mass"))
    d.set_forcing(ora.fgrid("meteo"))
    if ora.scalar("has_inflow"):
        d.set_inflow(ora.fgrid("inflow"), int(ora.scalar("inflow_nrow")), int(ora.scalar("inflow_ncol")))
    if sc.manning is not None:
        m = np.zeros(d.shape)
        m[1:-1, 1:-1] = sc.manning.T
        d.set_manning(m)
    if sc.melt_mult is not None:
        m = np.ones(d.shape)
        m[1:-1, 1:-1] = sc.melt_mult.T
        d.set_melt_field(m)
    d.set_option("store_all_fluxes", 1 if store_all else 0)
    d.prepare()
    return d


def advance_oracle(ora, n):
    for _ in range(n):
        if not ora.running():
            return
        ora.step()
        if ora.print_due():
            ora.print_done()


def advance_domain(d, n):
    """Exactly n steps (acknowledging outputs on the way), or until the end."""
    start = d.status()["steps"]
    while True:
        st = d.status()
        if st["print_pending"]:
            d.print_done()
            continue
        left = n - (st["steps"] - start)
        if left <= 0 or st["finished"]:
            return st
        d.step(left)


def rel_err(a, b, scale):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if np.array_equal(a, b, equal_nan=True):
        return 0.0
    d = np.abs(a - b)
    s = np.maximum(np.maximum(np.abs(a), np.abs(b)), scale)
    return float(np.nanmax(d / s))


def compare(ora, d, sc, fields=STATE, rtol=1e-10):
    """Per-field max relative error (floored at 1e-6 of the field's scale)
    and the number of cells whose wet/dry flags differ."""
    out = {}
    for k in list(fields) + [("conc" if i == 0 else f"conc{i}") for i in range(sc.nchem)] + ["soil_mass"]:
        a = ora.grid(k)[1:-1, 1:-1]
        b = d.download(k)[1:-1, 1:-1]
        scale = max(float(np.nanmax(np.abs(a))) if a.size else 0.0, 1e-300) * 1e-6
        out[k] = rel_err(a, b, scale)
    fl = d.download_flags()
    out["ldry_mismatch"] = int((fl["ldry"][1:-1, 1:-1] != ora.grid("ldry")[1:-1, 1:-1]).sum())
    out["ldry_prev_mismatch"] = int((fl["ldry_prev"][1:-1, 1:-1] != ora.grid("ldry_prev")[1:-1, 1:-1]).sum())
    st = d.status()
    out["tim"] = rel_err(st["tim"], ora.scalar("tim"), 1e-300)
    out["it"] = int(st["it"] - ora.scalar("it"))
    bad = {k: v for k, v in out.items()
           if (k.endswith("mismatch") and v) or (k == "it" and v) or
           (not k.endswith("mismatch") and k != "it" and v > rtol)}
    return out, bad

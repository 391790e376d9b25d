#!/usr/bin/env python
"""Benchmark of the FLUXOS-OVERLAND explicit step on one B200 per rank.

Workload (the large single-domain configuration): 4096 x 4096 cells of 2 m,
spectral-fractal terrain (P(k) ~ k^-3, seed 1, 0-3 m relief) with 200
circular depressions, a smooth melt-rate field of 5-40 mm/day (seed 2) as a
per-cell multiplier of the forcing rate, Manning n ~ U[0.03, 0.15], one
solute (D = 0.01 m^2/s). All inputs are seeded synthetic stand-ins generated
by fluxos_cpp_b200.scenarios. The state starts wet (a 5 mm film plus water
ponded in the depressions), as a snapshot taken during melt would be.

A step is one iteration of the reference's loop (main.cpp:271-406): Courant
dt, melt forcing, the hydrodynamic update and the ADE sweep over all cells.
metric = cell-updates/s = cells x steps / device time; with N ranks each rank
runs its own replica and value is the sum (weak scaling, no collective).

--impl reference times the FLUXOS reference sources compiled in oracle/_ref
(OpenMP hydrodynamics, serial ADE) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s FP32 vs FP64 at stated depth/mass error; p50/p99 request latency"
# Algorithmic bytes per cell-update of the step (read + write of h, qx, qy and
# the solute, read of bed and wall, read of Manning n and the melt field):
# 2*8*(3+1) + 8 + 1 + 8 + 4 = 85 B, and 89 B when the melt field is 8 bytes
# as here (FP64 storage). Split by kernel: the hydrodynamic kernel moves the
# flow state, bed, wall, n and melt (2*8*3 + 8 + 1 + 8 + 8 = 73 B), the ADE
# sweep the solute (2*8 = 16 B).
ALG_BYTES_STEP = 89
ALG_BYTES_HYDRO = 73
ALG_BYTES_ADE = 16


def _rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while running."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self.gpu_id, f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.15)

    def stop(self) -> dict:
        if self.proc is not None:
            time.sleep(0.06)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        rows = []
        try:
            for ln in open(self.path):
                parts = [x.strip() for x in ln.split(",")]
                if len(parts) >= 8:
                    rows.append(parts)
            os.unlink(self.path)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "", 1).isdigit()]
        mx = [float(r[1]) for r in rows if r[1].replace(".", "", 1).isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[4 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def gpu_id_of_device0() -> str:
    import torch
    try:
        u = str(torch.cuda.get_device_properties(0).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0]
        return vis or "0"


def make_workload(n: int, seed: int = 1):
    """Terrain, melt multiplier, Manning n, forcing table and the wet start."""
    from fluxos_cpp_b200 import scenarios as S
    sc = S.fractal_scenario(n, dxy=2, seed=seed, melt_seed=seed + 1, extensions=True)
    dem = sc.dem.astype(np.float64)
    film = 0.005
    h = film + np.maximum(S.box3(S.box3(dem)) - dem, 0.0)
    conc = np.where(h > 2 * film, 1.0, 0.0)
    return sc, h, conc


def forcing_table(sc) -> np.ndarray:
    tab = np.zeros((3, 2000), dtype=np.float32)
    rows = list(sc.meteo) + [(1.0e9, 0.0, 0.0), (sc.horizon, 0.0, 0.0)]
    for a, (t, r, c) in enumerate(rows, start=1):
        tab[:, a] = (t, r, c)
    return tab


def full(sc, interior: np.ndarray, fill: float = 0.0) -> np.ndarray:
    g = np.full((sc.ncols + 2, sc.nrows + 2), fill)
    g[1:-1, 1:-1] = interior.T
    return g


def build_domain(sc, h, conc, in_flight: int = 8):
    import fluxos_cpp_b200 as fx
    d = fx.Domain(sc.nrows, sc.ncols, sc.dxy, nchem=1, hdry=sc.ks, ntim=sc.horizon,
                  print_step=sc.print_step, print_next=sc.print_step, ade=True, d_coef=[sc.d_coef],
                  steps_in_flight=in_flight)
    zb_raw = full(sc, sc.dem.astype(np.float64))
    d.initiate(zb_raw)
    d.set_forcing(forcing_table(sc))
    d.set_melt_field(full(sc, sc.melt_mult, 1.0))
    d.set_manning(full(sc, sc.manning, 0.0))
    zb = d.download("zb")
    z = zb.copy()
    z[1:-1, 1:-1] += h.T
    hh = np.zeros_like(zb)
    hh[1:-1, 1:-1] = h.T
    d.upload("z", z)
    d.upload("h", hh)
    d.upload("conc", full(sc, conc))
    fl = d.download_flags()
    ld = np.zeros_like(fl["ldry"])
    ld[1:-1, 1:-1] = np.where(h.T > sc.ks, 0.0, 1.0)
    d.upload_flags(ld, fl["wall"])
    d.prepare()
    return d


def e2e_run(d, sc, steps: int):
    """Through the public API with host buffers: upload the state from
    pinned host memory, step (each step reads its status back), download the
    Results fields. Returns (seconds, h2d bytes, d2h bytes)."""
    import torch
    shape = d.shape
    names_up = ("z", "h", "qx", "qy", "conc", "twet")
    names_dn = ("z", "h", "qx", "qy", "conc")
    host = {k: torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy() for k in names_up}
    for k in names_up:
        d.download(k, host[k])
    fl = d.download_flags()
    ldry = torch.empty(shape, dtype=torch.float32, pin_memory=True).numpy()
    wall = torch.empty(shape, dtype=torch.float32, pin_memory=True).numpy()
    ldry[...] = fl["ldry"]
    wall[...] = fl["wall"]
    out = {k: torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy() for k in names_dn}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in names_up:
        d.upload(k, host[k])
    d.upload_flags(ldry, wall)
    d.prepare()
    for _ in range(steps):
        d.step(1)
    for k in names_dn:
        d.download(k, out[k])
    t1 = time.perf_counter()
    cells = shape[0] * shape[1]
    h2d = cells * (8 * len(names_up) + 8) + 8 * steps
    d2h = cells * 8 * len(names_dn) + 256 * steps
    return t1 - t0, h2d, d2h


def cpu_reference_run(sc, h, conc, warmup: int, steps: int, crop: int):
    """The reference sources (oracle/_ref) on a crop of the same workload,
    in parity mode (the reference has no melt field and no Manning term)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as P
    from fluxos_cpp_b200 import scenarios as S
    if not P.ref_available(0):
        return None
    n = min(crop, sc.nrows)
    sub = S.Scenario(name=f"crop{n}", dem=sc.dem[:n, :n].copy(), dxy=sc.dxy,
                     meteo=sc.meteo, horizon=sc.horizon, print_step=sc.print_step, ks=sc.ks,
                     ade=True, d_coef=sc.d_coef)
    with tempfile.TemporaryDirectory() as tmp:
        mp = sub.write(tmp)
        ref = P.RefRun(mp, sub, 0)
        ref.apply_wet_start(h[:n, :n], None, None, [conc[:n, :n]])
        for _ in range(warmup):
            ref.step()
        t0 = time.perf_counter()
        for _ in range(steps):
            ref.step()
        t1 = time.perf_counter()
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": n * n * steps / (t1 - t0), "unit": "cell-updates/s", "cores": threads,
            "kind": "reference", "seconds": t1 - t0,
            "sample": f"{n}x{n} crop of the workload (uniform melt at the field mean, no Manning: "
                      f"the reference has neither), {warmup} warm-up + {steps} timed steps, "
                      f"reference sources from oracle/_ref, OpenMP hydrodynamics on {threads} threads, "
                      f"serial ADE"}


def run_gpu(args):
    import torch
    import torch.distributed as dist
    rank, world, local = _rank()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    import fluxos_cpp_b200 as fx
    n = args.size
    k_batch = args.in_flight  # steps per ADE launch
    sc, h, conc = make_workload(n)
    d = build_domain(sc, h, conc, k_batch)
    cells = n * n
    d.step(args.warmup)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(gpu_id_of_device0())
    sampler.start()
    ms_total, ms_hydro, ms_ade = d.time_steps(args.steps)
    clocks = sampler.stop()
    torch.cuda.synchronize()
    t = torch.tensor([ms_total], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
    ms_max = float(t.item())
    st = d.status()
    if st["device_error"]:
        raise RuntimeError("device error during the timed steps")
    value = cells * args.steps * world / (ms_max / 1e3)
    # dominant kernel and its roofline
    peak, peak_kind = _peaks()
    ms_h, ms_a = ms_hydro / args.steps, ms_ade / args.steps
    kern = {"k_hydro": (ms_h, ALG_BYTES_HYDRO), "k_ade_sweep": (ms_a, ALG_BYTES_ADE)}
    dom = max(kern, key=lambda k: kern[k][0])
    dms, dbytes = kern[dom]
    achieved = cells * dbytes / (dms / 1e3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        try:
            traffic = json.load(open(tp)).get(f"{dom}_{n}")
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                "traffic": traffic, "alg_bytes_per_cell": dbytes,
                "ms_per_step": {"k_hydro": round(ms_h, 4), "k_ade_sweep": round(ms_a, 4)},
                "ade_steps_per_launch": k_batch,
                "step_alg_GBps": round(cells * ALG_BYTES_STEP / (ms_max / args.steps / 1e3) / 1e9, 1)}
    e2e = None
    if not args.no_e2e:
        secs, h2d, d2h = e2e_run(d, sc, args.steps)
        e2e = {"value": cells * args.steps / secs, "unit": "cell-updates/s",
               "h2d_bytes_per_step": int(h2d / args.steps), "d2h_bytes_per_step": int(d2h / args.steps),
               "note": "upload of the state from pinned host memory, K steps each reading its "
                       "status back, download of the Results fields; per-step bytes = totals / K"}
    batches = (args.steps + k_batch - 1) // k_batch
    launches = 2 * args.steps + 2 * batches  # finalize + hydro per step; batch open + sweep per batch
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_reference_run(sc, h, conc, 1, args.cpu_steps, args.cpu_crop)
    d.close()
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded fractal terrain, melt field and Manning n)",
                "config": {"workload": f"fractal {n}x{n} cells of 2 m, 200 depressions, melt field "
                                       f"5-40 mm/day, Manning n U[0.03,0.15], one solute, wet start",
                           "precision": "fp64 (parity path)", "cells": cells,
                           "l2": "inputs larger than L2 (about 2 GB of state per replica)",
                           "parallelism": f"replicas x{world}"},
                "roofline": roofline, "e2e": e2e, "gpu_launches": launches, "clocks": clocks,
                "cpu_baseline": cpu,
                "accuracy": {"reference": "FP64 oracle, tests/test_gpu_parity.py",
                             "max_rel_err_per_cell": "<= 1e-10"}}
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def run_reference(args):
    rank, world, local = _rank()
    if rank != 0:
        return
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    sc, h, conc = make_workload(args.size)
    r = cpu_reference_run(sc, h, conc, args.warmup, args.steps, args.cpu_crop)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref is not built (the "
                          "reference tree was absent when build() ran)"}))
        return
    line = {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": "cell-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": r["seconds"] / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"fractal {args.size}x{args.size} (crop {min(args.cpu_crop, args.size)}"
                                   f"^2 timed), parity mode", "precision": "fp64"},
            "cpu_baseline": {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": r["value"], "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=("b200", "reference"))
    ap.add_argument("--size", type=int, default=4096)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-crop", type=int, default=2048)
    ap.add_argument("--cpu-steps", type=int, default=12)
    ap.add_argument("--in-flight", type=int, default=8, help="steps per ADE launch (1..15)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()

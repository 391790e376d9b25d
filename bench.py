#!/usr/bin/env python
"""Benchmark of the FLUXOS-OVERLAND explicit step on one B200 per rank.

Headline workload (the large single-domain configuration, FP64 plain vs
FP32): 4096 x 4096 cells of 2 m, spectral-fractal terrain (P(k) ~ k^-3,
seed 1, 0-3 m relief) with 200 circular depressions, a smooth melt-rate
field of 5-40 mm/day (seed 2) as a per-cell multiplier of the forcing rate,
Manning n ~ U[0.03, 0.15], one solute (D = 0.01 m^2/s). All inputs are seeded
synthetic stand-ins generated by fluxos_cpp_b200.scenarios. The state starts
wet (a 5 mm film plus water ponded in the depressions), as a snapshot taken
during melt would be.

A step is one iteration of the reference's loop (main.cpp:271-406): Courant
dt, melt forcing, the hydrodynamic update and the ADE sweep over all cells.
metric = cell-updates/s = cells x steps / device time. `value` is the FP32
state's rate; the FP64 path (the reference's arithmetic) runs the same steps
from the same start, and the FP32 depth/discharge error and both runs'
mass-balance error are measured on the states after those steps. With N
ranks each rank runs its own replica and value is the sum (weak scaling, no
collective).

Also reported on the same line (skipped with --no-mix / --no-serve):
* mix: the 64-scenario ensemble (sizes 256^2-2048^2) advanced as one FP32
  batch (autotuned tiles), against the same scenarios as an FP64 batch and
  run one by one on the plain FP64 path;
* serve: a bounded sample of the serving configuration's request stream
  through the continuous-batching loop, with p50/p99 latency;
* dambreak (--no-dambreak): the circular dam break (2048^2 cells of 1 m,
  2 m of water within 300 m, flat bed, Manning n 0.02, two solutes, 600 s)
  run to its horizon in FP64 and FP32: front position along 8 rays, depth
  and discharge error of FP32 against FP64, both water balances;
* results_writer (--no-writer): one Results file of the headline state
  written from rows compacted on the device, asynchronously, and by the
  host writer from downloaded grids (text into /dev/null).

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
# Algorithmic bytes per cell-update, per kernel: read + write of the flow
# state and the solute, read of the bed, wall flag, Manning n and melt field
# (B = 2w(3+ns) + w_zb + 1 + w_n + 4 with ns = 1):
#   FP64: hydro 2*8*3 (z, qx, qy) + 8 (zb) + 1 + 8 (n) + 8 (melt, stored as
#         FP64 here) = 73 B, ADE 2*8 = 16 B, step 89 B;
#   FP32: hydro 2*4*3 + 4 + 1 + 4 + 4 = 37 B, ADE 2*4 = 8 B, step 45 B.
# The FP32 layout moves more than that (the depth's compensation word and an
# FP64 bed: 49 B of hydro state); the roofline's `traffic` field gives what
# the kernel actually moved.
ALG_BYTES = {"fp64": {"k_hydro": 73, "k_ade_sweep": 16, "step": 89},
             "fp32": {"k_hydro": 37, "k_ade_sweep": 8, "step": 45}}
# DRAM bytes per cell that each kernel actually moves per step
# (dram__bytes_read.sum + dram__bytes_write.sum from ncu on the 2048 x 2048
# case of this workload, one launch, divided by the cells and the steps the
# launch covers); traffic scales with the cells, so `traffic` in the line is
# this times the cells of the run.
DRAM_BYTES_PER_CELL = {"fp64": {"k_hydro": 143.59, "k_ade_sweep": 61.35},
                       "fp32": {"k_hydro": 80.38, "k_ade_sweep": 26.65}}


def _rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(x: float, device: str = "cuda") -> float:
    """The largest of every rank's x (a job is as slow as its slowest
    replica), or x itself without a process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: float, world: int, seconds: float) -> float:
    """Whole-job throughput of `world` replicas that each processed
    `units_per_rank` units, timed as the slowest rank's `seconds`."""
    return units_per_rank * world / seconds


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

    def _lines(self) -> int:
        try:
            with open(self.path) as f:
                return sum(1 for ln in f if ln.count(",") >= 7)
        except Exception:
            return 0

    def start(self):
        """Start sampling and return once samples are flowing (nvidia-smi
        takes a moment to start); samples before this point are not kept."""
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.n0 = 0
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self.gpu_id, f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        t0 = time.time()
        while self._lines() == 0 and time.time() - t0 < 10.0:
            time.sleep(0.02)
        self.n0 = self._lines()

    def stop(self) -> dict:
        """Stop after one more sample than there was at the end of the timed
        region (so a short region still has one); keep the samples taken
        since start() returned."""
        if self.proc is not None:
            n1 = self._lines()
            t0 = time.time()
            while self._lines() <= n1 and time.time() - t0 < 1.0:
                time.sleep(0.01)
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
        rows = rows[getattr(self, "n0", 0):]
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
    """The large-domain scenario with a wet start: a 5 mm film plus water
    ponded in the depressions, solute 1 where the depth exceeds 10 mm."""
    from fluxos_cpp_b200 import scenarios as S
    sc = S.fractal_scenario(n, dxy=2, seed=seed, melt_seed=seed + 1, extensions=True)
    dem = sc.dem.astype(np.float64)
    film = 0.005
    h = film + np.maximum(S.box3(S.box3(dem)) - dem, 0.0)
    sc.init_h = h
    sc.init_qx = np.zeros_like(h)
    sc.init_qy = np.zeros_like(h)
    sc.init_conc = [np.where(h > 2 * film, 1.0, 0.0)]
    return sc


def build_domain(sc, in_flight: int = 8, precision: str = "fp64"):
    from fluxos_cpp_b200 import scenarios as S
    return S.make_domain(sc, precision=precision, steps_in_flight=in_flight)


def e2e_run(d, sc, steps: int, chunk: int):
    """Through the public API with host buffers: upload the state from
    pinned host memory, step in calls of `chunk` steps (the steps whose ADE
    sweeps run in one launch; every call reads back the control block, which
    holds each of its steps' dt and clock record), download the Results
    fields. Returns (seconds, h2d bytes, d2h bytes)."""
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
    ta = time.perf_counter()
    left, calls = steps, 0
    while left > 0:
        n = min(chunk, left)
        d.step(n)
        left -= n
        calls += 1
    tb = time.perf_counter()
    for k in names_dn:
        d.download(k, out[k])
    t1 = time.perf_counter()
    cells = shape[0] * shape[1]
    h2d = cells * (8 * len(names_up) + 8) + 8 * calls
    d2h = cells * 8 * len(names_dn) + 1600 * calls
    return t1 - t0, h2d, d2h, {"upload_s": round(ta - t0, 4), "steps_s": round(tb - ta, 4),
                               "download_s": round(t1 - tb, 4)}


def results_writer_timing(d, target: str = "/dev/null") -> dict:
    """One Results file of the current state three ways, into `target`:
    rows compacted on the device then formatted on host threads
    (fx_write_results); the same started with fx_write_results_async, whose
    return is all the stepping waits for; and the host writer on the ten
    downloaded grids."""
    import fluxos_cpp_b200 as fx
    t0 = time.perf_counter()
    d.write_results(target)
    t1 = time.perf_counter()
    d.write_results(target, wait=False)
    t2 = time.perf_counter()
    d.results_wait()
    t3 = time.perf_counter()
    g = {k: d.download(k) for k in ("z", "zb", "h", "qx", "qy", "conc", "soil_mass", "fe_1", "fn_1", "twet")}
    fx.write_results_host(target, d.nrows, d.ncols, d.dxy, d.xll, d.yll, d.h_min_print, g)
    t4 = time.perf_counter()
    rows = int(((g["zb"][1:-1, 1:-1] != 0) & (g["h"][1:-1, 1:-1] > d.h_min_print)).sum())
    return {"rows": rows, "device_compaction_s": t1 - t0, "async_start_s": t2 - t1,
            "async_total_s": t3 - t1, "host_from_downloads_s": t4 - t3,
            "note": "text into /dev/null; async_start_s is the stall the stepping sees"}


class _stdout_to_stderr:
    """The reference's start-up prints progress to stdout (fd 1); keep the
    one JSON line of this program alone there."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)
        return False


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
    with tempfile.TemporaryDirectory() as tmp, _stdout_to_stderr():
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


def measure_domain(d, steps: int, warmup: int, cells: int, precision: str, peak: float, gpu: str,
                   tile_rows: int = 0):
    """Autotune the tile shape (real steps, part of the warm-up) unless one is
    given, warm-up, then `steps` timed steps (CUDA events on the domain's
    stream around every launch, fx_time_steps); roofline of the dominant
    kernel."""
    if tile_rows:
        d.set_option("tile_rows", tile_rows)
    else:
        tile_rows = d.autotune(8)
    d.step(warmup)
    sampler = ClockSampler(gpu)
    sampler.start()
    ms_total, ms_hydro, ms_ade = d.time_steps(steps)
    clocks = sampler.stop()
    st = d.status()
    if st["device_error"]:
        raise RuntimeError("device error during the timed steps")
    alg = ALG_BYTES[precision]
    ms_h, ms_a = ms_hydro / steps, ms_ade / steps
    kern = {"k_hydro": ms_h, "k_ade_sweep": ms_a}
    dom = max(kern, key=kern.get)
    achieved = cells * alg[dom] / (kern[dom] / 1e3) / 1e9
    traffic = int(DRAM_BYTES_PER_CELL[precision][dom] * cells)
    roof = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": traffic,
            "traffic_note": "DRAM bytes per step of this kernel, ncu on the 2048^2 case scaled by cells",
            "alg_bytes_per_cell": alg[dom],
            "ms_per_step": {"k_hydro": round(ms_h, 4), "k_ade_sweep": round(ms_a, 4)},
            "step_alg_GBps": round(cells * alg["step"] / (ms_total / steps / 1e3) / 1e9, 1)}
    return {"ms_total": ms_total, "value": cells * steps / (ms_total / 1e3), "roofline": roof,
            "clocks": clocks, "tile_rows": tile_rows}


def accuracy_of(d32, d64, w32: float, w64: float, hdry: float) -> dict:
    from fluxos_cpp_b200 import accuracy as A
    e = A.state_errors(d32, d64, hdry)
    b32, b64 = A.water_balance(d32, w32), A.water_balance(d64, w64)
    return {"against": "FP64 path (itself within 1e-10 per cell of the reference, tests/test_gpu_parity.py)",
            "steps": int(d32.status()["steps"]),
            "depth_l1_rel": e["depth"]["l1_rel"], "depth_linf_m": e["depth"]["linf_abs"],
            "depth_linf_rel": e["depth"]["linf_rel"],
            "discharge_l1_rel": e["discharge"]["l1_rel"], "discharge_linf_m2s": e["discharge"]["linf_abs"],
            "solute_l1_rel": e["solute_mass_density"][0]["l1_rel"],
            "wet_cells_differ": e["wet_cells"]["differ"], "wet_cells": e["wet_cells"]["ref"],
            "mass_balance_rel_fp32": b32["rel_err"], "mass_balance_rel_fp64": b64["rel_err"]}


def run_mix(args, peak: float) -> dict:
    """The 64-scenario ensemble: FP32 batch vs FP64 batch vs FP64 one by one."""
    import torch
    import fluxos_cpp_b200 as fx
    from fluxos_cpp_b200 import scenarios as S
    from concurrent.futures import ThreadPoolExecutor
    t0 = time.perf_counter()
    scs = S.ensemble_scenarios(args.mix_count, seed=3)
    gen_s = time.perf_counter() - t0
    cells = [sc.nrows * sc.ncols for sc in scs]
    steps = args.mix_steps

    def batch_rate(precision):
        # FP32 members hold 63 steps in flight (82 GB for the 64 scenarios); FP64 ones
        # args.mix_in_flight (memory: FP64 slot planes are twice as large)
        k_members = 63 if precision == "fp32" else args.mix_in_flight
        doms = [S.make_domain(sc, precision=precision, steps_in_flight=k_members) for sc in scs]
        b = fx.Batch()
        for d in doms:
            b.add(d)
        tuned = b.autotune(4) if precision == "fp32" else (8, args.mix_in_flight)
        if precision == "fp64":
            b.set_option("steps_in_flight", args.mix_in_flight)
        b.step(args.warmup)
        s0 = [d.status()["steps"] for d in doms]
        stream = torch.cuda.ExternalStream(b.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        b.step(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        done = sum((d.status()["steps"] - a) * c for d, a, c in zip(doms, s0, cells))
        nbytes = sum(d.device_bytes() for d in doms)
        b.close()
        for d in doms:
            d.close()
        return done / (ms / 1e3), ms, tuned, nbytes

    r32, ms32, tuned, bytes32 = batch_rate("fp32")
    r64b, ms64b, _, bytes64 = batch_rate("fp64")
    # plain FP64 path: each scenario alone, one after another
    tot_ms, tot_cells = 0.0, 0
    for sc, c in zip(scs, cells):
        d = S.make_domain(sc, precision="fp64", steps_in_flight=args.mix_in_flight)
        d.step(args.warmup)
        s0 = d.status()["steps"]
        ms, _, _ = d.time_steps(steps)
        tot_ms += ms
        tot_cells += (d.status()["steps"] - s0) * c
        d.close()
    r64 = tot_cells / (tot_ms / 1e3)
    return {"scenarios": len(scs), "cells": int(sum(cells)), "sizes": f"{min(sc.nrows for sc in scs)}^2.."
            f"{max(sc.nrows for sc in scs)}^2 (log-uniform, seed 3)", "steps": steps,
            "fp32_batch_cell_updates_per_s": r32, "fp32_batch_ms": round(ms32, 3),
            "fp32_batch_alg_GBps": round(r32 * ALG_BYTES["fp32"]["step"] / 1e9, 1),
            "fp32_batch_hbm_frac": round(r32 * ALG_BYTES["fp32"]["step"] / 1e9 / peak, 4),
            "fp64_batch_cell_updates_per_s": r64b, "fp64_plain_cell_updates_per_s": r64,
            "fp32_batch_over_fp64_plain": round(r32 / r64, 3),
            "fp32_batch_over_fp64_batch": round(r32 / r64b, 3),
            "autotuned": {"tile_rows": tuned[0], "steps_in_flight": tuned[1]},
            "device_bytes_fp32": bytes32, "device_bytes_fp64": bytes64,
            "host_generation_s": round(gen_s, 1),
            "note": "per-scenario dt; timed region = one fx_batch_step of all members (CUDA events on "
                    "the batch stream); plain FP64 = each scenario alone through fx_time_steps"}


def front_radii(d, sc, hdry: float) -> list:
    """Largest distance from the dam's centre at which the depth exceeds
    hdry, along 8 rays (every 45 degrees), sampled every quarter cell."""
    h = d.download("h")[1:-1, 1:-1]  # [icol - 1, irow - 1]
    n, dxy = sc.nrows, sc.dxy
    out = []
    for k in range(8):
        a = k * np.pi / 4
        r = np.arange(0.0, n * dxy / 2 * 1.5, dxy / 4)
        x = n * dxy / 2 + r * np.cos(a)
        y = n * dxy / 2 + r * np.sin(a)
        ok = (x >= 0) & (x < n * dxy) & (y >= 0) & (y < n * dxy)
        r, ix, iy = r[ok], (x[ok] // dxy).astype(int), (y[ok] // dxy).astype(int)
        wet = h[iy, ix] > hdry
        out.append(float(r[wet].max()) if wet.any() else 0.0)
    return out


def run_dambreak(args) -> dict:
    """The circular dam break (2048^2 cells of 1 m, 2 m of water within 300 m
    of the centre, flat bed, Manning n 0.02, two solutes, 600 s): FP32 against
    FP64 at the horizon, with the front position along 8 rays and both water
    balances."""
    from fluxos_cpp_b200 import accuracy as A
    from fluxos_cpp_b200 import scenarios as S
    n = args.dambreak_size
    sc = S.dambreak_scenario(n, dxy=1, radius=300.0 * n / 2048, depth=2.0, base=100.0,
                             horizon=args.dambreak_horizon)
    out = {"cells": n * n, "horizon_s": sc.horizon, "radius_m": sc.extra["radius"]}
    doms, w0 = {}, {}
    for p in ("fp64", "fp32"):
        d = S.make_domain(sc, precision=p, steps_in_flight=31)
        w0[p] = d.mass()[0]
        t0 = time.perf_counter()
        st = d.run_to_print()  # one output, at the horizon
        out[f"{p}_steps"] = st["steps"]
        out[f"{p}_wall_s"] = round(time.perf_counter() - t0, 3)
        out[f"{p}_tim"] = st["tim"]
        doms[p] = d
    e = A.state_errors(doms["fp32"], doms["fp64"], sc.ks)
    out["depth_l1_rel"] = e["depth"]["l1_rel"]
    out["depth_linf_abs"] = e["depth"]["linf_abs"]
    out["discharge_l1_rel"] = e["discharge"]["l1_rel"]
    out["wet_cells_differ"] = e["wet_cells"]["differ"]
    out["solute_mass_l1_rel"] = [c["l1_rel"] for c in e["solute_mass_density"]]
    for p in ("fp64", "fp32"):
        d = doms[p]
        out[f"{p}_front_m"] = front_radii(d, sc, sc.ks)
        out[f"{p}_mass_rel_err"] = A.water_balance(d, w0[p])["rel_err"]
        out[f"{p}_solute_mass"] = [float(x) for x in d.mass()[1]]
        out[f"{p}_conc_max"] = [float(d.download("conc" if k == 0 else f"conc{k}").max())
                                for k in range(sc.nchem)]
        d.close()
    out["note"] = ("the initial concentration is at most 1; the reference's ADE scheme (restated "
                   "bit for bit by the FP64 path) is not bounded at D = 1.0 m^2/s on 1 m cells: "
                   "the second solute's concentrations grow by orders of magnitude and then "
                   "collapse to ~0, so solute errors between the precisions compare two "
                   "unstable runs")
    return out


def run_serve(args) -> dict:
    from fluxos_cpp_b200 import serve
    reqs = serve.poisson_requests(rate=4.0, duration=args.serve_seconds, seed=4,
                                  horizon_scale=args.serve_horizon_scale)
    srv = serve.Server(cap_bytes=150e9, chunk_steps=32)
    stats = srv.run(reqs)
    srv.close()
    stats.update({"arrivals": f"Poisson 4/s for {args.serve_seconds:g} s (seed 4)",
                  "grids": "128^2..4096^2 log-uniform", "solutes": "1-3",
                  "horizon": f"1-12 h x {args.serve_horizon_scale:g} (bounded sample)",
                  "admission_cap_bytes": 150e9, "precision": "fp32",
                  "latency": "arrival to retirement, including host-side input generation"})
    return stats


def run_gpu(args):
    import torch
    import torch.distributed as dist
    rank, world, local = _rank()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    n = args.size
    k_batch = args.in_flight  # steps per ADE launch
    sc = make_workload(n)
    h, conc = sc.init_h, sc.init_conc[0]
    cells = n * n
    peak, peak_kind = _peaks()
    gpu = gpu_id_of_device0()
    precs = ["fp32", "fp64"] if args.precision == "both" else [args.precision]
    doms, w0, res = {}, {}, {}
    for p in precs:
        doms[p] = build_domain(sc, k_batch, p)
        w0[p] = doms[p].mass()[0]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    for p in precs:
        res[p] = measure_domain(doms[p], args.steps, args.warmup, cells, p, peak, gpu, args.tile_rows)
    torch.cuda.synchronize()
    head = precs[0]
    ms_max = max_over_ranks(res[head]["ms_total"])
    if world > 1:
        dist.barrier()
    value = job_rate(cells * args.steps, world, ms_max / 1e3)
    acc = None
    if len(precs) == 2:
        acc = accuracy_of(doms["fp32"], doms["fp64"], w0["fp32"], w0["fp64"], sc.ks)
    e2e = None
    if not args.no_e2e:
        secs, h2d, d2h, parts = e2e_run(doms[head], sc, args.steps, k_batch)
        secs = max_over_ranks(secs)
        e2e = {"value": job_rate(cells * args.steps, world, secs), "unit": "cell-updates/s", "parts": parts,
               "h2d_bytes_per_step": int(h2d / args.steps), "d2h_bytes_per_step": int(d2h / args.steps),
               "note": "upload of the state from pinned host memory, the K steps through fx_step in "
                       "calls of steps-in-flight steps (each call reads the control block with every "
                       "step's record back), download of the Results fields; per-step bytes = totals / K"}
    writer = None
    if rank == 0 and world == 1 and not args.no_writer:
        writer = results_writer_timing(doms[head])
    for d in doms.values():
        d.close()
    batches = (args.steps + k_batch - 1) // k_batch
    launches = 2 * args.steps + 2 * batches  # finalize + hydro per step; batch open + sweep per batch
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_reference_run(sc, h, conc, 1, args.cpu_steps, args.cpu_crop)
    mix = run_mix(args, peak) if (rank == 0 and world == 1 and not args.no_mix) else None
    dam = run_dambreak(args) if (rank == 0 and world == 1 and not args.no_dambreak) else None
    srv = run_serve(args) if (rank == 0 and world == 1 and not args.no_serve) else None
    if rank == 0:
        roof = dict(res[head]["roofline"])
        roof["peak_source"] = peak_kind
        line = {"metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32" if head == "fp32" else "f64",
                "data": "synthetic (seeded fractal terrain, melt field and Manning n)",
                "config": {"workload": f"fractal {n}x{n} cells of 2 m, 200 depressions, melt field "
                                       f"5-40 mm/day, Manning n U[0.03,0.15], one solute, wet start",
                           "precision": head + (" (FP64 clock, wet/dry threshold tests and budget)"
                                                if head == "fp32" else " (the reference's arithmetic)"),
                           "cells": cells,
                           "l2": "inputs larger than L2 (4-8 GB of state per replica)",
                           "parallelism": f"replicas x{world}"},
                "roofline": roof, "e2e": e2e, "gpu_launches": launches, "clocks": res[head]["clocks"],
                "cpu_baseline": cpu, "accuracy": acc,
                "autotuned": {"tile_rows": res[head]["tile_rows"]}}
        if "fp64" in res and head != "fp64":
            line["fp64"] = {"value": res["fp64"]["value"], "ms_per_step": res["fp64"]["ms_total"] / args.steps,
                            "autotuned": {"tile_rows": res["fp64"]["tile_rows"]},
                            "roofline": res["fp64"]["roofline"], "clocks": res["fp64"]["clocks"]}
            line["fp32_over_fp64"] = round(res[head]["value"] / res["fp64"]["value"], 3)
        if writer is not None:
            line["results_writer"] = writer
        if mix is not None:
            line["mix"] = mix
        if dam is not None:
            line["dambreak"] = dam
        if srv is not None:
            line["serve"] = srv
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def run_reference(args):
    rank, world, local = _rank()
    if rank != 0:
        return
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    sc = make_workload(args.size)
    h, conc = sc.init_h, sc.init_conc[0]
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
    ap.add_argument("--steps", type=int, default=63)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=("b200", "reference"))
    ap.add_argument("--size", type=int, default=4096)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-crop", type=int, default=2048)
    ap.add_argument("--cpu-steps", type=int, default=12)
    ap.add_argument("--in-flight", type=int, default=63, help="steps per ADE launch (1..63)")
    ap.add_argument("--mix-in-flight", type=int, default=31,
                    help="steps in flight of the FP64 ensemble members (memory: slot planes per step)")
    ap.add_argument("--precision", default="both", choices=("both", "fp64", "fp32"),
                    help="both: FP32 headline with FP64 beside it and the FP32 error")
    ap.add_argument("--no-mix", action="store_true")
    ap.add_argument("--no-writer", action="store_true", help="skip the Results writer timing")
    ap.add_argument("--no-dambreak", action="store_true")
    ap.add_argument("--tile-rows", type=int, default=0, choices=(0, 4, 8, 16),
                    help="hydrodynamic tile shape (0: autotune)")
    ap.add_argument("--dambreak-size", type=int, default=2048)
    ap.add_argument("--dambreak-horizon", type=float, default=600.0)
    ap.add_argument("--mix-count", type=int, default=64)
    ap.add_argument("--mix-steps", type=int, default=62)
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--serve-seconds", type=float, default=20.0)
    ap.add_argument("--serve-horizon-scale", type=float, default=1.0 / 120.0)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()

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
  host writer from downloaded grids (text into /dev/null);
* c1 (--no-c1): the small CPU configuration (200 x 200 plane with bumps, dry
  start, 6 h of melt, 36 Results files) run in full: the drop-in program
  fluxos_gpu (FP64) end to end, the same run's stepping timed on the device,
  and the reference program (oracle/_ref) on all host cores;
* parity_crop (with the CPU leg): the GPU FP64 path in parity mode on
  exactly the crop the reference times (2048^2, uniform melt at the field
  mean, no Manning, the same wet start), its state compared cell by cell with
  the reference's after the same steps, and its rate beside the reference's:
  the like-for-like ratio.

--impl reference times the FLUXOS reference sources compiled in oracle/_ref
(OpenMP hydrodynamics, serial ADE) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
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
             "fp32": {"k_hydro": 37, "k_ade_sweep": 8, "step": 45},
             # parity mode (no Manning n, no melt field): 2*8*3 + 8 + 1 = 57 B hydro
             "fp64_parity": {"k_hydro": 57, "k_ade_sweep": 16, "step": 73}}
# DRAM bytes per cell that each kernel actually moves per step
# (dram__bytes_read.sum + dram__bytes_write.sum from ncu on the 2048 x 2048
# case of this workload at 20 steps in flight, one launch, divided by the
# cells and the steps the launch covers; the FP32 hydrodynamic kernel with
# 16-row tiles, the FP64 one with 8-row tiles, the shapes the autotuner
# picks; the captures are summarised in profiles/); traffic scales with the
# cells, so `traffic` in the line is this times the cells of the run.
DRAM_BYTES_PER_CELL = {"fp64": {"k_hydro": 152.81, "k_ade_sweep": 55.78},
                       "fp32": {"k_hydro": 91.08, "k_ade_sweep": 34.86}}


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


def crop_scenario(sc, crop: int):
    """A square crop of the workload in parity mode: the reference has no
    melt field and no Manning term, so the melt is the field's mean rate,
    uniform, and there is no friction."""
    from fluxos_cpp_b200 import scenarios as S
    n = min(crop, sc.nrows)
    return S.Scenario(name=f"crop{n}", dem=sc.dem[:n, :n].copy(), dxy=sc.dxy, meteo=sc.meteo,
                      horizon=sc.horizon, print_step=sc.print_step, ks=sc.ks, ade=True, d_coef=sc.d_coef)


def cpu_reference_run(sc, h, conc, warmup: int, steps: int, crop: int, keep: bool = False):
    """The reference sources (oracle/_ref) on a crop of the same workload,
    in parity mode. With keep, the result also holds the reference run (its
    state after warmup + steps steps) and the crop's input folder, which the
    caller removes."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as P
    if not P.ref_available(0):
        return None
    sub = crop_scenario(sc, crop)
    n = sub.nrows
    tmp = tempfile.mkdtemp(prefix="fluxos_crop_")
    with _stdout_to_stderr():
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
    out = {"value": n * n * steps / (t1 - t0), "unit": "cell-updates/s", "cores": threads,
           "kind": "reference", "seconds": t1 - t0,
           "sample": f"{n}x{n} crop of the workload (uniform melt at the field mean, no Manning: "
                     f"the reference has neither), {warmup} warm-up + {steps} timed steps, "
                     f"reference sources from oracle/_ref, OpenMP hydrodynamics on {threads} threads, "
                     f"serial ADE"}
    if keep:
        out.update(_ref=ref, _dir=tmp, _modset=mp, _sub=sub)
    else:
        del ref
        shutil.rmtree(tmp, ignore_errors=True)
    return out


PARITY_FIELDS = ("z", "h", "qx", "qy", "conc", "twet", "h0", "fe_1", "fe_2", "fe_3", "fn_1", "fn_2", "fn_3")


def run_parity_crop(cpu: dict, h, conc, steps: int, in_flight: int, peak: float) -> dict:
    """The GPU FP64 path on the reference's crop, from the same input files
    and the same wet start: after the reference's warm-up + timed steps, the
    largest relative difference per field (floored at 1e-6 of the field's
    largest magnitude) and the wet/dry flags that differ; then `steps` steps
    timed with CUDA events beside the reference's rate."""
    import fluxos_cpp_b200 as fx
    ref, sub, mp = cpu["_ref"], cpu["_sub"], cpu["_modset"]
    n = sub.nrows
    ncmp = int(ref.scalar("it"))
    d = fx.Domain.from_modset_state(mp, steps_in_flight=in_flight)
    try:
        d.set_option("store_all_fluxes", 1)  # fe_2, fe_3, fn_2, fn_3 of wet cells too, as GlobVar holds them
        # the wet start exactly as the reference run got it (RefRun.apply_wet_start)
        zb, z, hh, cc = d.download("zb"), d.download("z"), d.download("h"), d.download("conc")
        hh[1:-1, 1:-1] = h[:n, :n].T
        z[1:-1, 1:-1] = zb[1:-1, 1:-1] + h[:n, :n].T
        cc[1:-1, 1:-1] = conc[:n, :n].T
        for k, g in (("z", z), ("h", hh), ("conc", cc)):
            d.upload(k, g)
        fl = d.download_flags()
        ld = fl["ldry"].copy()
        ld[1:-1, 1:-1] = np.where(h[:n, :n].T > 0, 0.0, 1.0)
        d.upload_flags(ld, fl["wall"])
        d.prepare()
        done = 0
        while done < ncmp:
            st = d.step(ncmp - done)
            done = int(st["it"])
            if st["finished"]:
                break
        errs = {}
        for k in PARITY_FIELDS:
            a, b = ref.grid(k)[1:-1, 1:-1], d.download(k)[1:-1, 1:-1]
            scale = max(float(np.abs(a).max()), 1e-300) * 1e-6
            errs[k] = 0.0 if np.array_equal(a, b) else float(
                (np.abs(a - b) / np.maximum(np.maximum(np.abs(a), np.abs(b)), scale)).max())
        fl = d.download_flags()
        flags_differ = int((fl["ldry"][1:-1, 1:-1] != ref.grid("ldry")[1:-1, 1:-1]).sum())
        tim_equal = d.status()["tim"] == ref.scalar("tim")
        ms, ms_h, ms_a = d.time_steps(steps)
        gpu_rate = n * n * steps / (ms / 1e3)
    finally:
        d.close()
        del cpu["_ref"]
        shutil.rmtree(cpu.pop("_dir"), ignore_errors=True)
        cpu.pop("_modset")
        cpu.pop("_sub")
    return {"cells": n * n, "steps_compared": ncmp, "max_rel_err": errs,
            "max_rel_err_all": max(errs.values()), "flags_differ": flags_differ, "clock_equal": bool(tim_equal),
            "gpu_fp64_cell_updates_per_s": gpu_rate, "gpu_ms_per_step": ms / steps,
            "gpu_ms_per_step_hydro_ade": [round(ms_h / steps, 4), round(ms_a / steps, 4)],
            "gpu_alg_GBps": round(gpu_rate * ALG_BYTES["fp64_parity"]["step"] / 1e9, 1),
            "gpu_hbm_frac": round(gpu_rate * ALG_BYTES["fp64_parity"]["step"] / 1e9 / peak, 4),
            "cpu_reference_cell_updates_per_s": cpu["value"], "cpu_cores": cpu["cores"],
            "gpu_over_cpu": round(gpu_rate / cpu["value"], 1),
            "note": "same input files, same wet start, FP64 on both sides, parity mode (uniform melt, no "
                    "Manning); state compared after the reference's warm-up + timed steps; GPU rate from "
                    f"{steps} further steps timed with CUDA events (state larger than L2)"}


def run_c1(args) -> dict:
    """The small CPU configuration run in full: 200 x 200 cells of 2 m, dry
    start, 20 mm/day for 6 h, 36 Results files. The drop-in program
    fluxos_gpu (FP64, files written) end to end; the same run's stepping on
    the device alone (a context from the same modset, run to each output, no
    files; CUDA events on the context's stream); the reference program
    (oracle/_ref/fluxos_ref, OpenMP on all host cores) end to end."""
    import torch
    import fluxos_cpp_b200 as fx
    from fluxos_cpp_b200 import scenarios as S
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as P
    sc = S.plane_scenario()
    cells = sc.nrows * sc.ncols
    out = {"workload": "plane 200x200 cells of 2 m with smoothed bumps (seed 0), dry start, 20 mm/day "
                       "for 6 h at 1 mg/L, D 0.01 m^2/s, output every 600 s (36 Results files)",
           "precision": "fp64 (the reference's arithmetic)"}
    with tempfile.TemporaryDirectory() as tmp:
        mp = sc.write(tmp)
        t0 = time.perf_counter()
        r = subprocess.run([fx.EXE_PATH, mp], capture_output=True, text=True)
        out["gpu_program_s"] = round(time.perf_counter() - t0, 3)
        if r.returncode != 0:
            raise RuntimeError("fluxos_gpu failed: " + r.stderr[-500:])
        out["results_files"] = len(os.listdir(os.path.join(tmp, "Results")))
        d = fx.Domain.from_modset_state(mp, steps_in_flight=args.c1_in_flight)
        stream = torch.cuda.ExternalStream(d.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0.record(stream)
        while True:
            st = d.run_to_print()
            if st["print_pending"]:
                d.print_done()
                continue
            if st["finished"]:
                break
        e1.record(stream)
        torch.cuda.synchronize()
        host_s = time.perf_counter() - t0
        it, steps = int(st["it"]), int(st["steps"])
        d.close()
        updates = it * cells  # cells advanced in every step the solver runs (hpall != 0)
        out.update({"iterations": steps, "solver_iterations": it, "cell_updates": updates,
                    "steps_in_flight": args.c1_in_flight,
                    "gpu_steps_device_s": round(e0.elapsed_time(e1) / 1e3, 4),
                    "gpu_steps_host_s": round(host_s, 4),
                    "gpu_cell_updates_per_s": updates / (e0.elapsed_time(e1) / 1e3),
                    "gpu_program_cell_updates_per_s": updates / out["gpu_program_s"]})
        if P.ref_available(0) and not args.no_c1_ref:
            ref_dir = os.path.join(tmp, "ref")
            mp2 = sc.write(ref_dir)
            threads = os.cpu_count() or 1
            env = dict(os.environ, OMP_NUM_THREADS=str(threads))
            t0 = time.perf_counter()
            r = subprocess.run([P.REF_BIN, mp2], capture_output=True, text=True, env=env)
            ref_s = time.perf_counter() - t0
            if r.returncode == 0:
                out.update({"reference_program_s": round(ref_s, 3), "reference_cores": threads,
                            "reference_cell_updates_per_s": updates / ref_s,
                            "gpu_program_over_reference": round(ref_s / out["gpu_program_s"], 1)})
    out["note"] = ("program times are wall clock of the whole process (start-up, 46k steps, 36 files of "
                   "text); the state (2 MB) is L2-resident, so the GPU stepping is launch-bound, not a "
                   "roofline case")
    return out


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


def mix_accuracy(st32: list, st64: list) -> dict:
    """FP32 batch against FP64 batch, member by member after the same steps:
    relative L1 and absolute L-infinity depth and discharge error (|q|), per
    member and over all members, and both precisions' water balances."""
    per, num_h, den_h, num_q, den_q = [], 0.0, 0.0, 0.0, 0.0
    linf_h = linf_q = 0.0
    for a, b in zip(st32, st64):
        dh, dq = np.abs(a["h"] - b["h"]), np.abs(a["q"] - b["q"])
        sh, sq = float(np.abs(b["h"]).sum()), float(np.abs(b["q"]).sum())
        num_h, den_h, num_q, den_q = num_h + float(dh.sum()), den_h + sh, num_q + float(dq.sum()), den_q + sq
        linf_h, linf_q = max(linf_h, float(dh.max())), max(linf_q, float(dq.max()))
        per.append({"depth_l1_rel": float(dh.sum()) / sh if sh else 0.0, "depth_linf_m": float(dh.max()),
                    "discharge_l1_rel": float(dq.sum()) / sq if sq else 0.0,
                    "same_steps": a["steps"] == b["steps"], "tim_fp32": a["tim"], "tim_fp64": b["tim"]})
    d_l1 = [p["depth_l1_rel"] for p in per]
    return {"against": "the FP64 batch (each member the reference's arithmetic) after the same steps",
            "depth_l1_rel": num_h / den_h, "depth_linf_m": linf_h,
            "discharge_l1_rel": num_q / den_q, "discharge_linf_m2s": linf_q,
            "depth_l1_rel_per_member": {"max": max(d_l1), "median": float(np.median(d_l1)),
                                        "all": [float(f"{x:.3g}") for x in d_l1]},
            "discharge_l1_rel_max_member": max(p["discharge_l1_rel"] for p in per),
            "members_with_equal_steps": sum(p["same_steps"] for p in per),
            "mass_balance_rel_fp32_max": max(a["mass_rel_err"] for a in st32),
            "mass_balance_rel_fp64_max": max(b["mass_rel_err"] for b in st64)}


def mix_envelope(scs: list, steps: list, count: int) -> dict:
    """The scheme's own sensitivity on some of the ensemble's scenarios (the
    smallest `count`): each runs alone in FP32, in FP64 and in two FP64 copies
    whose initial depths are perturbed by a relative 1e-7, for the steps its
    batch member ran; the relative L1 depth error of FP32 and of the
    perturbed runs against FP64."""
    from fluxos_cpp_b200 import accuracy as A
    from fluxos_cpp_b200 import scenarios as S
    order = sorted(range(len(scs)), key=lambda i: scs[i].nrows)[:count]
    rows = []
    for i in order:
        sc, n = scs[i], steps[i]
        runs = [S.make_domain(sc, precision="fp32", steps_in_flight=8),
                S.make_domain(sc, precision="fp64", steps_in_flight=8)]
        runs += [_perturbed(sc, seed, in_flight=8) for seed in (0, 1)]
        for d in runs:
            left = n
            while left > 0:
                st = d.step(left)
                if st["print_pending"]:
                    d.print_done()
                left = n - st["steps"]
                if st["finished"]:
                    break
        ref = runs[1]
        e32 = A.state_errors(runs[0], ref, sc.ks)["depth"]["l1_rel"]
        ep = [A.state_errors(d, ref, sc.ks)["depth"]["l1_rel"] for d in runs[2:]]
        rows.append({"scenario": i, "cells": sc.nrows * sc.ncols, "steps": n, "fp32_depth_l1_rel": e32,
                     "perturbed_fp64_depth_l1_rel": ep, "fp32_over_envelope": e32 / max(ep) if max(ep) else None})
        for d in runs:
            d.close()
    return {"what": "members run alone: FP32 and two FP64 runs with initial depths perturbed by a relative "
                    "1e-7, each against FP64, after the steps of the batch run", "members": rows}


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

    def batch_rate(precision, match_steps=None):
        # FP32 members hold 63 steps in flight (about 130 GB for the 64 scenarios: a
        # 33-byte slot record per cell and step); FP64 ones args.mix_in_flight (41 bytes)
        from fluxos_cpp_b200 import accuracy as A
        k_members = 63 if precision == "fp32" else args.mix_in_flight
        doms = [S.make_domain(sc, precision=precision, steps_in_flight=k_members) for sc in scs]
        w0 = [d.mass()[0] for d in doms]
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
        # the members' states after the timed steps (interior depth and
        # discharge on the host) and their water balances, for the error of
        # FP32 against FP64; with match_steps, each member first steps on
        # alone to the other precision's step count (the autotuner's trial
        # steps advance the members too)
        if match_steps is not None:
            b.close()
            for d, n in zip(doms, match_steps):
                left = n - d.status()["steps"]
                while left > 0:
                    st = d.step(left)
                    if st["print_pending"]:
                        d.print_done()
                    left = n - st["steps"]
                    if st["finished"]:
                        break
        states = []
        for d, w in zip(doms, w0):
            st = d.status()
            states.append({"h": d.download("h")[1:-1, 1:-1].copy(),
                           "q": np.hypot(d.download("qx")[1:-1, 1:-1], d.download("qy")[1:-1, 1:-1]),
                           "steps": int(st["steps"]), "tim": st["tim"],
                           "mass_rel_err": A.water_balance(d, w)["rel_err"]})
        if match_steps is None:
            b.close()
        for d in doms:
            d.close()
        return done / (ms / 1e3), ms, tuned, nbytes, states

    r32, ms32, tuned, bytes32, st32 = batch_rate("fp32")
    envelope = mix_envelope(scs, [x["steps"] for x in st32], args.mix_envelope_members)
    r64b, ms64b, _, bytes64, st64 = batch_rate("fp64", match_steps=[x["steps"] for x in st32])
    acc = mix_accuracy(st32, st64)
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
            "host_generation_s": round(gen_s, 1), "accuracy": acc, "accuracy_envelope": envelope,
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


def _perturbed(sc, seed: int, in_flight: int = 31):
    """An FP64 domain of the scenario whose initial depths are perturbed by
    a relative 1e-7 (seeded, uniform in [-1, 1]): about one FP32 rounding."""
    from fluxos_cpp_b200 import scenarios as S
    d = S.make_domain(sc, precision="fp64", steps_in_flight=in_flight)
    h, z = d.download("h"), d.download("z")
    dh = h * 1e-7 * np.random.default_rng(seed).uniform(-1, 1, h.shape)
    d.upload("h", h + dh)
    d.upload("z", z + dh)
    d.prepare()
    return d


def _linf_at(a, b, sc) -> dict:
    """Where |a - b| of two interior depth grids is largest: the cell, its
    distance from the grid centre and both depths."""
    diff = np.abs(a - b)
    ic, ir = np.unravel_index(int(np.argmax(diff)), diff.shape)  # [icol - 1, irow - 1]
    x, y = (ic + 0.5) * sc.dxy - sc.ncols * sc.dxy / 2, (ir + 0.5) * sc.dxy - sc.nrows * sc.dxy / 2
    return {"irow": int(ir) + 1, "icol": int(ic) + 1, "r_m": round(float(np.hypot(x, y)), 2),
            "abs": float(diff[ic, ir]), "depth_test": float(a[ic, ir]), "depth_ref": float(b[ic, ir])}


def run_dambreak(args) -> dict:
    """The circular dam break (2048^2 cells of 1 m, 2 m of water within 300 m
    of the centre, flat bed, Manning n 0.02, two solutes, 600 s): FP32 against
    FP64 at the horizon, with the front position along 8 rays and both water
    balances. Two FP64 runs whose initial depths are perturbed by a relative
    1e-7 give the scheme's own sensitivity to one rounding (the envelope the
    FP32 error is read against); every 60 s of the run the depth error of
    FP32 and of the perturbed runs against FP64 is recorded, with the cell of
    the largest difference."""
    from fluxos_cpp_b200 import accuracy as A
    from fluxos_cpp_b200 import scenarios as S
    n = args.dambreak_size
    sc = S.dambreak_scenario(n, dxy=1, radius=300.0 * n / 2048, depth=2.0, base=100.0,
                             horizon=args.dambreak_horizon)
    sc.print_step = int(min(60, sc.horizon))
    out = {"cells": n * n, "horizon_s": sc.horizon, "radius_m": sc.extra["radius"]}
    doms, w0 = {}, {}
    for p in ("fp64", "fp32"):
        doms[p] = S.make_domain(sc, precision=p, steps_in_flight=31)
        w0[p] = doms[p].mass()[0]
    pert = [_perturbed(sc, seed) for seed in (0, 1)] if not args.no_envelope else []
    history = []
    wall = {"fp64": 0.0, "fp32": 0.0}
    while True:
        for p in ("fp64", "fp32"):
            t0 = time.perf_counter()
            doms[p].run_to_print()
            wall[p] += time.perf_counter() - t0
        for d in pert:
            d.run_to_print()
        t_out = doms["fp64"].status()["tim"]
        h64 = doms["fp64"].download("h")[1:-1, 1:-1]
        h32 = doms["fp32"].download("h")[1:-1, 1:-1]
        rec = {"t": round(t_out, 3), "fp32_depth_l1_rel": float(np.abs(h32 - h64).sum() / np.abs(h64).sum()),
               "fp32_linf": _linf_at(h32, h64, sc)}
        if pert:
            hp = [d.download("h")[1:-1, 1:-1] for d in pert]
            rec["perturbed_depth_l1_rel"] = [float(np.abs(x - h64).sum() / np.abs(h64).sum()) for x in hp]
            rec["perturbed_linf"] = [_linf_at(x, h64, sc) for x in hp]
        history.append(rec)
        if all(d.status()["finished"] or d.status()["tim"] >= sc.horizon for d in doms.values()):
            break
        for d in list(doms.values()) + pert:
            if d.status()["print_pending"]:
                d.print_done()
    for p in ("fp64", "fp32"):
        st = doms[p].status()
        out[f"{p}_steps"] = int(st["steps"])
        out[f"{p}_wall_s"] = round(wall[p], 3)
        out[f"{p}_tim"] = st["tim"]
    e = A.state_errors(doms["fp32"], doms["fp64"], sc.ks)
    out["depth_l1_rel"] = e["depth"]["l1_rel"]
    out["depth_linf_abs"] = e["depth"]["linf_abs"]
    out["discharge_l1_rel"] = e["discharge"]["l1_rel"]
    out["wet_cells_differ"] = e["wet_cells"]["differ"]
    out["solute_mass_l1_rel"] = [c["l1_rel"] for c in e["solute_mass_density"]]
    out["depth_linf_at"] = history[-1]["fp32_linf"]
    if pert:
        ep = [A.state_errors(d, doms["fp64"], sc.ks) for d in pert]
        out["envelope"] = {"what": "two FP64 runs with initial depths perturbed by a relative 1e-7, "
                                   "against the unperturbed FP64 run",
                           "depth_l1_rel": [x["depth"]["l1_rel"] for x in ep],
                           "depth_linf_abs": [x["depth"]["linf_abs"] for x in ep],
                           "discharge_l1_rel": [x["discharge"]["l1_rel"] for x in ep],
                           "wet_cells_differ": [x["wet_cells"]["differ"] for x in ep]}
        lim = max(out["envelope"]["depth_l1_rel"])
        out["fp32_depth_l1_over_envelope"] = round(out["depth_l1_rel"] / lim, 3) if lim > 0 else None
    out["history"] = history
    for p in ("fp64", "fp32"):
        d = doms[p]
        out[f"{p}_front_m"] = front_radii(d, sc, sc.ks)
        out[f"{p}_mass_rel_err"] = A.water_balance(d, w0[p])["rel_err"]
        out[f"{p}_solute_mass"] = [float(x) for x in d.mass()[1]]
        out[f"{p}_conc_max"] = [float(d.download("conc" if k == 0 else f"conc{k}").max())
                                for k in range(sc.nchem)]
        d.close()
    for d in pert:
        d.close()
    out["note"] = ("the initial concentration is at most 1; the reference's ADE scheme (restated "
                   "bit for bit by the FP64 path) is not bounded at D = 1.0 m^2/s on 1 m cells: "
                   "the second solute's concentrations grow by orders of magnitude and then "
                   "collapse to ~0, so solute errors between the precisions compare two "
                   "unstable runs")
    return out


def serve_accuracy(reqs: list, count: int) -> dict:
    """The FP32 error of served requests: the `count` smallest run alone to
    their horizons (the same states as in the batch: the serving test checks
    that each result is bit-identical alone and in the mix) in FP32, FP64 and
    two FP64 copies with depths perturbed by a relative 1e-7; the relative L1
    depth error of FP32 and of the perturbed runs against FP64."""
    from fluxos_cpp_b200 import accuracy as A
    from fluxos_cpp_b200 import scenarios as S
    rows = []
    for r in sorted(reqs, key=lambda x: x.cells)[:count]:
        sc = r.make()
        runs = [S.make_domain(sc, precision="fp32", steps_in_flight=r.steps_in_flight),
                S.make_domain(sc, precision="fp64", steps_in_flight=r.steps_in_flight)]
        runs += [_perturbed(sc, seed, in_flight=r.steps_in_flight) for seed in (0, 1)]
        w0 = [d.mass()[0] for d in runs]
        for d in runs:
            while True:
                st = d.step(512)
                if st["print_pending"]:
                    d.print_done()
                if st["finished"]:
                    break
        e32 = A.state_errors(runs[0], runs[1], sc.ks)
        ep = [A.state_errors(d, runs[1], sc.ks)["depth"]["l1_rel"] for d in runs[2:]]
        rows.append({"request": r.rid, "cells": r.cells, "horizon_s": sc.horizon, "solutes": sc.nchem,
                     "steps": int(runs[0].status()["steps"]),
                     "fp32_depth_l1_rel": e32["depth"]["l1_rel"], "fp32_depth_linf_m": e32["depth"]["linf_abs"],
                     "fp32_discharge_l1_rel": e32["discharge"]["l1_rel"],
                     "perturbed_fp64_depth_l1_rel": ep,
                     "fp32_mass_rel_err": A.water_balance(runs[0], w0[0])["rel_err"],
                     "fp64_mass_rel_err": A.water_balance(runs[1], w0[1])["rel_err"]})
        for d in runs:
            d.close()
    return {"what": "the smallest requests run alone to their horizons: FP32, and two FP64 runs with depths "
                    "perturbed by a relative 1e-7, against FP64", "requests": rows}


def run_serve(args, rank: int = 0, world: int = 1):
    """The serving configuration's request stream (Poisson arrivals at
    4/s, seed 4, grids 128^2-4096^2, 1-12 h horizons, 1-3 solutes, FP32,
    admission capped at 150 GB) over a bounded arrival window, with the
    horizons scaled (printed, with the reason); inputs generated ahead of
    arrival, off the latency clock. With several ranks each serves its share
    (serve.shard) on its own GPU and rank 0 merges the records. Returns the
    merged figures on rank 0, None elsewhere."""
    import torch.distributed as dist
    from fluxos_cpp_b200 import serve
    reqs = serve.poisson_requests(rate=4.0, duration=args.serve_seconds, seed=4,
                                  horizon_scale=args.serve_horizon_scale)
    srv = serve.Server(cap_bytes=150e9, chunk_steps=31)
    srv.run(serve.shard(reqs, rank, world), generate_ahead=args.serve_generate_ahead, generator_threads=8)
    part = srv.last_part
    srv.close()
    if world > 1:
        parts = [None] * world
        dist.all_gather_object(parts, part)
    else:
        parts = [part]
    if rank != 0:
        return None
    stats = serve.summarize(parts)
    stats["accuracy_sample"] = serve_accuracy(reqs, args.serve_accuracy_requests)
    # the load the configuration's full horizons would offer: the same
    # requests' measured steps per simulated second, over unscaled horizons
    full_offer = (stats["offered_cell_updates_per_s"] / args.serve_horizon_scale
                  if stats["offered_cell_updates_per_s"] else None)
    stats.update({"arrivals": f"Poisson 4/s for {args.serve_seconds:g} s (seed 4; the configuration: 600 s)",
                  "grids": "128^2..4096^2 log-uniform", "solutes": "1-3",
                  "horizon": f"1-12 h x {args.serve_horizon_scale:g}",
                  "offered_cell_updates_per_s_full_horizons": full_offer,
                  "horizon_scale_reason": "with 1-12 h horizons the stream offers about "
                                          f"{(full_offer or 0) / 1e9:.0f} G cell-updates/s, far beyond one "
                                          "GPU (every request would wait without bound); scaled horizons "
                                          "keep the arrival process and grid sizes and put the offered load "
                                          "at about 85 % of what one GPU serves (x 1/100 offers 2.4 G, served "
                                          "at 2.3 G with the GPU stepping 87 % of the time and a growing "
                                          "queue), so latency measures the solver and the admission, not a "
                                          "queue at saturation",
                  "admission_cap_bytes": 150e9, "precision": "fp32",
                  "latency": "arrival to retirement; inputs generated ahead of arrival (off the clock); parts: "
                             "admission wait (arrival to preparation start), preparation (context creation "
                             "and upload), join wait, device residency (in the batch until retirement)",
                  "ranks": world})
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
    cpu = crop = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_reference_run(sc, h, conc, 1, args.cpu_steps, args.cpu_crop, keep=True)
        if cpu is not None:
            crop = run_parity_crop(cpu, h, conc, args.steps, k_batch, peak)
    c1 = run_c1(args) if (rank == 0 and world == 1 and not args.no_c1) else None
    mix = run_mix(args, peak) if (rank == 0 and world == 1 and not args.no_mix) else None
    dam = run_dambreak(args) if (rank == 0 and world == 1 and not args.no_dambreak) else None
    srv = run_serve(args, rank, world) if not args.no_serve else None
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
                           "parallelism": f"replicas x{world}",
                           "reference_arm": f"the reference's CPU path on a {min(args.cpu_crop, n)}^2 crop "
                                            "of this workload in parity mode (uniform melt at the field "
                                            "mean, no Manning), FP64: not this configuration; the "
                                            "like-for-like GPU rate on that crop is "
                                            "parity_crop.gpu_fp64_cell_updates_per_s"},
                "roofline": roof, "e2e": e2e, "gpu_launches": launches, "clocks": res[head]["clocks"],
                "cpu_baseline": cpu, "accuracy": acc,
                "autotuned": {"tile_rows": res[head]["tile_rows"]}}
        if "fp64" in res and head != "fp64":
            line["fp64"] = {"value": res["fp64"]["value"], "ms_per_step": res["fp64"]["ms_total"] / args.steps,
                            "autotuned": {"tile_rows": res["fp64"]["tile_rows"]},
                            "roofline": res["fp64"]["roofline"], "clocks": res["fp64"]["clocks"]}
            line["fp32_over_fp64"] = round(res[head]["value"] / res["fp64"]["value"], 3)
        if crop is not None:
            line["parity_crop"] = crop
        if c1 is not None:
            line["c1"] = c1
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
    ap.add_argument("--no-envelope", action="store_true",
                    help="dam break without the two perturbed FP64 runs")
    ap.add_argument("--mix-count", type=int, default=64)
    ap.add_argument("--mix-steps", type=int, default=62)
    ap.add_argument("--mix-envelope-members", type=int, default=4,
                    help="ensemble scenarios also run alone in FP32, FP64 and perturbed FP64")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-c1", action="store_true", help="skip the small CPU configuration run in full")
    ap.add_argument("--no-c1-ref", action="store_true",
                    help="in the c1 section, skip the reference program's full run")
    ap.add_argument("--c1-in-flight", type=int, default=0,
                    help="steps in flight of the c1 section's device-timed run (0: the library's default, "
                         "as the program uses)")
    ap.add_argument("--serve-seconds", type=float, default=60.0,
                    help="arrival window of the serving sample (the configuration's: 600 s)")
    ap.add_argument("--serve-horizon-scale", type=float, default=1.0 / 120.0)
    ap.add_argument("--serve-accuracy-requests", type=int, default=3,
                    help="served requests also run alone in FP64 and perturbed FP64 for their error")
    ap.add_argument("--serve-generate-ahead", type=float, default=3.0,
                    help="seconds before arrival at which a request's inputs are generated")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()

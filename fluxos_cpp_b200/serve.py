"""Continuous batching of scenario solves on one GPU.

The reference runs one domain per process to the end of its forcing
(main.cpp:271-470). Here a request is such a run: a scenario (terrain,
forcing, horizon, solutes) to be advanced from its start state to its
horizon. The loop keeps every admitted scenario's state resident on the GPU
as a member of one fx_batch, so all of them advance through the same
launches, each with its own clock and dt:

* admission: requests are taken in arrival order as soon as they have
  arrived and their device footprint (fx_footprint) fits under the cap
  beside the members already resident;
* stepping: the batch advances a chunk of steps at a time; members whose
  output falls due stop inside the chunk and are acknowledged (optionally
  written out) before the next one;
* retirement: a member whose clock passed its horizon leaves the batch
  between chunks, its result is taken and its memory freed, which makes room
  for the next arrivals.

A request's inputs (terrain, forcing, start state) come with it, as a real
request's would: a look-ahead generator builds them on host threads before
the request's arrival time, off the latency clock. Its preparation (context
creation and upload on the context's own stream) runs on a host thread once
it has arrived and fits, while the batch keeps stepping. Latency of a
request is the time from its arrival to its retirement, reported with its
parts: admission wait (arrival to the start of its preparation),
preparation, join wait and device residency (joining the batch to
retirement).

With several GPUs, each rank serves its own share of the request stream
(`shard`: request id modulo the number of ranks), with its own batch and no
collective on the data path; `summarize` merges the ranks' records.
"""
from __future__ import annotations

import collections
import concurrent.futures as cf
import math
import time
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional

import numpy as np

import fluxos_cpp_b200 as fx
from fluxos_cpp_b200 import scenarios as S


@dataclass(eq=False)
class Request:
    """One scenario solve. `make` builds the Scenario (called on a host
    thread); `cells`, `nchem` and `extension_grids` size the admission."""

    rid: int
    arrival: float
    make: Callable[[], S.Scenario]
    nrows: int
    ncols: int
    nchem: int = 1
    extension_grids: int = 2
    precision: str = "fp32"
    steps_in_flight: int = 31  # the batch launch sweeps this many steps per ADE launch
    # filled in by the server
    inputs: Optional[S.Scenario] = None  # generated ahead of arrival
    prep_start: Optional[float] = None
    prepared: Optional[float] = None
    admitted: Optional[float] = None
    done: Optional[float] = None
    steps: int = 0
    status: Optional[dict] = None
    water: Optional[float] = None
    state: Dict[str, np.ndarray] = field(default_factory=dict)

    @property
    def cells(self) -> int:
        return self.nrows * self.ncols

    @property
    def latency(self) -> Optional[float]:
        return None if self.done is None else self.done - self.arrival


class Server:
    """The request loop. `keep` names fields to download at retirement
    (e.g. ("h", "conc")); `on_output(req, domain)` runs for every due output
    before it is acknowledged. `batch_factory` and `make_domain` build the
    batch and a request's domain (fx.Batch and scenarios.make_domain; tests
    of the host logic pass stand-ins)."""

    def __init__(self, cap_bytes: float = 150e9, chunk_steps: int = 31, keep=(),
                 on_output: Optional[Callable] = None, host_threads: int = 4,
                 clock: Callable[[], float] = time.perf_counter,
                 batch_factory: Optional[Callable] = None, make_domain: Optional[Callable] = None):
        self.cap = float(cap_bytes)
        self.chunk = int(chunk_steps)
        self.keep = tuple(keep)
        self.on_output = on_output
        self.clock = clock
        self.pool = cf.ThreadPoolExecutor(max_workers=host_threads)
        self.lookahead = host_threads
        # retired domains are released on their own thread (freeing device
        # memory waits for the device), so the loop goes on stepping; their
        # bytes count against the cap until the release has finished
        self.closer = cf.ThreadPoolExecutor(max_workers=1)
        self.closing: List[tuple] = []  # (future, bytes)
        self.batch = (batch_factory or fx.Batch)()
        self.make_domain = make_domain or S.make_domain
        self.active: List[tuple] = []  # (request, domain, bytes)
        self.used = 0
        self.peak_used = 0
        self.peak_members = 0
        self.cell_updates = 0
        self.gpu_busy = 0.0
        # host time of the request loop outside the batch steps, by part
        self.host_s = {"admit": 0.0, "retire": 0.0, "status": 0.0, "idle": 0.0}

    def close(self) -> None:
        for _, d, _ in self.active:
            d.close()
        self.active = []
        self._released(wait=True)
        self.batch.close()
        self.pool.shutdown(wait=False)
        self.closer.shutdown(wait=True)

    def _released(self, wait: bool = False) -> None:
        """Drop finished releases of retired domains from the memory count."""
        keep = []
        for f, nbytes in self.closing:
            if wait or f.done():
                f.result()
                self.used -= nbytes
            else:
                keep.append((f, nbytes))
        self.closing = keep

    @staticmethod
    def footprint(r: Request) -> int:
        return fx.footprint(r.nrows, r.ncols, nchem=r.nchem, precision=r.precision,
                            steps_in_flight=r.steps_in_flight, extension_grids=r.extension_grids)

    def _retire(self, i: int, now: float) -> None:
        r, d, nbytes = self.active.pop(i)
        self.batch.remove(d)
        r.status = d.status()
        r.steps = int(r.status["steps"])
        r.water = d.mass()[0]
        for k in self.keep:
            r.state[k] = d.download(k)
        self.closing.append((self.closer.submit(d.close), nbytes))
        r.done = now

    def _prepare(self, r: Request, t0: float, gen: Optional[cf.Future] = None):
        """Host thread: the request's resident domain from its inputs (made
        here only if the look-ahead generator has not made them; `gen` is the
        generator's unfinished job for them, if any)."""
        r.prep_start = self.clock() - t0
        if gen is not None:
            gen.result()
        sc = r.inputs if r.inputs is not None else r.make()
        r.inputs = None
        d = self.make_domain(sc, precision=r.precision, steps_in_flight=r.steps_in_flight)
        r.prepared = self.clock() - t0
        return d

    def run(self, requests: List[Request], generate_ahead: float = 0.0,
            generator_threads: int = 4) -> dict:
        """Serve `requests` (arrival times in seconds from the call) to the
        end; returns throughput and latency figures (summarize).

        With generate_ahead > 0, a request's inputs are generated on
        `generator_threads` host threads from that many seconds before its
        arrival (off the latency clock; the count of requests whose inputs
        were not ready at arrival is reported). A request's preparation
        (device allocation and upload on the request's own stream) starts
        when it has arrived and its footprint fits under the cap beside the
        resident members and the preparations in progress; it runs on a host
        thread while the batch keeps stepping. Prepared requests join the
        batch between chunks."""
        order = sorted(requests, key=lambda r: r.arrival)
        pending = collections.deque(order)
        to_generate = collections.deque(order if generate_ahead > 0 else [])
        gen_pool = cf.ThreadPoolExecutor(max_workers=generator_threads) if generate_ahead > 0 else None
        generating: Dict[int, cf.Future] = {}
        late_inputs = 0
        preparing = collections.OrderedDict()  # rid -> (request, future, reserved bytes)
        seen: Dict[int, int] = {}  # rid -> the member's step count after its last chunk
        reserved = 0
        t0 = self.clock()

        def _gen(r):
            r.inputs = r.make()

        while pending or preparing or self.active:
            self._released()
            now = self.clock() - t0
            # the look-ahead generator: inputs of requests arriving within generate_ahead
            while to_generate and to_generate[0].arrival <= now + generate_ahead and \
                    len(generating) < 2 * generator_threads:
                r = to_generate.popleft()
                generating[r.rid] = gen_pool.submit(_gen, r)
            for rid in [k for k, f in generating.items() if f.done()]:
                generating.pop(rid).result()
            # start preparations in arrival order while memory and threads allow
            while pending and pending[0].arrival <= now and len(preparing) < self.lookahead:
                r = pending[0]
                need = self.footprint(r)
                if (self.active or preparing) and self.used + reserved + need > self.cap:
                    break
                gen = None
                if gen_pool is not None:
                    gen = generating.pop(r.rid, None)
                    if gen is not None and not gen.done():
                        late_inputs += 1  # its preparation waits for the generator
                    elif gen is None and r.inputs is None:
                        late_inputs += 1  # not started: its preparation makes the inputs
                        if r in to_generate:
                            to_generate.remove(r)
                preparing[r.rid] = (r, self.pool.submit(self._prepare, r, t0, gen), need)
                reserved += need
                pending.popleft()
            # admit finished preparations
            ta = self.clock()
            for rid in [k for k, (_, f, _) in preparing.items() if f.done()]:
                r, f, need = preparing.pop(rid)
                reserved -= need
                d = f.result()
                self.batch.add(d)
                nbytes = d.device_bytes()
                self.active.append((r, d, nbytes))
                seen[r.rid] = d.status()["steps"]
                self.used += nbytes
                self.peak_used = max(self.peak_used, self.used + reserved)
                self.peak_members = max(self.peak_members, len(self.active))
                r.admitted = self.clock() - t0
            self.host_s["admit"] += self.clock() - ta
            if not self.active:
                ti = self.clock()
                time.sleep(0.001)
                self.host_s["idle"] += self.clock() - ti
                continue
            # step counts before the chunk: from the last chunk's statuses
            # (or the admission's), with no device round trip per member
            ts = self.clock()
            before = [seen[r.rid] for r, _, _ in self.active]
            g0 = self.clock()
            self.host_s["status"] += g0 - ts
            sts = self.batch.step(self.chunk)
            self.gpu_busy += self.clock() - g0
            now = self.clock() - t0
            for (r, d, _), st, s0 in zip(self.active, sts, before):
                self.cell_updates += (st["steps"] - s0) * r.cells
                seen[r.rid] = st["steps"]
            for i in range(len(self.active) - 1, -1, -1):
                r, d, _ = self.active[i]
                st = sts[i]
                if st["device_error"]:
                    raise fx.FluxosError(-5, f"request {r.rid}: device error")
                if st["print_pending"]:
                    if self.on_output:
                        self.on_output(r, d)
                    d.print_done()
                if st["finished"]:
                    tr = self.clock()
                    self._retire(i, now)
                    self.host_s["retire"] += self.clock() - tr
        wall = self.clock() - t0
        self._released(wait=True)
        if gen_pool is not None:
            gen_pool.shutdown(wait=True)
        part = {"records": [record(r) for r in requests], "wall_s": wall, "cell_updates": self.cell_updates,
                "inputs_late": late_inputs if gen_pool is not None else None,
                "peak_device_bytes": self.peak_used, "peak_members": self.peak_members,
                "batch_step_s": self.gpu_busy, "host_s": dict(self.host_s)}
        self.last_part = part  # this server's records, for merging with other ranks' (summarize)
        return summarize([part])


def record(r: Request) -> dict:
    """The times and work of one served request (seconds from the start of
    its server's run)."""
    return {"rid": r.rid, "arrival": r.arrival, "prep_start": r.prep_start, "prepared": r.prepared,
            "admitted": r.admitted, "done": r.done, "cells": r.cells, "steps": r.steps}


def summarize(parts: List[dict]) -> dict:
    """Throughput and latency of one or more servers' runs (one part per
    rank, each serving its share of one request stream): latency
    percentiles over every request, with its parts; throughput = all cell
    updates / the slowest server's wall time; offered load = the cell
    updates the requests asked for / the arrival window."""
    recs = [x for p in parts for x in p["records"]]
    done = [x for x in recs if x["done"] is not None]

    def pct(vals):
        a = np.array(vals, dtype=np.float64)
        return ({"p50_s": float(np.percentile(a, 50)), "p99_s": float(np.percentile(a, 99))}
                if a.size else {"p50_s": None, "p99_s": None})

    wall = max(p["wall_s"] for p in parts)
    updates = sum(p["cell_updates"] for p in parts)
    window = max((x["arrival"] for x in recs), default=0.0)
    offered = sum(x["steps"] * x["cells"] for x in done)
    lat = pct([x["done"] - x["arrival"] for x in done])
    late = [p["inputs_late"] for p in parts if p.get("inputs_late") is not None]
    return {"requests": len(recs), "completed": len(done), "servers": len(parts), "wall_s": wall,
            "cell_updates": updates, "cell_updates_per_s": updates / wall if wall > 0 else 0.0,
            "arrival_window_s": window,
            "offered_cell_updates_per_s": offered / window if window > 0 else None,
            "p50_s": lat["p50_s"], "p99_s": lat["p99_s"],
            "latency_parts": {
                "admission_wait": pct([x["prep_start"] - x["arrival"] for x in done]),
                "preparation": pct([x["prepared"] - x["prep_start"] for x in done]),
                "join_wait": pct([x["admitted"] - x["prepared"] for x in done]),
                "device_residency": pct([x["done"] - x["admitted"] for x in done])},
            "inputs_late": sum(late) if late else None,
            "peak_device_bytes": max(p["peak_device_bytes"] for p in parts),
            "peak_members": max(p["peak_members"] for p in parts),
            "batch_step_s": max(p["batch_step_s"] for p in parts),
            "host_s": {k: max(p.get("host_s", {}).get(k, 0.0) for p in parts)
                       for k in ("admit", "retire", "status", "idle")}}


def shard(requests: List[Request], rank: int, world: int) -> List[Request]:
    """This rank's share of a request stream: request id modulo the number
    of ranks. Every request belongs to exactly one rank, and the shares'
    sizes differ by at most one."""
    return [r for r in requests if r.rid % world == rank]


def poisson_requests(rate: float, duration: float, seed: int, *, n_min: int = 128, n_max: int = 4096,
                     horizon_h=(1.0, 12.0), horizon_scale: float = 1.0, nchem=(1, 3),
                     precision: str = "fp32", dxy: int = 2, wet: bool = True) -> List[Request]:
    """Seeded request stream of the serving configuration: Poisson arrivals,
    square grids log-uniform in [n_min, n_max], horizon uniform in hours
    (times `horizon_scale`), 1-3 solutes, terrain and melt field as the
    large-domain configuration (fractal DEM, melt 5-40 mm/day field, Manning
    n U[0.03, 0.15]) and a wet start."""
    rng = np.random.default_rng(seed)
    out, t, rid = [], 0.0, 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        hor = float(rng.uniform(*horizon_h)) * 3600.0 * horizon_scale
        k = int(rng.integers(nchem[0], nchem[1] + 1))
        s = int(rng.integers(0, 2**31 - 1))

        def make(n=n, hor=hor, k=k, s=s):
            sc = S.fractal_scenario(n, dxy=dxy, seed=s, melt_seed=s + 1, extensions=True, horizon=hor)
            sc.print_step = max(1, int(hor))
            if k > 1:
                sc.d_coefs = [0.01 * (10 ** j) for j in range(k)]
            if wet:
                S.wet_start(sc, depth=0.005, seed=s + 2)
            return sc

        out.append(Request(rid=rid, arrival=t, make=make, nrows=n, ncols=n, nchem=k,
                           precision=precision))
        rid += 1
    return out

"""Scenario-sharded serving on the CPU: two gloo ranks (127.0.0.1) each run
the real request loop (fluxos_cpp_b200.serve.Server) over their share of one
seeded request stream, with stand-ins for the GPU batch and domains, then
merge their records as bench.py does. Every request must be served exactly
once, by the rank serve.shard gives it, to its horizon, with the look-ahead
input generator and the footprint admission in the loop."""
import socket

import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class FakeDomain:
    """Steps to a horizon of `need` steps; an output falls due halfway."""

    def __init__(self, rid: int, need: int, nbytes: int):
        self.rid, self.need, self.nbytes = rid, need, nbytes
        self.steps, self.pending, self.printed = 0, False, False

    def advance(self, n: int) -> dict:
        if not self.pending:
            half = self.need // 2
            stop = half if (not self.printed and self.steps < half) else self.need
            self.steps = min(self.steps + n, stop)
            self.pending = self.steps == half and not self.printed
        return self.status()

    def status(self) -> dict:
        return {"steps": self.steps, "print_pending": self.pending, "finished": self.steps >= self.need,
                "device_error": 0, "tim": float(self.steps)}

    def print_done(self) -> None:
        self.pending, self.printed = False, True

    def device_bytes(self) -> int:
        return self.nbytes

    def mass(self):
        return 0.0, []

    def download(self, k):
        return None

    def close(self) -> None:
        pass


class FakeBatch:
    def __init__(self):
        self.members = []

    def add(self, d):
        self.members.append(d)

    def remove(self, d):
        self.members.remove(d)

    def step(self, n):
        return [d.advance(n) for d in self.members]

    def close(self):
        self.members = []


def _worker(rank: int, world: int, port: int, q) -> None:
    import torch.distributed as dist
    from fluxos_cpp_b200 import serve
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        reqs = serve.poisson_requests(rate=40.0, duration=0.5, seed=4, n_min=16, n_max=64)
        made = []
        for r in reqs:  # inputs: a stand-in scenario naming its request
            r.make = (lambda r=r: made.append(r.rid) or r.rid)
        mine = serve.shard(reqs, rank, world)

        def make_domain(rid, precision, steps_in_flight):
            r = next(x for x in mine if x.rid == rid)
            return FakeDomain(rid, need=10 + (rid % 7) * 5, nbytes=serve.Server.footprint(r))

        srv = serve.Server(cap_bytes=3 * max(serve.Server.footprint(r) for r in reqs), chunk_steps=4,
                           batch_factory=FakeBatch, make_domain=make_domain)
        srv.run(mine, generate_ahead=0.2, generator_threads=2)
        part = srv.last_part
        part["rank"] = rank
        part["made"] = sorted(made)
        srv.close()
        parts = [None] * world
        dist.all_gather_object(parts, part)
        if rank == 0:
            q.put((len(reqs), parts, serve.summarize(parts)))
    finally:
        dist.destroy_process_group()


def test_two_ranks_serve_disjoint_shares_of_the_stream():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    n, parts, stats = q.get(timeout=10)
    assert n >= 10
    served = {}
    for p in parts:
        for x in p["records"]:
            assert x["rid"] not in served, "a request served twice"
            served[x["rid"]] = p["rank"]
            assert x["done"] is not None and x["steps"] == 10 + (x["rid"] % 7) * 5
            assert x["arrival"] <= x["prep_start"] <= x["prepared"] <= x["admitted"] <= x["done"]
        # each rank generated the inputs of its own share only, once each
        assert p["made"] == sorted(x["rid"] for x in p["records"])
    assert sorted(served) == list(range(n))
    assert all(rank == rid % 2 for rid, rank in served.items())
    assert stats["requests"] == stats["completed"] == n and stats["servers"] == 2
    assert stats["wall_s"] == max(p["wall_s"] for p in parts)
    assert stats["cell_updates"] == sum(p["cell_updates"] for p in parts)
    assert stats["p99_s"] >= stats["p50_s"] > 0


def test_shares_partition_the_stream():
    from fluxos_cpp_b200 import serve
    reqs = serve.poisson_requests(rate=4.0, duration=60.0, seed=4)
    for world in (1, 2, 3, 8):
        shares = [serve.shard(reqs, k, world) for k in range(world)]
        rids = sorted(r.rid for s in shares for r in s)
        assert rids == [r.rid for r in reqs]
        sizes = [len(s) for s in shares]
        assert max(sizes) - min(sizes) <= 1

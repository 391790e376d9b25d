"""The multi-rank path of bench.py on CPU: two ranks in a gloo process
group (127.0.0.1) run replicas with no data-path collective; the job's time
is the slowest rank's and its rate is the sum over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, q) -> None:
    import torch.distributed as dist
    import bench
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        ms = [12.5, 30.25][rank]  # this rank's replica time
        ms_max = bench.max_over_ranks(ms, device="cpu")
        rate = bench.job_rate(1000 * 63, world, ms_max / 1e3)
        dist.barrier()
        q.put((rank, ms_max, rate, bench._rank()))
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time_and_sum_the_work():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms_max, rate, rk in got:
        assert ms_max == 30.25
        assert rate == pytest.approx(2 * 1000 * 63 / 0.03025)
        assert rk == (rank, 2, rank)


def test_reference_arm_other_ranks_exit_without_work(capsys, monkeypatch):
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    bench.run_reference(None)  # rank 1 returns before reading its arguments
    assert capsys.readouterr().out == ""


def test_single_process_max_is_identity():
    import bench
    assert bench.max_over_ranks(7.5, device="cpu") == 7.5

"""The N>1 host logic of bench.py on CPU: world-size-2 gloo ranks each run
their own shard (phantom seed), time it, and the job throughput is all ranks'
units over the slowest rank's time (max-reduction), as bench.py does on GPUs."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = torch.tensor([100.0 + 50.0 * rank], dtype=torch.float64)  # rank 1 is the slow one
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
        seeds = [None] * world
        dist.all_gather_object(seeds, bench.shard_seed(2024, rank))
        out[rank] = (float(ms.item()), seeds)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_max_time_and_distinct_shards():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank_main, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    assert out[0][0] == out[1][0] == 150.0
    seeds = out[0][1]
    assert len(set(seeds)) == world
    # whole-job throughput uses the max over ranks
    v = bench.aggregate([100.0, 150.0], units_per_rank=1000, steps=3)
    assert v == pytest.approx(2 * 1000 * 3 / 0.150)


def test_updates_of_workloads():
    assert bench.updates(bench.WORKLOADS["cone512"]) == 48318382080
    assert bench.updates(bench.WORKLOADS["cone256"]) == 6039797760


def test_clock_summary_uses_samples_under_load():
    """The reported SM clock is the median over samples taken under load; a
    throttle reason seen in any sample is reported."""
    c = bench.ClockSampler(0)
    idle = ["0", "345", "1965", "90", "0x0", "Not Active", "Not Active", "Not Active", "Not Active", "0"]
    busy = ["0", "1965", "1965", "700", "0x0", "Not Active", "Not Active", "Not Active", "Active", "100"]
    c.rows = [idle, busy, busy, idle, idle]
    s = c.summary()
    assert s["sm_mhz"] == 1965.0 and s["samples_under_load"] == 2
    assert s["reasons"] == ["sw_power_cap"]

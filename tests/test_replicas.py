"""Replica mode on CPU: two gloo ranks, each with its own scene seed, meet
only in the barrier and the max-over-ranks timing reduction."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, results):
    import datetime
    import torch.distributed as dist
    from vapor_b200.replicas import aggregate_steps_per_second, max_over_ranks, scene_seed
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        local_ms = 100.0 + 50.0 * rank  # rank 1 is the slow one
        ms = max_over_ranks(local_ms, dist)
        results[rank] = (scene_seed(2024, rank), ms, aggregate_steps_per_second(world, 3, ms))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_replicas_take_the_slowest_rank():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        results = m.dict()
        mp.spawn(_rank, args=(world, port, results), nprocs=world, join=True)
        res = dict(results)
    assert res[0][0] != res[1][0]  # independent scenes
    assert res[0][1] == res[1][1] == pytest.approx(150.0)  # both see the max
    assert res[0][2] == pytest.approx(2 * 3 / 0.15)


def test_single_process_needs_no_group():
    from vapor_b200.replicas import max_over_ranks, rank_info
    assert max_over_ranks(12.5) == 12.5
    assert rank_info()[0] >= 1

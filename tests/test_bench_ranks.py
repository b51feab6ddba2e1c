"""The multi-GPU bench path on the CPU: two gloo ranks agree on the slowest
rank's time, the whole-job value counts every rank's points, and each rank
draws its own points (weak scaling, no collective on the data path)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local = [4.0, 7.5][rank]
        ms = bench.max_over_ranks(local, world)
        out[rank] = (ms, bench.whole_job_mpts(1 << 20, world, ms))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    for r in (0, 1):
        ms, v = res[r]
        assert ms == 7.5
        assert v == pytest.approx(2 * (1 << 20) / 7.5e-3 / 1e6)


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(3.0, 1) == 3.0
    assert bench.whole_job_mpts(1000, 1, 1.0) == pytest.approx(1.0)


def test_ranks_draw_distinct_points():
    import bench
    a = bench.rank_states(53, 256, 0)
    b = bench.rank_states(53, 256, 1)
    assert a[2].shape == (53, 256) and b[2].shape == (53, 256)
    assert not np.array_equal(a[1], b[1])
    assert np.array_equal(a[1], bench.rank_states(53, 256, 0)[1])

"""The multi-GPU bench path on the CPU: two gloo ranks agree on the slowest
rank's time, the whole-job value counts every rank's points, each rank
draws its own points and computes them without a collective (weak scaling),
and every rank times the headline mode rank 0 chose."""
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


def _data_path_rank(rank, world, port, out):
    """One rank of the sharded data path: its own states, rates computed on
    its slice alone (the oracle stands in for the rank's GPU), then the only
    collectives the bench makes -- the mode broadcast and the max of the
    timings."""
    import datetime
    import torch.distributed as dist
    import bench
    from chemgen_b200 import pack, synthetic
    from oracle import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mech = synthetic.h2o2_10sp()
        blob = pack.pack(mech).to_blob()
        P, T, Y = bench.rank_states(mech.ns, 512, rank)
        w = oracle.getrates(blob, P, T, Y, nthreads=1)
        modes = ["fp64", "mixed", "mixed_tc"]
        # each rank sees different timings; only rank 0 checks errors
        results = {m: {"value": v} for m, v in zip(modes, [[500.0, 800.0, 100.0], [500.0, 100.0, 900.0]][rank])}
        err = {"fp64": {"norm_max": 1e-14}, "mixed": {"norm_max": 3e-7}, "mixed_tc": {"norm_max": 4e-7}} \
            if rank == 0 else {}
        head = bench.choose_head(modes, results, err, "auto", world)
        ms = bench.max_over_ranks([2.0, 3.0][rank], world)
        out[rank] = (head, ms, float(T.sum()), w.copy())
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_points_and_agree_on_the_headline_mode():
    from chemgen_b200 import pack, synthetic
    from oracle import oracle
    import bench
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_data_path_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    # rank 0's choice (the fastest mode within 1e-6 on rank 0's timings) on both ranks
    assert res[0][0] == res[1][0] == "mixed"
    assert res[0][1] == res[1][1] == 3.0
    # the ranks' slices differ, and each rank's result is what one process
    # computes for that slice alone: no exchange on the data path
    assert res[0][2] != res[1][2]
    mech = synthetic.h2o2_10sp()
    blob = pack.pack(mech).to_blob()
    for r in (0, 1):
        P, T, Y = bench.rank_states(mech.ns, 512, r)
        np.testing.assert_array_equal(res[r][3], oracle.getrates(blob, P, T, Y, nthreads=1))


def test_headline_mode_single_rank():
    import bench
    modes = ["fp64", "mixed"]
    results = {"fp64": {"value": 500.0}, "mixed": {"value": 800.0}}
    assert bench.choose_head(modes, results, {"fp64": {"norm_max": 1e-14}, "mixed": {"norm_max": 2e-6}},
                             "auto", 1) == "fp64"
    assert bench.choose_head(modes, results, {"fp64": {"norm_max": 1e-14}, "mixed": {"norm_max": 2e-7}},
                             "auto", 1) == "mixed"
    assert bench.choose_head(modes, results, {}, "fp64", 1) == "fp64"

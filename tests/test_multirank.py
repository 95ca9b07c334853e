"""The multi-rank bench path on CPU: two gloo ranks, as torchrun would start
them (one process per GPU on a B200 node, replicas sharded by rank)."""

import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    import bench
    from jaxrens_b200 import nested_sampling as nsm

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # the slowest rank's time is the job's time
        t = bench.max_over_ranks(1.5 + rank, world, torch.device("cpu"))
        # each rank builds its own runs; they must not coincide across ranks
        case = bench.build_case(bench.rank_seed(0, rank))
        keys = torch.tensor(np.stack(case[6]).astype(np.int64))
        gathered = [torch.zeros_like(keys) for _ in range(world)]
        dist.all_gather(gathered, keys)
        pos0 = torch.tensor(case[3][0][0])
        allpos = [torch.zeros_like(pos0) for _ in range(world)]
        dist.all_gather(allpos, pos0)
        out[rank] = (t, [g.numpy() for g in gathered], [p.numpy() for p in allpos])
        dist.barrier()
    finally:
        dist.destroy_process_group()
    del nsm


def test_two_gloo_ranks_shard_runs_and_take_the_max_time():
    import torch.multiprocessing as mp

    world = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    t0, keys0, pos0 = out[0]
    t1, keys1, _ = out[1]
    assert t0 == t1 == 2.5
    assert not np.array_equal(keys0[0], keys0[1])        # distinct runs per rank
    assert not np.array_equal(pos0[0], pos0[1])
    np.testing.assert_array_equal(keys0[0], keys1[0])   # both ranks agree on the gather


def test_whole_job_throughput_counts_every_rank():
    import bench

    v1, i1 = bench.job_throughput(1, 100, 50.0)
    v2, i2 = bench.job_throughput(2, 100, 50.0)
    assert v2 == 2 * v1 and i2 == 2 * i1
    assert v1 == bench.P_RUNS * bench.T * 100 / 0.05

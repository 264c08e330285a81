"""The N > 1 path of bench.py on CPU: two gloo ranks (127.0.0.1). Each rank solves its own
densities (disjoint seeds, no data-path collective), the step time is the maximum over
ranks, and the whole-job value counts every rank's instances."""

import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime

    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    r, w, _ = bench.dist_env()
    seed = bench.rank_first_seed(r)
    t = bench.max_over_ranks(10.0 * (r + 1), w, device="cpu")  # rank 1 is the slower one
    dens = bench.densities(16, 2, seed)
    out[r] = (w, seed, t, bench.job_value(2, w, t / 3), float(dens[0].sum()))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_gloo_ranks_shard_and_time_as_the_bench_does():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(150)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        res = dict(out)
    assert res[0][0] == res[1][0] == 2
    assert res[0][1] != res[1][1]  # disjoint densities per rank
    assert res[0][4] != res[1][4]
    assert res[0][2] == res[1][2] == 20.0  # max over ranks on every rank
    assert res[0][3] == res[1][3] == 2 * 2 / (20.0 / 3 / 1e3)


def test_one_rank_is_the_identity():
    import sys

    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.job_value(8, 1, 40.0) == 200.0

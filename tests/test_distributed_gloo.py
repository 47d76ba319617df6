"""Multi-rank plumbing on CPU: two gloo ranks shard independent solves,
bracket a 'timed region' with barriers and reduce its results the way
bench.py does on NCCL ranks (sum of units, max of time)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from teuk_b200 import distributed as td


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, solves, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world),
                       "LOCAL_RANK": str(rank), "MASTER_ADDR": "127.0.0.1",
                       "MASTER_PORT": str(port)})
    info = td.init("gloo", timeout_seconds=60)
    assert (info.rank, info.world_size) == (rank, world)
    mine = td.shard(solves, rank, world)
    td.barrier()
    # rank r 'took' (r + 1) seconds for its solves of 10 units each
    rate, slowest = td.whole_job_rate(10.0 * len(mine), float(rank + 1))
    td.barrier()
    out.put((rank, list(mine), rate, slowest))
    td.finalize()


@pytest.mark.parametrize("world,solves", [(2, 7), (2, 64)])
def test_two_gloo_ranks_shard_and_reduce(world, solves):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, solves, out))
             for r in range(world)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    owned = [i for _, mine, _, _ in results for i in mine]
    assert owned == list(range(solves))          # disjoint, complete
    for _, _, rate, slowest in results:
        assert slowest == float(world)            # max over ranks
        assert rate == 10.0 * solves / world      # whole-job units / slowest


def test_single_process_needs_no_group():
    info = td.rank_info()
    assert td.shard(5, 0, 1) == range(0, 5)
    assert td.whole_job_rate(12.0, 3.0) == (4.0, 3.0)
    with pytest.raises(ValueError):
        td.shard(5, 2, 2)
    assert info.world_size >= 1

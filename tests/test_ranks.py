"""The multi-GPU rank plumbing (string_vext_b200/ranks.py) with world size 2
on CPU (gloo, 127.0.0.1): disjoint covering shards and the max-over-ranks
step time the benchmark reports, as two real processes."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, queue):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port),
                       "RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    import torch.distributed as dist

    from string_vext_b200 import ranks
    r, w, lr = ranks.rank_info()
    ranks.init("gloo", lr, timeout_s=60)
    mine = ranks.shard(range(11), r, w)
    ms = ranks.max_over_ranks(10.0 + 5.0 * r)     # rank 1 is the slow one
    gathered = [None] * w
    dist.all_gather_object(gathered, mine)
    ranks.barrier()
    dist.destroy_process_group()
    queue.put((r, w, mine, ms, gathered))


def test_two_gloo_ranks_shard_and_max_time():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, queue)) for r in range(world)]
    for p in procs:
        p.start()
    results = [queue.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, w, mine, ms, gathered in results:
        assert w == world
        assert ms == pytest.approx(15.0)                    # the slowest rank's time
        flat = sorted(x for part in gathered for x in part)
        assert flat == list(range(11))                       # disjoint and covering
        assert mine == list(range(11))[r::world]


def test_single_process_defaults():
    from string_vext_b200 import ranks
    assert ranks.max_over_ranks(3.5) == 3.5
    assert ranks.shard([1, 2, 3], 0, 1) == [1, 2, 3]

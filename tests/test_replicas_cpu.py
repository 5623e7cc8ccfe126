"""The multi-GPU path (replicas) on CPU: two gloo ranks shard a pair list without
overlap, draw disjoint synthetic seeds, and agree on the max-over-ranks duration that
whole-job throughput is computed from."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from doubleeye_b200 import replicas
    mine = replicas.shard(list(range(11)), rank, world)
    slowest = replicas.max_over_ranks(1.5 + rank)        # rank 1 is the slow one
    q.put((rank, mine, replicas.rank_seed(rank), slowest))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replicas():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, a, sa, ma), (_, b, sb, mb) = got
    assert sorted(a + b) == list(range(11)) and not set(a) & set(b)
    assert abs(len(a) - len(b)) <= 1
    assert sa != sb
    assert ma == mb == 2.5


def test_shard_rejects_bad_rank():
    from doubleeye_b200 import replicas
    with pytest.raises(ValueError):
        replicas.shard([1, 2], 2, 2)

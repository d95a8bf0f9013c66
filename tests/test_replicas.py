"""The multi-GPU path is replicas: the host-side steps (rank 0's configuration on every rank, timings as the max over
ranks, whole-block arena ranges) checked with two gloo ranks on the CPU."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import replicas

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cfg = replicas.broadcast_config({"mode": "binned", "block": 448 + rank, "rank": rank}, dist)
        t = replicas.max_over_ranks(10.0 + rank * 2.5, dist)
        out.put((rank, cfg, t))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_config_and_max():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, cfg, t in res:
        assert cfg == {"mode": "binned", "block": 448, "rank": 0}
        assert t == 12.5


@pytest.mark.parametrize("total,world", [(65536, 2), (1000, 3), (31, 2), (262144, 8), (100, 7)])
def test_shards_cover_whole_blocks(total, world):
    import replicas

    spans = [replicas.shard(total, r, world) for r in range(world)]
    pos = 0
    for first, count in spans:
        assert first == pos or count == 0
        assert first % 32 == 0
        pos = first + count if count else pos
    assert pos == total
    assert sum(c for _, c in spans) == total

"""The multi-GPU path of bench.py (replicas, no collective on the data path) on CPU: 2 and 4 gloo ranks take disjoint
round-robin shares of the waves that cover them all, and the timing reduction gives the slowest rank's time and
the summed work."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, ws, port, q):
    import torch.distributed as dist
    from pcbroute_b200 import replicas
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        waves = list(range(8))
        mine = replicas.my_waves(waves, ws, rank)
        ms, work = replicas.max_time_sum_work(10.0 * (rank + 1), 100 * len(mine), "cpu", ws)
        q.put((rank, mine, ms, work))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("ws", [2, 4])
def test_gloo_ranks_share_waves_and_reduce_timing(ws):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(ws))
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    shares = [set(r[1]) for r in res]
    for i in range(ws):
        for j in range(i + 1, ws):
            assert shares[i].isdisjoint(shares[j])
    assert set().union(*shares) == set(range(8))
    for r in res:
        assert r[2] == 10.0 * ws          # the slowest rank's time
        assert r[3] == 100 * 8            # all waves' work


def test_more_ranks_than_waves_wrap_around():
    from pcbroute_b200 import replicas
    waves = list(range(3))
    shares = [replicas.my_waves(waves, 8, r) for r in range(8)]
    assert all(len(s) == 1 for s in shares)
    assert {s[0] for s in shares} == set(waves)

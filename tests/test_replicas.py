"""CPU: the multi-rank bookkeeping of bench.py (one replica per GPU, barrier,
max of the ranks' times, shares of independent objects) on the gloo backend
with two processes."""
import os
import socket

import pytest

from hiparti_b200.replicas import shard


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from hiparti_b200 import replicas
    r, w, _ = replicas.setup("gloo", timeout_s=60)
    replicas.barrier(w)
    # each rank reports its own "time"; all must see the maximum
    m = replicas.max_over_ranks(1.5 + r, w)
    items = list(replicas.shard(11, r, w))
    out.put((r, w, m, items))
    replicas.barrier(w)
    replicas.shutdown(w)


def test_two_gloo_ranks_agree_on_the_max_and_split_the_objects():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [2, 2]
    assert [r[2] for r in res] == [2.5, 2.5]
    assert res[0][3] + res[1][3] == list(range(11))


@pytest.mark.parametrize("n,world", [(0, 3), (5, 8), (11, 2), (256, 8), (7, 7)])
def test_shard_covers_every_object_once(n, world):
    got = [i for r in range(world) for i in shard(n, r, world)]
    assert got == list(range(n))
    sizes = [len(shard(n, r, world)) for r in range(world)]
    assert max(sizes) - min(sizes) <= 1

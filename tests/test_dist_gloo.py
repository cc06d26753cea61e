"""The multi-rank plumbing on CPU with two gloo ranks (no GPU)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from crava_b200 import dist as D

    dist = D.init("gloo", timeout_s=60)
    r, w, _ = D.rank_env()
    m = D.max_over_ranks(dist, 10.0 * (r + 1))
    D.barrier(dist)
    items = list(range(11))
    mine = D.shard(items, r, w)
    out.put((r, m, mine))
    dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [20.0, 20.0]
    shares = res[0][2] + res[1][2]
    assert sorted(shares) == list(range(11)) and not set(res[0][2]) & set(res[1][2])


def test_single_process_identity():
    from crava_b200 import dist as D
    assert D.max_over_ranks(None, 3.5) == 3.5
    assert D.shard([1, 2, 3], 0, 1) == [1, 2, 3]

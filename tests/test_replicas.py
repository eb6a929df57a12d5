"""The multi-rank path of the benchmark ("replicas only": no data-path collective) on two gloo
ranks on the CPU: barrier, maximum of per-rank times, contiguous member partition, host gather,
and a rank that fails while the other waits ends with an error instead of hanging."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402

from fip_b200 import replicas  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, n, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(n), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    dist = replicas.init("gloo", timeout_s=30)
    replicas.barrier(dist)
    mx = replicas.max_over_ranks(dist, 10.0 + rank)
    share = list(replicas.partition(64, rank, n))
    got = replicas.gather_to_root(dist, share)
    if rank == 0:
        q.put((mx, got))
    replicas.finish(dist)


def test_two_gloo_ranks():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    mx, got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert mx == 11.0
    assert got[0] + got[1] == list(range(64)) and abs(len(got[0]) - len(got[1])) <= 1


def _dying_worker(rank, n, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(n), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    dist = replicas.init("gloo", timeout_s=5)
    if rank == 1:
        os._exit(3)  # leaves between steps, with nothing in flight
    try:
        replicas.max_over_ranks(dist, 1.0)
        q.put("no error")
    except Exception as exc:  # the survivor learns of it through the collective's timeout / error
        q.put(type(exc).__name__)


def test_lost_rank_ends_with_an_error():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_dying_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    assert res != "no error"


def test_partition_covers_every_member_once():
    for n_items in (0, 1, 7, 64, 65):
        for n in (1, 2, 3, 8):
            parts = [list(replicas.partition(n_items, r, n)) for r in range(n)]
            assert sum(parts, []) == list(range(n_items))
            assert max(map(len, parts)) - min(map(len, parts)) <= 1

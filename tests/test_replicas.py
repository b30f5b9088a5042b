"""Replica bookkeeping on two gloo ranks (CPU): the max-over-ranks timing
and whole-job throughput that bench.py reports for N > 1 GPUs."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist
import torch.multiprocessing as mp

from openhurricane_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms = [10.0 + rank, 100.0 - rank]
        mx = replicas.max_over_ranks(ms)
        cells = replicas.sum_over_ranks([1000.0 * (rank + 1)])
        b, e = replicas.cell_slice(10, world, rank)
        q.put((rank, mx, cells, (b, e)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_max_time():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    for rank, mx, cells, _ in out:
        assert mx == [11.0, 100.0]
        assert cells == [3000.0]
    assert [o[3] for o in out] == [(0, 5), (5, 10)]


def test_cell_slices_cover_exactly():
    for n in (0, 1, 7, 1048576, 1048577):
        for w in (1, 2, 3, 8):
            spans = [replicas.cell_slice(n, w, r) for r in range(w)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [e - b for b, e in spans]
            assert max(sizes) - min(sizes) <= 1


def test_whole_job_rate_and_single_process_identity():
    assert replicas.max_over_ranks([1.0, 2.0]) == [1.0, 2.0]
    assert replicas.whole_job_rate([100, 100], 1000.0) == 200.0

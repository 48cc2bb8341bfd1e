"""Host logic of the multi-GPU (replica) path with world_size 2 gloo ranks on CPU."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402

from conftest import PKG  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys

    sys.path.insert(0, PKG)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    from erq_b200 import replicas

    w, r, _ = replicas.init(backend="gloo", timeout_s=60)
    replicas.barrier(w)
    mx = replicas.max_over_ranks(1.5 + r, w)
    sm = replicas.sum_over_ranks(10.0 * (r + 1), w)
    lo, hi = replicas.shard(10, r, w)
    replicas.finish(w)
    out.put((r, mx, sm, lo, hi))


def test_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [2.5, 2.5]          # slowest rank's time
    assert [r[2] for r in res] == [30.0, 30.0]
    assert [(r[3], r[4]) for r in res] == [(0, 5), (5, 10)]


def test_shard_tiles_the_range():
    import sys

    sys.path.insert(0, PKG)
    from erq_b200 import replicas

    for n in (0, 1, 7, 10, 1000):
        for world in (1, 2, 3, 8):
            spans = [replicas.shard(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))

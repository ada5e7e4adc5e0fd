"""The N>1 path of bench.py on the CPU: two gloo ranks exercise the process-group
setup, the barrier and the max-over-ranks timing reduction that `bench.py --gpus N`
(independent solves per rank, weak scaling) uses with NCCL on GPUs."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench

    w, r, local = bench.dist_setup()
    dist = bench.dist_init(w, local, "gloo")
    bench.dist_barrier(dist)
    slowest = bench.dist_max(dist, 10.0 * (r + 1), "gloo")  # rank-dependent "elapsed ms"
    bench.dist_barrier(dist)
    dist.destroy_process_group()
    q.put((r, w, slowest))


def test_two_gloo_ranks_agree_on_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out == [(0, 2, 20.0), (1, 2, 20.0)]


def test_single_rank_needs_no_process_group(monkeypatch):
    import bench

    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    w, r, local = bench.dist_setup()
    assert (w, r, local) == (1, 0, 0)
    assert bench.dist_init(w, local, "gloo") is None
    assert bench.dist_max(None, 3.5, "gloo") == 3.5

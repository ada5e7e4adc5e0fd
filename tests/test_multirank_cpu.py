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


def _slab_rank_main(rank, world, port, q, stype, steps):
    """One rank of the row-slab decomposition on the CPU: its local grid stepped by the
    oracle (the reference step, clamped at the local top and bottom), at most two steps
    between exchanges, the 4 owned rows beside each cut swapped through gloo by the same
    SlabExchange the GPU path drives with NCCL; rank 0 gathers the owned rows."""
    import datetime

    import numpy as np
    import torch.distributed as dist

    from le2d_b200.dist_slabs import SlabExchange, local_rows
    from oracle.oracle import Oracle

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        nx, ny = 70, 64
        o = Oracle("d")
        c = (0.21, 0.97, 1.03, 2.1, 1.13, 1.37)  # dt, hx, hy, c1, c2, rho
        whole = np.zeros(5 * nx * ny)
        for d in ((20.0, 15.0, 9.0, 1.0), (50.0, 40.0, 12.0, -0.7), (35.0, 62.0, 8.0, 0.5)):
            o.set_ball(whole, nx, ny, c[1], c[2], stype, *d)
        x = SlabExchange(dist, rank, world, nx, ny, lambda shape: torch.zeros(shape, dtype=torch.float64))
        loc = local_rows(whole, nx, ny, stype, x.r0 - x.h0, x.r1 + x.h1)
        view = loc.reshape(x.nyl, nx, 5).transpose(2, 0, 1) if stype == 1 else loc.reshape(5, x.nyl, nx)

        def get_rows(row0, n, buf):
            buf.copy_(torch.from_numpy(np.ascontiguousarray(view[:, row0:row0 + n])))

        def put_rows(row0, n, buf):
            view[:, row0:row0 + n] = buf.numpy()

        left = steps
        while left > 0:
            k = min(2, left)
            o.run(loc, nx, x.nyl, c[0], c[1], c[2], c[3], c[4], c[5], stype, k)
            x.exchange(get_rows, put_rows)
            left -= k
        own = local_rows(loc, nx, x.nyl, stype, x.h0, x.h0 + x.own)
        parts = [None] * world if rank == 0 else None
        dist.gather_object(own, parts, dst=0)
        if rank == 0:
            want = whole.copy()
            o.run(want, nx, ny, c[0], c[1], c[2], c[3], c[4], c[5], stype, steps)
            if stype == 1:
                got = np.concatenate(parts)
            else:
                got = np.concatenate([p.reshape(5, -1, nx) for p in parts], axis=1).reshape(-1)
            q.put(("equal", bool(got.tobytes() == want.tobytes())))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,stype,steps", [(2, 1, 7), (3, 1, 6), (2, 0, 5)])
def test_slab_exchange_gloo_equals_whole_grid(world, stype, steps):
    """The one-process-per-rank row-slab decomposition (le2d_b200.dist_slabs) on CPU ranks:
    the gathered owned rows equal the whole grid stepped alone, bit for bit, for AoS
    (le_step) and SoA (le_step_soa, whose far end only touches halo rows at a cut)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_slab_rank_main, args=(r, world, port, q, stype, steps)) for r in range(world)]
    for p in procs:
        p.start()
    out = q.get(timeout=180)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out == ("equal", True)

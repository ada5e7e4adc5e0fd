"""One grid in row slabs (le2d_slabs_*): every slab steps with the whole-task kernels on its
own rows plus 4 copied rows beside each cut and refreshes those after every launch, so the
result must equal, bit for bit, the same grid stepped by one task.  With one GPU the slabs
share it (the copies between slabs are then device-local); with more, slabs go round-robin
over the visible devices."""
import ctypes

import numpy as np
import pytest

from le2d_b200 import capi
from oracle.oracle import ST_AOS, ST_SOA

pytestmark = pytest.mark.gpu


def _device_count():
    rt = ctypes.CDLL("libcudart.so")
    n = ctypes.c_int(0)
    return n.value if rt.cudaGetDeviceCount(ctypes.byref(n)) == 0 else 0


def _whole(lib, c, g0, steps):
    mat = lib.le_init_material(c["c1"], c["c2"], c["rho"])
    t = lib.le_init_task(c["dt"], (c["hx"], c["hy"]), mat, (c["nx"], c["ny"]), c["stype"])
    try:
        assert lib.upload(t, g0.copy()) == 0
        assert lib.step_n(t, steps) == 0
        out = np.zeros_like(g0)
        assert lib.download(t, out) == 0
        assert lib.last_error(t) == 0
        return out
    finally:
        lib.le_free_task(t)


@pytest.mark.parametrize("stype", [ST_AOS, ST_SOA])
@pytest.mark.parametrize("prec", ["f", "d"])
def test_slabs_equal_whole_grid(prec, stype):
    lib = capi.Lib(prec)
    ndev = max(1, _device_count())
    rng = np.random.default_rng(17)
    for nx, ny, nslabs, steps in ((160, 97, 2, 9), (131, 120, 3, 20), (70, 64, 8, 7)):
        c = dict(nx=nx, ny=ny, hx=1.0, hy=0.9, c1=2.0, c2=1.1, rho=1.3, dt=0.2, stype=stype)
        g0 = rng.uniform(-1, 1, size=5 * nx * ny).astype(lib.dtype)
        want = _whole(lib, c, g0, steps)
        mat = lib.le_init_material(c["c1"], c["c2"], c["rho"])
        t = lib.le_init_task(c["dt"], (c["hx"], c["hy"]), mat, (nx, ny), stype)
        try:
            with capi.Slabs(lib, t, [k % ndev for k in range(nslabs)]) as s:
                rows = [s.rows(k) for k in range(nslabs)]
                assert rows[0][0] == 0 and rows[-1][1] == ny
                assert all(rows[k][1] == rows[k + 1][0] for k in range(nslabs - 1))
                assert s.upload(g0) == 0
                assert s.step_n(steps - 3) == 0
                assert s.step_n(3) == 0  # a second call continues from the first
                got = s.download()
        finally:
            lib.le_free_task(t)
        assert got.tobytes() == want.tobytes(), (prec, stype, nx, ny, nslabs, steps)


def test_slabs_reject_thin_slabs():
    lib = capi.Lib("f")
    mat = lib.le_init_material(2.0, 1.0, 1.0)
    t = lib.le_init_task(0.25, (1.0, 1.0), mat, (64, 30), ST_AOS)
    try:
        with pytest.raises(RuntimeError):
            capi.Slabs(lib, t, [0, 0, 0, 0])  # 30 rows: fewer than 8 per slab
    finally:
        lib.le_free_task(t)


@pytest.mark.parametrize("prec", ["f", "d"])
def test_rank_slabs_exchange_rows_on_device(prec):
    """The one-process-per-rank decomposition (le2d_b200.dist_slabs) with its ranks'
    slabs as tasks on this one GPU: the 4 owned rows beside each cut leave through
    le2d_rows_out into the ranks' CUDA send buffers and come back through le2d_rows_in
    from their receive buffers as the neighbour's halo rows (copied here buffer to buffer
    where NCCL send/recv carries them between processes); the gathered owned rows equal
    the whole grid stepped by one task, bit for bit."""
    torch = pytest.importorskip("torch")
    from le2d_b200.dist_slabs import SlabExchange, local_rows

    lib = capi.Lib(prec)
    c = dict(nx=300, ny=90, hx=1.0, hy=0.9, c1=2.3, c2=1.2, rho=1.6, dt=0.17, stype=ST_AOS)
    rng = np.random.default_rng(3)
    g0 = rng.uniform(-1, 1, 5 * c["nx"] * c["ny"]).astype(lib.dtype)
    steps, world = 9, 3
    want = _whole(lib, c, g0, steps)
    dtype = torch.float32 if prec == "f" else torch.float64
    stream = torch.cuda.current_stream().cuda_stream
    ranks = []
    for r in range(world):
        x = SlabExchange(None, r, world, c["nx"], c["ny"], lambda s: torch.empty(s, dtype=dtype, device="cuda"))
        mat = lib.le_init_material(c["c1"], c["c2"], c["rho"])
        t = lib.le_init_task(c["dt"], (c["hx"], c["hy"]), mat, (c["nx"], x.nyl), ST_AOS)
        assert lib.upload(t, local_rows(g0, c["nx"], c["ny"], ST_AOS, x.r0 - x.h0, x.r1 + x.h1)) == 0
        ranks.append((x, t))
    try:
        left = steps
        while left > 0:
            k = min(2, left)
            for x, t in ranks:
                assert lib.step_n(t, k) == 0
            for (a, ta), (b, tb) in zip(ranks, ranks[1:]):  # each cut, both directions
                assert lib.rows_out(ta, a.h0 + a.own - a.halo, a.halo, a.down[0].data_ptr(), stream) == 0
                assert lib.rows_out(tb, b.h0, b.halo, b.up[0].data_ptr(), stream) == 0
                b.up[1].copy_(a.down[0])
                a.down[1].copy_(b.up[0])
                assert lib.rows_in(tb, 0, b.halo, b.up[1].data_ptr(), stream) == 0
                assert lib.rows_in(ta, a.h0 + a.own, a.halo, a.down[1].data_ptr(), stream) == 0
            left -= k
        parts = []
        for x, t in ranks:
            g = np.zeros(5 * c["nx"] * x.nyl, lib.dtype)
            assert lib.download(t, g) == 0 and lib.last_error(t) == 0
            parts.append(local_rows(g, c["nx"], x.nyl, ST_AOS, x.h0, x.h0 + x.own))
        assert np.concatenate(parts).tobytes() == want.tobytes()
    finally:
        for x, t in ranks:
            lib.le_free_task(t)

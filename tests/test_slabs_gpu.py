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

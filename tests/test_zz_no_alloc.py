"""le2d_diagnostics_noalloc: diagnostics for callers that cannot allocate device memory.

Such callers (a host with a fixed device-memory budget, or a time loop where an
allocation would synchronise the device) hold their state on the device themselves;
this entry point takes that state and allocates nothing, using a static device array
as scratch.  The test places a state on the device with the CUDA runtime (the test
allocates; the entry point does not), calls the entry point twice in a row through the
C ABI and checks both calls against le2d_diagnostics on the same state, with the
tolerance the diagnostics tests use (1e-12 relative on the sums, exact on the maxima).
This file is collected last so that a failure here leaves every other test run.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

from le2d_b200 import capi, workloads
from oracle.oracle import ST_AOS, aos_to_soa

pytestmark = pytest.mark.gpu


def _cudart():
    rt = ctypes.CDLL("libcudart.so")
    rt.cudaMalloc.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_size_t]
    rt.cudaFree.argtypes = [ctypes.c_void_p]
    rt.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    rt.cudaDeviceSynchronize.argtypes = []
    return rt


@pytest.mark.parametrize("prec", ["f", "d"])
def test_noalloc_matches_allocating_diagnostics(prec):
    lib = capi.Lib(prec)
    rt = _cudart()
    p = workloads.Problem(nx=321, ny=207, hx=1.0, hy=0.9, c1=2.2, c2=1.1, rho=1.7, dt=0.18, steps=30,
                          disks=[(100.0, 80.0, 30.0, 1.5), (230.0, 120.0, 20.0, -0.8)])
    mat = lib.le_init_material(p.c1, p.c2, p.rho)
    t = lib.le_init_task(p.dt, (p.hx, p.hy), mat, (p.nx, p.ny), ST_AOS)
    d_ptr = ctypes.c_void_p()
    try:
        for cx, cy, r, s in p.disks:
            lib.le_set_ball(t, (cx, cy), r, s)
        assert lib.step_n(t, p.steps) == 0
        rc, want = lib.diagnostics(t)
        assert rc == 0
        g = np.zeros(5 * p.nx * p.ny, lib.dtype)
        assert lib.download(t, g) == 0
        soa = aos_to_soa(g, p.nx, p.ny)
        assert rt.cudaMalloc(ctypes.byref(d_ptr), soa.nbytes) == 0
        assert rt.cudaMemcpy(d_ptr, soa.ctypes.data, soa.nbytes, 1) == 0  # host to device
        got = []
        for _ in range(2):  # two calls in a row share the static scratch
            rc, d = lib.diagnostics_noalloc(d_ptr.value, p.nx, p.ny, p.nx, p.nx * p.ny, p.hx, p.hy,
                                            p.c1, p.c2, p.rho)
            assert rc == 0, lib.strerror(rc)
            got.append(d)
        for d in got:
            assert abs(d["energy"] - want["energy"]) <= 1e-12 * abs(want["energy"])
            assert np.allclose(d["sumsq"], want["sumsq"], rtol=1e-12, atol=0)
            assert d["maxabs"] == want["maxabs"]
        assert got[0] == got[1]  # fixed-order reduction: identical results
    finally:
        if d_ptr.value:
            rt.cudaFree(d_ptr)
        lib.le_free_task(t)


def test_noalloc_rejects_too_many_rows():
    lib = capi.Lib("f")
    ny = capi.LE2D_DIAG_NOALLOC_MAX_ROWS + 1
    # rejected by the host-side size check before any device work
    rc, _ = lib.diagnostics_noalloc(256, 8, ny, 8, 8 * ny, 1.0, 1.0, 2.0, 1.0, 1.0)
    assert rc == capi.LE2D_EINVAL


# Run in a child process: it resets the device, which ends every context of the process.
_RESET_SCRIPT = r"""
import ctypes, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from le2d_b200 import capi
from oracle.oracle import ST_AOS, Oracle, aos_to_soa
prec = sys.argv[2]
lib, o = capi.Lib(prec), Oracle(prec)
rt = ctypes.CDLL("libcudart.so")
rt.cudaMalloc.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_size_t]
rt.cudaFree.argtypes = [ctypes.c_void_p]
rt.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
nx, ny = 257, 131
for rnd in range(2):
    g = np.random.default_rng(rnd).uniform(-1, 1, 5 * nx * ny).astype(o.dtype)
    want = o.diag(g, nx, ny, 1.0, 1.0, 2.0, 1.0, 1.5, ST_AOS)
    soa = aos_to_soa(g, nx, ny)
    d = ctypes.c_void_p()
    assert rt.cudaMalloc(ctypes.byref(d), soa.nbytes) == 0
    assert rt.cudaMemcpy(d, soa.ctypes.data, soa.nbytes, 1) == 0
    rc, got = lib.diagnostics_noalloc(d.value, nx, ny, nx, nx * ny, 1.0, 1.0, 2.0, 1.0, 1.5)
    assert rc == 0, lib.strerror(rc)
    assert abs(got["energy"] - want[0]) <= 1e-12 * abs(want[0]), (rnd, got["energy"], want[0])
    assert np.allclose(got["sumsq"], want[1:6], rtol=1e-12, atol=0), rnd
    assert got["maxabs"] == list(want[6:11]), rnd
    assert rt.cudaFree(d) == 0
    if rnd == 0:
        assert rt.cudaDeviceReset() == 0  # a new context: the cached scratch address is stale
print("ok")
"""


@pytest.mark.parametrize("prec", ["f", "d"])
def test_noalloc_after_device_reset(prec):
    """A caller that resets the device (cudaDeviceReset) between two calls: the second call
    looks the scratch array's address up again in the new context and is still correct
    (against the oracle's diagnostics of the same state)."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _RESET_SCRIPT, root, prec], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr

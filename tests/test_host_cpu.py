"""Host-side logic of the library that needs no GPU: material products, the
pressure-disk initial condition, the VTK writer and the error behaviour, against
the golden fixtures made by the reference solver.  On a machine without a CUDA
device the library must refuse to step (LE2D_ENODEV) rather than compute on the CPU."""
import os
import tempfile

import numpy as np
import pytest

from golden_cases import arrays, cases
from le2d_b200 import capi
from oracle.oracle import fields

PRECS = ("f", "d")


@pytest.mark.parametrize("prec", PRECS)
def test_material_bitwise(prec):
    lib = capi.Lib(prec)
    a = arrays(prec)
    for (c1, c2, rho), want in zip(a["materials_in"], a["materials_out"]):
        got = capi.material_array(lib, lib.le_init_material(c1, c2, rho))
        assert got.tobytes() == want.tobytes()


def _no_gpu():
    import ctypes

    try:
        rt = ctypes.CDLL("libcudart.so")
    except OSError:
        return True
    n = ctypes.c_int(0)
    return rt.cudaGetDeviceCount(ctypes.byref(n)) != 0 or n.value == 0


pytestmark_cpu = pytest.mark.skipif(not _no_gpu(), reason="exercises the no-device host path")


@pytestmark_cpu
@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("name", ["ball_64x48", "disks_noise_37x53", "soa_40x32", "tiny_3x7"])
def test_set_ball_host_path_bitwise(prec, name):
    c = cases()[name]
    lib = capi.Lib(prec)
    mat = lib.le_init_material(c["c1"], c["c2"], c["rho"])
    t = lib.le_init_task(c["dt"], (c["hx"], c["hy"]), mat, (c["nx"], c["ny"]), c["stype"])
    try:
        for cx, cy, r, s in c["disks"]:
            lib.le_set_ball(t, (cx, cy), r, s)
        got = fields(lib.grid_view(t).copy(), c["nx"], c["ny"], c["stype"])
        want = fields(arrays(prec)[f"{name}__in"], c["nx"], c["ny"], c["stype"])
        assert got[2:].tobytes() == want[2:].tobytes()
        assert lib.last_error(t) == capi.LE2D_ENODEV
    finally:
        lib.le_free_task(t)


@pytestmark_cpu
@pytest.mark.parametrize("prec", PRECS)
def test_save_task_vtk_bytes(prec):
    c = cases()["ball_64x48"]
    lib = capi.Lib(prec)
    mat = lib.le_init_material(c["c1"], c["c2"], c["rho"])
    t = lib.le_init_task(c["dt"], (c["hx"], c["hy"]), mat, (c["nx"], c["ny"]), c["stype"])
    try:
        lib.grid_view(t)[:] = arrays(prec)["ball_64x48__out"]
        with tempfile.TemporaryDirectory() as td:
            p = os.path.join(td, "x.vtk")
            assert lib.le_save_task(t, p) == 0
            assert open(p, "rb").read() == arrays(prec)["ball_64x48__vtk"].tobytes()
            assert lib.le_save_task(t, os.path.join(td, "no", "such", "dir.vtk")) == 1
    finally:
        lib.le_free_task(t)


@pytestmark_cpu
@pytest.mark.parametrize("prec", PRECS)
def test_step_without_device_fails_loudly(prec, capfd):
    lib = capi.Lib(prec)
    mat = lib.le_init_material(2.0, 1.0, 1.0)
    t = lib.le_init_task(0.25, (1.0, 1.0), mat, (16, 16), capi.ST_AOS)
    try:
        before = lib.grid_view(t).copy()
        lib.le_step(t)
        assert lib.step_n(t, 5) == capi.LE2D_ENODEV
        assert np.array_equal(lib.grid_view(t), before)  # nothing computed on the CPU
        assert "le2d" in capfd.readouterr().err
    finally:
        lib.le_free_task(t)


@pytest.mark.parametrize("prec", PRECS)
def test_error_codes(prec):
    lib = capi.Lib(prec)
    mat = lib.le_init_material(2.0, 1.0, 1.0)
    # a task the library did not create
    stranger = lib.le_task()
    assert lib.last_error(stranger) == capi.LE2D_ENOTASK
    assert lib.step_n(stranger, 1) == capi.LE2D_ENOTASK
    # wrong storage type for the step function
    t = lib.le_init_task(0.25, (1.0, 1.0), mat, (8, 8), capi.ST_SOA)
    try:
        lib.clear_error(t)
        lib.le_step(t)
        assert lib.last_error(t) == capi.LE2D_ESTYPE
        assert lib.strerror(capi.LE2D_ESTYPE)
    finally:
        lib.le_free_task(t)
    # the scheme needs at least 3 nodes per axis
    t = lib.le_init_task(0.25, (1.0, 1.0), mat, (2, 9), capi.ST_AOS)
    try:
        assert lib.last_error(t) == capi.LE2D_EINVAL
        lib.clear_error(t)
        assert lib.step_n(t, 1) in (capi.LE2D_EINVAL,)
    finally:
        lib.le_free_task(t)


def test_device_bytes_accounting():
    lib = capi.Lib("f")
    # two SoA buffers of 5 planes, rows padded to 128 bytes, plus a small diagnostics block
    assert lib.task_device_bytes(100, 10) == 4 * 2 * 5 * 128 * 10 + 128
    assert capi.Lib("d").task_device_bytes(100, 10) == 8 * 2 * 5 * 112 * 10 + 128

"""ctypes binding of the le2d C ABI (include/le_core.h, include/le2d.h).

Mirrors the reference task API (le2d ``simple/le_core.h:217-254``) with the same
names, argument meaning and struct layouts, for Python callers and the test
suite.  ``Lib('f')`` binds lible2d_f.so (real = float), ``Lib('d')`` lible2d_d.so
(real = double).  The library is the product path: if it is missing this module
raises instead of computing anything itself.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(PKG, "lib")

ST_SOA = 0
ST_AOS = 1

LE2D_OK = 0
LE2D_EINVAL = 1
LE2D_ENOTASK = 2
LE2D_ESTYPE = 3
LE2D_ECUDA = 4
LE2D_ENOMEM = 5
LE2D_ENODEV = 6
LE2D_EBUDGET = 7
LE2D_ETIMEOUT = 8
LE2D_ESTATE = 9

LE2D_METHOD_FUSED = 0
LE2D_METHOD_SPLIT = 1

# Every function the headers declare (checked by tests/test_abi.py).
EXPORTS = [
    "le_init_material", "le_init_task", "le_free_task", "le_set_ball", "le_save_task", "le_step",
    "le_step_soa", "le2d_strerror", "le2d_set_device", "le2d_last_error", "le2d_clear_error", "le2d_sync_host",
    "le2d_sync_device", "le2d_wait", "le2d_upload", "le2d_download", "le2d_step_n",
    "le2d_step_n_timed", "le2d_set_method", "le2d_set_variant", "le2d_get_plan", "le2d_sim_time",
    "le2d_diagnostics",
    "le2d_device_layout", "le2d_task_device_bytes", "le2d_host_alloc", "le2d_host_free",
    "le2d_batch_create", "le2d_batch_destroy", "le2d_batch_add", "le2d_batch_run", "le2d_batch_count",
    "le2d_batch_fields", "le2d_batch_receivers", "le2d_batch_diagnostics", "le2d_batch_set_wait_limit",
    "le2d_server_create", "le2d_server_destroy", "le2d_server_submit", "le2d_server_poll",
    "le2d_server_wait", "le2d_server_result", "le2d_server_times", "le2d_server_release",
    "le2d_server_stats", "le2d_now", "le2d_diagnostics_noalloc", "le2d_autotune", "le2d_autotune_reset",
    "le2d_batch_autotune", "le2d_batch_autotune_reset",
    "le2d_slabs_create", "le2d_slabs_destroy", "le2d_slabs_rows", "le2d_slabs_upload",
    "le2d_slabs_download", "le2d_slabs_step_n", "le2d_slabs_wait", "le2d_selftest_ratio", "le2d_selftest_limiter", "le2d_launch_parts",
    "le2d_rows_out", "le2d_rows_in", "le2d_check_violations",
]

LE2D_DIAG_NOALLOC_MAX_ROWS = 16384

LE2D_WANT_FIELDS = 0
LE2D_WANT_RECEIVERS = 1


class le2d_server_stats_t(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_longlong), ("admitted", ctypes.c_longlong),
                ("completed", ctypes.c_longlong), ("failed", ctypes.c_longlong),
                ("node_updates", ctypes.c_longlong), ("windows", ctypes.c_longlong),
                ("device_busy_s", ctypes.c_double), ("arena_used", ctypes.c_size_t),
                ("arena_capacity", ctypes.c_size_t), ("active", ctypes.c_int), ("queued", ctypes.c_int)]


class LibraryMissing(RuntimeError):
    pass


def lib_path(prec: str, checked: bool = False) -> str:
    return os.path.join(LIBDIR, "checked" if checked else "", f"lible2d_{prec}.so")


def _types(prec: str):
    real = ctypes.c_float if prec == "f" else ctypes.c_double

    class le_vec2(ctypes.Structure):
        _fields_ = [("x", real), ("y", real)]

    class le_point2(ctypes.Structure):
        _fields_ = [("x", ctypes.c_int), ("y", ctypes.c_int)]

    class le_material(ctypes.Structure):
        _fields_ = [(n, real) for n in ("c1", "c2", "rho", "irhoc1", "irhoc2", "rhoc1", "rhoc2", "rhoc3")]

    class le_task(ctypes.Structure):
        _fields_ = [("dt", real), ("h", le_vec2), ("n", le_point2), ("mat", le_material),
                    ("stype", ctypes.c_int), ("grid", ctypes.POINTER(real))]

    class le2d_diag_t(ctypes.Structure):
        _fields_ = [("energy", ctypes.c_double), ("sumsq", ctypes.c_double * 5),
                    ("maxabs", ctypes.c_double * 5)]

    class le2d_problem(ctypes.Structure):
        _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("hx", real), ("hy", real), ("dt", real),
                    ("c1", real), ("c2", real), ("rho", real), ("steps", ctypes.c_int), ("stype", ctypes.c_int),
                    ("receiver_row", ctypes.c_int), ("receiver_every", ctypes.c_int)]

    return real, le_vec2, le_point2, le_material, le_task, le2d_diag_t, le2d_problem


class Lib:
    """One precision of the library ('f' or 'd')."""

    def __init__(self, prec: str = "f", checked: bool = False):
        path = lib_path(prec, checked)
        if not os.path.exists(path):
            raise LibraryMissing(f"{path} is not built (python -m le2d_b200.build)")
        self.prec = prec
        self.dtype = np.float32 if prec == "f" else np.float64
        self.lib = ctypes.CDLL(path)
        (self.real, self.le_vec2, self.le_point2, self.le_material, self.le_task,
         self.le2d_diag_t, self.le2d_problem) = _types(prec)
        L, R = self.lib, self.real
        P = ctypes.POINTER
        L.le_init_material.argtypes = [R, R, R, P(self.le_material)]
        L.le_init_material.restype = None
        L.le_init_task.argtypes = [P(self.le_task), R, self.le_vec2, self.le_material, self.le_point2,
                                   ctypes.c_int]
        L.le_init_task.restype = None
        L.le_free_task.argtypes = [P(self.le_task)]
        L.le_free_task.restype = None
        L.le_set_ball.argtypes = [P(self.le_task), self.le_vec2, R, R]
        L.le_set_ball.restype = None
        L.le_save_task.argtypes = [P(self.le_task), ctypes.c_char_p]
        L.le_step.argtypes = [P(self.le_task)]
        L.le_step.restype = None
        L.le_step_soa.argtypes = [P(self.le_task)]
        L.le_step_soa.restype = None
        L.le2d_strerror.argtypes = [ctypes.c_int]
        L.le2d_strerror.restype = ctypes.c_char_p
        L.le2d_set_device.argtypes = [ctypes.c_int]
        for name in ("le2d_last_error", "le2d_clear_error", "le2d_sync_host", "le2d_sync_device",
                     "le2d_wait"):
            getattr(L, name).argtypes = [P(self.le_task)]
        L.le2d_upload.argtypes = [P(self.le_task), ctypes.c_void_p]
        L.le2d_download.argtypes = [P(self.le_task), ctypes.c_void_p]
        L.le2d_step_n.argtypes = [P(self.le_task), ctypes.c_int]
        L.le2d_step_n_timed.argtypes = [P(self.le_task), ctypes.c_int, P(ctypes.c_float)]
        L.le2d_set_method.argtypes = [P(self.le_task), ctypes.c_int]
        L.le2d_set_variant.argtypes = [P(self.le_task), ctypes.c_int, ctypes.c_int]
        L.le2d_get_plan.argtypes = [P(self.le_task), P(ctypes.c_int)]
        L.le2d_sim_time.argtypes = [P(self.le_task), P(ctypes.c_double), P(ctypes.c_longlong)]
        L.le2d_diagnostics.argtypes = [P(self.le_task), P(self.le2d_diag_t)]
        L.le2d_device_layout.argtypes = [P(self.le_task), P(ctypes.c_longlong), P(ctypes.c_longlong)]
        L.le2d_task_device_bytes.argtypes = [ctypes.c_int, ctypes.c_int]
        L.le2d_task_device_bytes.restype = ctypes.c_size_t
        L.le2d_host_alloc.argtypes = [ctypes.c_size_t]
        L.le2d_host_alloc.restype = ctypes.c_void_p
        L.le2d_host_free.argtypes = [ctypes.c_void_p]
        L.le2d_host_free.restype = None
        L.le2d_batch_create.argtypes = [ctypes.c_size_t]
        L.le2d_batch_create.restype = ctypes.c_void_p
        L.le2d_batch_destroy.argtypes = [ctypes.c_void_p]
        L.le2d_batch_destroy.restype = None
        L.le2d_batch_add.argtypes = [ctypes.c_void_p, P(self.le2d_problem), ctypes.c_void_p, ctypes.c_int,
                                     ctypes.c_void_p]
        L.le2d_batch_run.argtypes = [ctypes.c_void_p, ctypes.c_int, P(ctypes.c_float)]
        L.le2d_batch_count.argtypes = [ctypes.c_void_p]
        L.le2d_batch_fields.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.le2d_batch_receivers.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, P(ctypes.c_int)]
        L.le2d_batch_diagnostics.argtypes = [ctypes.c_void_p, ctypes.c_int, P(self.le2d_diag_t)]
        L.le2d_batch_set_wait_limit.argtypes = [ctypes.c_void_p, ctypes.c_ulonglong]
        L.le2d_server_create.argtypes = [ctypes.c_size_t, ctypes.c_int, ctypes.c_int]
        L.le2d_server_create.restype = ctypes.c_void_p
        L.le2d_server_destroy.argtypes = [ctypes.c_void_p]
        L.le2d_server_destroy.restype = None
        L.le2d_server_submit.argtypes = [ctypes.c_void_p, P(self.le2d_problem), ctypes.c_void_p, ctypes.c_int,
                                         ctypes.c_void_p, ctypes.c_int]
        L.le2d_server_submit.restype = ctypes.c_longlong
        L.le2d_server_poll.argtypes = [ctypes.c_void_p, ctypes.c_longlong]
        L.le2d_server_wait.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_double]
        L.le2d_server_result.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p, ctypes.c_size_t,
                                         P(ctypes.c_int)]
        L.le2d_server_times.argtypes = [ctypes.c_void_p, ctypes.c_longlong, P(ctypes.c_double),
                                        P(ctypes.c_double), P(ctypes.c_double)]
        L.le2d_server_release.argtypes = [ctypes.c_void_p, ctypes.c_longlong]
        L.le2d_server_stats.argtypes = [ctypes.c_void_p, P(le2d_server_stats_t)]
        L.le2d_now.restype = ctypes.c_double
        L.le2d_autotune.argtypes = [ctypes.c_int, ctypes.c_int, P(ctypes.c_int), P(ctypes.c_double)]
        L.le2d_autotune_reset.argtypes = []
        L.le2d_batch_autotune.argtypes = [ctypes.c_int, ctypes.c_int, P(ctypes.c_int), P(ctypes.c_double)]
        L.le2d_batch_autotune_reset.argtypes = []
        L.le2d_slabs_create.restype = ctypes.c_void_p
        L.le2d_slabs_create.argtypes = [P(self.le_task), ctypes.c_int, P(ctypes.c_int)]
        L.le2d_slabs_destroy.argtypes = [ctypes.c_void_p]
        L.le2d_slabs_rows.argtypes = [ctypes.c_void_p, ctypes.c_int, P(ctypes.c_int), P(ctypes.c_int),
                                      P(ctypes.c_int)]
        L.le2d_slabs_upload.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.le2d_slabs_download.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.le2d_slabs_step_n.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.le2d_slabs_wait.argtypes = [ctypes.c_void_p]
        L.le2d_check_violations.argtypes = [P(ctypes.c_ulonglong)]
        L.le2d_rows_out.argtypes = [P(self.le_task), ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        L.le2d_rows_in.argtypes = [P(self.le_task), ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        L.le2d_selftest_ratio.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong,
                                          ctypes.c_void_p, ctypes.c_void_p]
        L.le2d_launch_parts.argtypes = [P(self.le_task), P(ctypes.c_int)]
        L.le2d_selftest_limiter.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_longlong,
                                            ctypes.c_void_p]
        L.le2d_diagnostics_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_longlong,
                                               ctypes.c_longlong, R, R, R, R, R, ctypes.c_void_p,
                                               P(self.le2d_diag_t)]

    # --- the reference task API, same names ---
    def le_init_material(self, c1, c2, rho):
        m = self.le_material()
        self.lib.le_init_material(c1, c2, rho, ctypes.byref(m))
        return m

    def le_init_task(self, dt, h, mat, n, stype):
        t = self.le_task()
        self.lib.le_init_task(ctypes.byref(t), dt, self.le_vec2(*h), mat, self.le_point2(*n), stype)
        return t

    def le_free_task(self, t):
        self.lib.le_free_task(ctypes.byref(t))

    def le_set_ball(self, t, c, r, s):
        self.lib.le_set_ball(ctypes.byref(t), self.le_vec2(*c), r, s)

    def le_save_task(self, t, path: str) -> int:
        return self.lib.le_save_task(ctypes.byref(t), path.encode())

    def le_step(self, t):
        self.lib.le_step(ctypes.byref(t))

    def le_step_soa(self, t):
        self.lib.le_step_soa(ctypes.byref(t))

    # --- extensions ---
    def strerror(self, code: int) -> str:
        return self.lib.le2d_strerror(code).decode()

    def set_device(self, device: int) -> int:
        return self.lib.le2d_set_device(device)

    def last_error(self, t) -> int:
        return self.lib.le2d_last_error(ctypes.byref(t))

    def clear_error(self, t) -> int:
        return self.lib.le2d_clear_error(ctypes.byref(t))

    def sync_host(self, t) -> int:
        return self.lib.le2d_sync_host(ctypes.byref(t))

    def sync_device(self, t) -> int:
        return self.lib.le2d_sync_device(ctypes.byref(t))

    def wait(self, t) -> int:
        return self.lib.le2d_wait(ctypes.byref(t))

    def upload(self, t, src: np.ndarray) -> int:
        assert src.dtype == self.dtype and src.flags["C_CONTIGUOUS"]
        return self.lib.le2d_upload(ctypes.byref(t), src.ctypes.data)

    def download(self, t, dst: np.ndarray) -> int:
        assert dst.dtype == self.dtype and dst.flags["C_CONTIGUOUS"]
        return self.lib.le2d_download(ctypes.byref(t), dst.ctypes.data)

    def step_n(self, t, n: int) -> int:
        return self.lib.le2d_step_n(ctypes.byref(t), n)

    def step_n_timed(self, t, n: int):
        ms = ctypes.c_float(0.0)
        rc = self.lib.le2d_step_n_timed(ctypes.byref(t), n, ctypes.byref(ms))
        return rc, ms.value

    def set_method(self, t, method: int) -> int:
        return self.lib.le2d_set_method(ctypes.byref(t), method)

    def set_variant(self, t, variant: int, seg_len: int = 0) -> int:
        return self.lib.le2d_set_variant(ctypes.byref(t), variant, seg_len)

    PLAN_KEYS = ("variant", "lanes", "seg_len", "nstrips", "ntasks", "blocks", "depth", "warps_per_task")

    def launch_parts(self, t) -> int:
        """Kernel launches per fused launch of the grid (3 when the task launches in halves)."""
        v = ctypes.c_int(0)
        rc = self.lib.le2d_launch_parts(ctypes.byref(t), ctypes.byref(v))
        if rc:
            raise RuntimeError(self.strerror(rc))
        return v.value

    def get_plan(self, t) -> dict:
        out = (ctypes.c_int * len(self.PLAN_KEYS))()
        rc = self.lib.le2d_get_plan(ctypes.byref(t), out)
        if rc:
            raise RuntimeError(self.strerror(rc))
        return dict(zip(self.PLAN_KEYS, list(out)))

    def autotune(self, nx: int, ny: int):
        out = (ctypes.c_int * len(self.PLAN_KEYS))()
        nus = ctypes.c_double(0.0)
        rc = self.lib.le2d_autotune(nx, ny, out, ctypes.byref(nus))
        if rc:
            raise RuntimeError(self.strerror(rc))
        return dict(zip(self.PLAN_KEYS, list(out))), nus.value

    def autotune_reset(self) -> int:
        return self.lib.le2d_autotune_reset()

    def batch_autotune(self, nx: int, ny: int):
        """Tunes the batched path for the size class of nx x ny: ({seg_len, depth}, nu/s)."""
        out = (ctypes.c_int * 2)()
        nus = ctypes.c_double(0.0)
        rc = self.lib.le2d_batch_autotune(nx, ny, out, ctypes.byref(nus))
        if rc:
            raise RuntimeError(self.strerror(rc))
        return {"seg_len": out[0], "depth": out[1]}, nus.value

    def batch_autotune_reset(self) -> int:
        return self.lib.le2d_batch_autotune_reset()

    def selftest_ratio(self, a: np.ndarray, b: np.ndarray):
        """The step kernels' FP64 slope-ratio division and IEEE division of a / b, on the device."""
        a = np.ascontiguousarray(a, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        assert a.shape == b.shape and a.ndim == 1
        fast, ieee = np.empty_like(a), np.empty_like(a)
        rc = self.lib.le2d_selftest_ratio(a.ctypes.data, b.ctypes.data, a.size, fast.ctypes.data,
                                          ieee.ctypes.data)
        if rc:
            raise RuntimeError(self.strerror(rc))
        return fast, ieee

    def selftest_limiter(self, a: np.ndarray, b: np.ndarray, kc: float) -> np.ndarray:
        """kc * superbee(a / b) as the FP64 step kernels form it, on the device."""
        a = np.ascontiguousarray(a, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        assert a.shape == b.shape and a.ndim == 1
        out = np.empty_like(a)
        rc = self.lib.le2d_selftest_limiter(a.ctypes.data, b.ctypes.data, kc, a.size, out.ctypes.data)
        if rc:
            raise RuntimeError(self.strerror(rc))
        return out

    def sim_time(self, t):
        tt, st = ctypes.c_double(0.0), ctypes.c_longlong(0)
        rc = self.lib.le2d_sim_time(ctypes.byref(t), ctypes.byref(tt), ctypes.byref(st))
        return rc, tt.value, st.value

    def diagnostics(self, t):
        d = self.le2d_diag_t()
        rc = self.lib.le2d_diagnostics(ctypes.byref(t), ctypes.byref(d))
        return rc, {"energy": d.energy, "sumsq": list(d.sumsq), "maxabs": list(d.maxabs)}

    def diagnostics_noalloc(self, d_state: int, nx: int, ny: int, pitch: int, plane: int, hx, hy, c1, c2, rho,
                            stream: int = 0):
        """Diagnostics of a device state the caller holds (device pointer `d_state`)."""
        d = self.le2d_diag_t()
        rc = self.lib.le2d_diagnostics_noalloc(d_state, nx, ny, pitch, plane, hx, hy, c1, c2, rho,
                                               stream or None, ctypes.byref(d))
        return rc, {"energy": d.energy, "sumsq": list(d.sumsq), "maxabs": list(d.maxabs)}

    def check_violations(self):
        """(is_checked_build, state accesses refused since the last call)."""
        n = ctypes.c_ulonglong(0)
        checked = self.lib.le2d_check_violations(ctypes.byref(n))
        return bool(checked), n.value

    def rows_out(self, t, row0: int, nrows: int, dev_ptr: int, stream: int = 0) -> int:
        """Rows of the task's state into a device buffer [5][nrows][nx] (e.g. a CUDA tensor)."""
        return self.lib.le2d_rows_out(ctypes.byref(t), row0, nrows, dev_ptr, stream or None)

    def rows_in(self, t, row0: int, nrows: int, dev_ptr: int, stream: int = 0) -> int:
        """Rows of the task's state from a device buffer [5][nrows][nx]."""
        return self.lib.le2d_rows_in(ctypes.byref(t), row0, nrows, dev_ptr, stream or None)

    def device_layout(self, t):
        p, q = ctypes.c_longlong(0), ctypes.c_longlong(0)
        rc = self.lib.le2d_device_layout(ctypes.byref(t), ctypes.byref(p), ctypes.byref(q))
        return rc, p.value, q.value

    def task_device_bytes(self, nx: int, ny: int) -> int:
        return self.lib.le2d_task_device_bytes(nx, ny)

    def host_array(self, n: int):
        """A page-locked numpy array of n reals and its release function."""
        ptr = self.lib.le2d_host_alloc(n * np.dtype(self.dtype).itemsize)
        if not ptr:
            raise MemoryError("le2d_host_alloc failed")
        buf = (self.real * n).from_address(ptr)
        arr = np.ctypeslib.as_array(buf)
        return arr, (lambda: self.lib.le2d_host_free(ptr))

    # --- helpers ---
    def grid_view(self, t) -> np.ndarray:
        """The host grid (task->grid) as a numpy array (no copy)."""
        n = 5 * t.n.x * t.n.y
        return np.ctypeslib.as_array(t.grid, shape=(n,))


class Batch:
    """le2d_batch_*: many independent solves advanced by one persistent kernel."""

    def __init__(self, lib: Lib, budget_bytes: int = 0):
        self.lib = lib
        self.h = lib.lib.le2d_batch_create(budget_bytes)
        if not self.h:
            raise RuntimeError("le2d_batch_create failed")
        self.problems = []

    def close(self):
        if self.h:
            self.lib.lib.le2d_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def problem(self, p, stype=ST_AOS, receiver_row=-1, receiver_every=10):
        """A le2d_problem from a workloads.Problem."""
        return self.lib.le2d_problem(p.nx, p.ny, p.hx, p.hy, p.dt, p.c1, p.c2, p.rho, p.steps, stype,
                                     receiver_row, receiver_every)

    def add(self, prob, init: np.ndarray | None = None, disks=()) -> int:
        d = np.ascontiguousarray(np.asarray(disks, dtype=self.lib.dtype).reshape(-1))
        ip = None
        if init is not None:
            init = np.ascontiguousarray(init, dtype=self.lib.dtype)
            ip = init.ctypes.data
        rid = self.lib.lib.le2d_batch_add(self.h, ctypes.byref(prob), ip, len(d) // 4,
                                          d.ctypes.data if len(d) else None)
        if rid >= 0:
            self.problems.append(prob)
        return rid

    def run(self, window_steps: int = 256):
        ms = ctypes.c_float(0.0)
        rc = self.lib.lib.le2d_batch_run(self.h, window_steps, ctypes.byref(ms))
        return rc, ms.value

    def fields(self, rid: int) -> np.ndarray:
        p = self.problems[rid]
        out = np.zeros(5 * p.nx * p.ny, self.lib.dtype)
        rc = self.lib.lib.le2d_batch_fields(self.h, rid, out.ctypes.data)
        if rc:
            raise RuntimeError(self.lib.strerror(rc))
        return out

    def receivers(self, rid: int) -> np.ndarray:
        p = self.problems[rid]
        n = ctypes.c_int(0)
        rc = self.lib.lib.le2d_batch_receivers(self.h, rid, None, ctypes.byref(n))
        out = np.zeros((n.value, 2, p.nx), self.lib.dtype)
        rc = self.lib.lib.le2d_batch_receivers(self.h, rid, out.ctypes.data, ctypes.byref(n))
        if rc:
            raise RuntimeError(self.lib.strerror(rc))
        return out

    def diagnostics(self, rid: int):
        d = self.lib.le2d_diag_t()
        rc = self.lib.lib.le2d_batch_diagnostics(self.h, rid, ctypes.byref(d))
        return rc, {"energy": d.energy, "sumsq": list(d.sumsq), "maxabs": list(d.maxabs)}

    def set_wait_limit(self, ns: int) -> int:
        return self.lib.lib.le2d_batch_set_wait_limit(self.h, ns)


class Slabs:
    """le2d_slabs_*: one grid split into row slabs over several devices."""

    def __init__(self, lib: Lib, task, devices):
        self.lib = lib
        self.n = 5 * task.n.x * task.n.y
        devs = (ctypes.c_int * len(devices))(*devices)
        self.h = lib.lib.le2d_slabs_create(ctypes.byref(task), len(devices), devs)
        if not self.h:
            raise RuntimeError("le2d_slabs_create failed")
        self.count = len(devices)

    def close(self):
        if self.h:
            self.lib.lib.le2d_slabs_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def rows(self, i: int):
        r0, r1, d = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
        rc = self.lib.lib.le2d_slabs_rows(self.h, i, ctypes.byref(r0), ctypes.byref(r1), ctypes.byref(d))
        if rc:
            raise RuntimeError(self.lib.strerror(rc))
        return r0.value, r1.value, d.value

    def upload(self, src: np.ndarray) -> int:
        src = np.ascontiguousarray(src, dtype=self.lib.dtype)
        assert src.size == self.n
        return self.lib.lib.le2d_slabs_upload(self.h, src.ctypes.data)

    def download(self) -> np.ndarray:
        out = np.zeros(self.n, self.lib.dtype)
        rc = self.lib.lib.le2d_slabs_download(self.h, out.ctypes.data)
        if rc:
            raise RuntimeError(self.lib.strerror(rc))
        return out

    def step_n(self, n: int) -> int:
        return self.lib.lib.le2d_slabs_step_n(self.h, n)

    def wait(self) -> int:
        return self.lib.lib.le2d_slabs_wait(self.h)


class Server:
    """le2d_server_*: continuous-batching request loop (a background thread in the library)."""

    def __init__(self, lib: Lib, budget_bytes: int = 0, window_steps: int = 100, max_active: int = 1024):
        self.lib = lib
        self.h = lib.lib.le2d_server_create(budget_bytes, window_steps, max_active)
        if not self.h:
            raise RuntimeError("le2d_server_create failed")
        self.meta = {}

    def close(self):
        if self.h:
            self.lib.lib.le2d_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, prob, init=None, disks=(), want=LE2D_WANT_FIELDS) -> int:
        d = np.ascontiguousarray(np.asarray(disks, dtype=self.lib.dtype).reshape(-1))
        ip = None
        if init is not None:
            init = np.ascontiguousarray(init, dtype=self.lib.dtype)
            ip = init.ctypes.data
        t = self.lib.lib.le2d_server_submit(self.h, ctypes.byref(prob), ip, len(d) // 4,
                                            d.ctypes.data if len(d) else None, want)
        if t > 0:
            self.meta[t] = (prob.nx, prob.ny, want)
        return t

    def poll(self, ticket) -> int:
        return self.lib.lib.le2d_server_poll(self.h, ticket)

    def wait(self, ticket, timeout_s: float = -1.0) -> int:
        return self.lib.lib.le2d_server_wait(self.h, ticket, timeout_s)

    def result(self, ticket) -> np.ndarray:
        nx, ny, want = self.meta[ticket]
        n = ctypes.c_int(0)
        if want == LE2D_WANT_FIELDS:
            out = np.zeros(5 * nx * ny, self.lib.dtype)
        else:
            rc = self.lib.lib.le2d_server_result(self.h, ticket, None, 0, ctypes.byref(n))
            if rc:
                raise RuntimeError(self.lib.strerror(rc))
            out = np.zeros((n.value, 2, nx), self.lib.dtype)
        rc = self.lib.lib.le2d_server_result(self.h, ticket, out.ctypes.data, out.size, ctypes.byref(n))
        if rc:
            raise RuntimeError(self.lib.strerror(rc))
        return out

    def times(self, ticket):
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        rc = self.lib.lib.le2d_server_times(self.h, ticket, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        if rc:
            raise RuntimeError(self.lib.strerror(rc))
        return a.value, b.value, c.value

    def release(self, ticket) -> int:
        self.meta.pop(ticket, None)
        return self.lib.lib.le2d_server_release(self.h, ticket)

    def stats(self) -> dict:
        s = le2d_server_stats_t()
        self.lib.lib.le2d_server_stats(self.h, ctypes.byref(s))
        return {k: getattr(s, k) for k, _ in s._fields_}

    def now(self) -> float:
        return self.lib.lib.le2d_now()


def material_array(lib: Lib, m) -> np.ndarray:
    return np.array([m.c1, m.c2, m.rho, m.irhoc1, m.irhoc2, m.rhoc1, m.rhoc2, m.rhoc3], dtype=lib.dtype)

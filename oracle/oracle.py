"""ctypes wrapper for the CPU checker -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline / reference
legs use this module.  It loads:

* ``oracle/_build/liboracle_{f,d}.so`` -- ``le2d_oracle.c``, a C restatement of the
  reference solver's step (le2d ``simple/le_core.c:48-69,171-257,435-627``) that
  matches the reference's float and double builds bit for bit;
* ``oracle/_ref/libref_simple_{f,d}.so`` -- the reference's own ``simple/le_core.c``
  behind ``ref_simple_driver.c`` (present when it was built from the reference
  sources);
* ``oracle/_ref/libref_pthread_{f,d}.so`` -- the reference's ``pthread/le_core.c``
  (speed baseline only; its tvd2 differs numerically from ``simple/``).

Grids are numpy arrays of 5*nx*ny reals: AOS ``[j][i][field]`` (ST_AOS = 1) or
SoA ``[field][j][i]`` (ST_SOA = 0), fields (vx, vy, sxx, sxy, syy).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD_DIR = os.path.join(HERE, "_build")
REF_DIR = os.path.join(HERE, "_ref")
# Where the reference project's sources are mounted (read-only): LE2D_REFERENCE, else the
# mount point of this build environment.  Absent on machines that only run the prebuilt
# oracle/_ref libraries.
REFERENCE_ROOT = os.environ.get("LE2D_REFERENCE", "/root/reference")

ST_SOA = 0
ST_AOS = 1

_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double


def build(reference_root: str | None = REFERENCE_ROOT) -> None:
    """Compile the restatement and, when the reference sources exist, oracle/_ref."""
    cmd = ["make", "-s", "-C", HERE, "oracle"]
    subprocess.run(cmd, check=True)
    if reference_root and os.path.exists(os.path.join(reference_root, "simple", "le_core.c")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={reference_root}"], check=True)


def _real(prec: str):
    return ctypes.c_float if prec == "f" else ctypes.c_double


def np_dtype(prec: str):
    return np.float32 if prec == "f" else np.float64


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_P)


class Oracle:
    """The C restatement, one precision ('f' or 'd')."""

    def __init__(self, prec: str):
        self.prec = prec
        path = os.path.join(BUILD_DIR, f"liboracle_{prec}.so")
        if not os.path.exists(path):
            build(None)
        self.lib = ctypes.CDLL(path)
        R = _real(prec)
        L = self.lib
        L.oracle_material.argtypes = [R, R, R, _P]
        L.oracle_step.argtypes = [_P, _I, _I, R, R, R, _P, _I]
        L.oracle_run.argtypes = [_P, _I, _I, R, R, R, _P, _I, _I]
        L.oracle_set_ball.argtypes = [_P, _I, _I, R, R, _I, R, R, R, R]
        L.oracle_save_vtk.argtypes = [_P, _I, _I, R, R, _I, ctypes.c_char_p]
        L.oracle_diag.argtypes = [_P, _I, _I, _D, _D, _D, _D, _D, _I, _P]
        assert L.oracle_real_size() == (4 if prec == "f" else 8)
        self.dtype = np_dtype(prec)

    def material(self, c1, c2, rho) -> np.ndarray:
        out = np.zeros(8, self.dtype)
        self.lib.oracle_material(c1, c2, rho, _ptr(out))
        return out

    def set_ball(self, grid, nx, ny, hx, hy, stype, cx, cy, r, s):
        rc = self.lib.oracle_set_ball(_ptr(grid), nx, ny, hx, hy, stype, cx, cy, r, s)
        assert rc == 0

    def run(self, grid, nx, ny, dt, hx, hy, c1, c2, rho, stype, steps):
        mat = self.material(c1, c2, rho)
        rc = self.lib.oracle_run(_ptr(grid), nx, ny, dt, hx, hy, _ptr(mat), stype, steps)
        assert rc == 0

    def save_vtk(self, grid, nx, ny, hx, hy, stype, path):
        return self.lib.oracle_save_vtk(_ptr(grid), nx, ny, hx, hy, stype, path.encode())

    def diag(self, grid, nx, ny, hx, hy, c1, c2, rho, stype) -> np.ndarray:
        out = np.zeros(11, np.float64)
        self.lib.oracle_diag(_ptr(grid), nx, ny, hx, hy, c1, c2, rho, stype, _ptr(out))
        return out


class Reference:
    """The reference's own simple/ solver (oracle/_ref), one precision."""

    def __init__(self, prec: str):
        path = os.path.join(REF_DIR, f"libref_simple_{prec}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.prec = prec
        self.dtype = np_dtype(prec)
        R = _real(prec)
        L = self.lib = ctypes.CDLL(path)
        L.ref_material.argtypes = [R, R, R, _P]
        L.ref_initial_state.argtypes = [_I, _I, R, R, _I, _I, _P, _P, _P, _P, _P]
        L.ref_run.argtypes = [_I, _I, R, R, R, R, R, R, _I, _P, _I, _I]
        L.ref_run.restype = _D
        L.ref_save.argtypes = [_I, _I, R, R, _I, _P, ctypes.c_char_p]
        assert L.ref_real_size() == (4 if prec == "f" else 8)

    @staticmethod
    def available(prec: str = "d") -> bool:
        return os.path.exists(os.path.join(REF_DIR, f"libref_simple_{prec}.so"))

    def material(self, c1, c2, rho) -> np.ndarray:
        out = np.zeros(8, self.dtype)
        self.lib.ref_material(c1, c2, rho, _ptr(out))
        return out

    def initial_state(self, nx, ny, hx, hy, stype, disks) -> np.ndarray:
        out = np.zeros(5 * nx * ny, self.dtype)
        d = np.asarray(disks, dtype=self.dtype).reshape(-1, 4)
        cols = [np.ascontiguousarray(d[:, k]) for k in range(4)]
        rc = self.lib.ref_initial_state(nx, ny, hx, hy, stype, len(d), *[_ptr(c) for c in cols], _ptr(out))
        assert rc == 0
        return out

    def run(self, grid, nx, ny, dt, hx, hy, c1, c2, rho, stype, steps, threads=0) -> float:
        t = self.lib.ref_run(nx, ny, dt, hx, hy, c1, c2, rho, stype, _ptr(grid), steps, threads)
        assert t >= 0
        return t

    def save_vtk(self, grid, nx, ny, hx, hy, stype, path):
        return self.lib.ref_save(nx, ny, hx, hy, stype, _ptr(grid), path.encode())


class ReferencePthread:
    """The reference's pthread/ solver (speed baseline only)."""

    def __init__(self, prec: str):
        path = os.path.join(REF_DIR, f"libref_pthread_{prec}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.dtype = np_dtype(prec)
        R = _real(prec)
        L = self.lib = ctypes.CDLL(path)
        L.ref_pthread_run.argtypes = [_I, _I, R, R, R, R, R, R, _P, _I, _I]
        L.ref_pthread_run.restype = _D

    @staticmethod
    def available(prec: str = "d") -> bool:
        return os.path.exists(os.path.join(REF_DIR, f"libref_pthread_{prec}.so"))

    def run(self, grid, nx, ny, dt, hx, hy, c1, c2, rho, steps, threads) -> float:
        p = _ptr(grid) if grid is not None else None
        t = self.lib.ref_pthread_run(nx, ny, dt, hx, hy, c1, c2, rho, p, steps, threads)
        assert t >= 0, t
        return t


class ReferenceTiling:
    """The reference's two-buffer schedule tiling/ le_step_all2 (oracle/_ref), one precision:
    zero ring of two nodes around the grid, increments associated (v + d1) + d2."""

    def __init__(self, prec: str):
        path = os.path.join(REF_DIR, f"libref_tiling_{prec}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.dtype = np_dtype(prec)
        L = self.lib = ctypes.CDLL(path)
        R = _real(prec)
        L.ref_tiling_run.argtypes = [_I, _I, R, R, R, R, R, R, _P, _I]
        assert L.ref_tiling_real_size() == (4 if prec == "f" else 8)

    @staticmethod
    def available(prec: str = "d") -> bool:
        return os.path.exists(os.path.join(REF_DIR, f"libref_tiling_{prec}.so"))

    def run(self, grid, nx, ny, dt, hx, hy, c1, c2, rho, steps):
        assert self.lib.ref_tiling_run(nx, ny, dt, hx, hy, c1, c2, rho, _ptr(grid), steps) == 0


def aos_to_soa(g: np.ndarray, nx: int, ny: int) -> np.ndarray:
    return np.ascontiguousarray(g.reshape(ny, nx, 5).transpose(2, 0, 1)).reshape(-1)


def soa_to_aos(g: np.ndarray, nx: int, ny: int) -> np.ndarray:
    return np.ascontiguousarray(g.reshape(5, ny, nx).transpose(1, 2, 0)).reshape(-1)


def fields(g: np.ndarray, nx: int, ny: int, stype: int) -> np.ndarray:
    """(5, ny, nx) view-copy of a grid in either layout."""
    if stype == ST_AOS:
        return np.ascontiguousarray(g.reshape(ny, nx, 5).transpose(2, 0, 1))
    return g.reshape(5, ny, nx).copy()


def rel_l2(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Per-field relative L2 of a against b, both (5, ny, nx); computed in float64."""
    a = a.astype(np.float64).reshape(5, -1)
    b = b.astype(np.float64).reshape(5, -1)
    num = np.sqrt(((a - b) ** 2).sum(axis=1))
    den = np.sqrt((b**2).sum(axis=1))
    return np.where(den > 0, num / np.where(den > 0, den, 1.0), num)


def max_abs(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    a = a.astype(np.float64).reshape(5, -1)
    b = b.astype(np.float64).reshape(5, -1)
    return np.abs(a - b).max(axis=1)

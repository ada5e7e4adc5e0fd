"""One grid over several processes, one per GPU: row slabs with a halo exchange over
torch.distributed (NCCL send/recv of device buffers on the GPU path).

The decomposition is the one le2d_slabs_* use inside one process (the reference's
multi-GPU scheme, le2d cuda5/cuda6 le_core.cu:374-509): rank k owns the global rows
[r0, r1) of an ny-row grid and keeps kHalo = 4 copied rows beside each cut, so its local
grid is the rows [r0 - h0, r1 + h1).  It steps its local grid with the library's
unmodified step (clamped ends at the local top and bottom, which spoil only the halo
rows: two rows per step), at most two steps between exchanges, and then swaps the 4
owned rows beside each cut with the neighbour: they become the neighbour's halo rows.
So after every exchange the owned rows equal those of the whole grid stepped by one task.

SlabExchange does the swap for any pair of row accessors (device rows through
le2d_rows_out / le2d_rows_in on the GPU path, host arrays in the CPU tests) with one
batch of torch.distributed point-to-point operations per exchange; GpuRankSlab drives a
library task on this rank's GPU.
"""
from __future__ import annotations

import numpy as np

from le2d_b200 import capi

HALO = 4  # rows: two steps between exchanges, two rows per step
MIN_ROWS = 8  # owned rows per rank


def partition(ny: int, world: int, rank: int, halo: int = HALO):
    """(r0, r1, h0, h1): owned global rows [r0, r1) and halo rows above / below."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank")
    if ny < MIN_ROWS * world:
        raise ValueError(f"needs at least {MIN_ROWS} rows per rank")
    r0 = ny * rank // world
    r1 = ny * (rank + 1) // world
    return r0, r1, (halo if rank > 0 else 0), (halo if rank + 1 < world else 0)


class SlabExchange:
    """Swaps the owned rows beside each cut with the neighbouring ranks.

    get_rows(row0, nrows, buf) fills buf[5, nrows, nx] from local rows [row0, row0+nrows);
    put_rows(row0, nrows, buf) writes them back.  Local row indices: the owned rows are
    [h0, h0 + r1 - r0)."""

    def __init__(self, dist, rank: int, world: int, nx: int, ny: int, make_buffer, halo: int = HALO):
        self.dist, self.rank, self.world, self.halo = dist, rank, world, halo
        self.r0, self.r1, self.h0, self.h1 = partition(ny, world, rank, halo)
        self.own = self.r1 - self.r0
        self.nyl = self.h0 + self.own + self.h1
        self.up = [make_buffer((5, halo, nx)) for _ in range(2)] if rank > 0 else None
        self.down = [make_buffer((5, halo, nx)) for _ in range(2)] if rank + 1 < world else None

    def exchange(self, get_rows, put_rows):
        d, h = self.dist, self.halo
        ops = []
        if self.up:  # my first owned rows up; the rank above's last owned rows into my top halo
            get_rows(self.h0, h, self.up[0])
            ops += [d.P2POp(d.isend, self.up[0], self.rank - 1), d.P2POp(d.irecv, self.up[1], self.rank - 1)]
        if self.down:  # my last owned rows down; the rank below's first owned rows into my bottom halo
            get_rows(self.h0 + self.own - h, h, self.down[0])
            ops += [d.P2POp(d.isend, self.down[0], self.rank + 1),
                    d.P2POp(d.irecv, self.down[1], self.rank + 1)]
        if ops:
            for w in d.batch_isend_irecv(ops):
                w.wait()
        if self.up:
            put_rows(0, h, self.up[1])
        if self.down:
            put_rows(self.h0 + self.own, h, self.down[1])


def local_rows(grid: np.ndarray, nx: int, ny: int, stype: int, g0: int, g1: int) -> np.ndarray:
    """Rows [g0, g1) of a whole grid in the task layout, as a new grid of g1 - g0 rows."""
    if stype == capi.ST_AOS:
        return np.array(grid.reshape(ny, nx, 5)[g0:g1]).reshape(-1)
    return np.array(grid.reshape(5, ny, nx)[:, g0:g1]).reshape(-1)


class GpuRankSlab:
    """This rank's slab as a library task on its GPU; the halo rows travel through
    torch.distributed (NCCL) on torch's current stream."""

    def __init__(self, lib: capi.Lib, dist, rank: int, world: int, nx: int, ny: int, dt, h, c1, c2, rho,
                 stype: int = capi.ST_AOS):
        import torch

        self.torch = torch
        self.lib, self.nx, self.ny, self.stype = lib, nx, ny, stype
        dtype = torch.float32 if lib.prec == "f" else torch.float64
        self.x = SlabExchange(dist, rank, world, nx, ny,
                              lambda shape: torch.empty(shape, dtype=dtype, device="cuda"))
        mat = lib.le_init_material(c1, c2, rho)
        self.task = lib.le_init_task(dt, h, mat, (nx, self.x.nyl), stype)
        if not self.task.grid or lib.last_error(self.task):
            raise RuntimeError("le_init_task failed")

    def close(self):
        if self.task is not None:
            self.lib.le_free_task(self.task)
            self.task = None

    def upload(self, whole: np.ndarray) -> int:
        x = self.x
        rows = local_rows(whole, self.nx, self.ny, self.stype, x.r0 - x.h0, x.r1 + x.h1)
        return self.lib.upload(self.task, rows.astype(self.lib.dtype, copy=False))

    def _exchange(self):
        stream = self.torch.cuda.current_stream().cuda_stream
        lib, t = self.lib, self.task

        def get_rows(row0, n, buf):
            assert lib.rows_out(t, row0, n, buf.data_ptr(), stream) == 0

        def put_rows(row0, n, buf):
            assert lib.rows_in(t, row0, n, buf.data_ptr(), stream) == 0

        self.x.exchange(get_rows, put_rows)

    def step_n(self, nsteps: int) -> int:
        """nsteps steps of the whole grid: at most two per exchange."""
        left = nsteps
        while left > 0:
            k = min(2, left)
            rc = self.lib.step_n(self.task, k)
            if rc:
                return rc
            if self.x.world > 1:
                self._exchange()
            left -= k
        return 0

    def owned(self) -> np.ndarray:
        """This rank's owned rows (task layout) of the current state."""
        x = self.x
        g = np.zeros(5 * self.nx * x.nyl, self.lib.dtype)
        assert self.lib.download(self.task, g) == 0
        return local_rows(g, self.nx, x.nyl, self.stype, x.h0, x.h0 + x.own)

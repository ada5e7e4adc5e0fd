"""Seeded synthetic solve problems for le2d's step (no dataset is involved).

A problem is the input of one forward-modelling solve: grid size, spacing,
material, time step, step count, pressure disks applied in order with
``le_set_ball`` semantics (le2d ``simple/le_core.c:71-94``: sxx = syy = s inside
the open disk, overwrite) and optional uniform noise on vx and vy.

The generators below define the five workloads this project is measured on:
the plain 512x512 case, the 8192x8192 single solve, the 4096x4096 precision study,
the 256-instance uneven batch and the Poisson serving stream.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Tuple

import numpy as np


@dataclasses.dataclass
class Problem:
    nx: int
    ny: int
    hx: float
    hy: float
    c1: float
    c2: float
    rho: float
    dt: float
    steps: int
    disks: List[Tuple[float, float, float, float]]  # (cx, cy, r, s) in grid units
    noise: float = 0.0  # amplitude of uniform noise added to vx and vy
    seed: int = 0

    @property
    def nodes(self) -> int:
        return self.nx * self.ny

    @property
    def node_updates(self) -> int:
        return self.nx * self.ny * self.steps

    def noise_fields(self, dtype) -> Tuple[np.ndarray, np.ndarray] | None:
        """(vx, vy) noise planes of shape (ny, nx) in the given dtype, or None."""
        if self.noise <= 0.0:
            return None
        rng = np.random.default_rng(self.seed + 7919)
        vx = rng.uniform(-self.noise, self.noise, size=(self.ny, self.nx)).astype(dtype)
        vy = rng.uniform(-self.noise, self.noise, size=(self.ny, self.nx)).astype(dtype)
        return vx, vy


def _seeded_disks(rng, nx, ny, count, rmin, rmax, amin, amax):
    disks = []
    for _ in range(count):
        cx = float(rng.uniform(0.1 * (nx - 1), 0.9 * (nx - 1)))
        cy = float(rng.uniform(0.1 * (ny - 1), 0.9 * (ny - 1)))
        r = float(rng.uniform(rmin, rmax))
        a = float(rng.uniform(amin, amax)) * (1.0 if rng.uniform() < 0.5 else -1.0)
        disks.append((cx, cy, r, a))
    return disks


def plain_512(steps: int = 200) -> Problem:
    """512x512, h=1, c1=2, c2=1, rho=1, dt=0.5*h/c1, one disk r=25 at the centre, s=1."""
    return Problem(512, 512, 1.0, 1.0, 2.0, 1.0, 1.0, 0.5 * 1.0 / 2.0, steps,
                   [(256.0, 256.0, 25.0, 1.0)])


def single_8192(steps: int = 1000, seed: int = 2, n: int = 8192) -> Problem:
    """8192x8192, c1=3, c2=1.7, rho=2.5, dt=0.5*h/c1, 8 seeded disks r in [20,200], |s| in [0.5,2]."""
    rng = np.random.default_rng(seed)
    disks = _seeded_disks(rng, n, n, 8, 20.0, 200.0, 0.5, 2.0)
    return Problem(n, n, 1.0, 1.0, 3.0, 1.7, 2.5, 0.5 / 3.0, steps, disks, 0.0, seed)


def precision_4096(steps: int = 4000, seed: int = 3, n: int = 4096) -> Problem:
    """4096x4096, c1=2, c2=1, rho=1, disks as the 8192 case plus U(+-1e-3) noise on vx, vy."""
    rng = np.random.default_rng(seed)
    disks = _seeded_disks(rng, n, n, 8, 20.0, 200.0, 0.5, 2.0)
    return Problem(n, n, 1.0, 1.0, 2.0, 1.0, 1.0, 0.5 / 2.0, steps, disks, 1e-3, seed)


def random_instance(rng, side_lo: int, side_hi: int, steps_lo: int, steps_hi: int,
                    seed: int) -> Problem:
    """One instance drawn as the batched workload draws them: sides log-uniform, c1 in [1,4],
    c2/c1 in [0.3,0.6], rho in [1,3], h=1, dt=0.5*h/c1, 1-4 disks, steps uniform."""
    nx = int(round(math.exp(rng.uniform(math.log(side_lo), math.log(side_hi)))))
    ny = int(round(math.exp(rng.uniform(math.log(side_lo), math.log(side_hi)))))
    c1 = float(rng.uniform(1.0, 4.0))
    c2 = c1 * float(rng.uniform(0.3, 0.6))
    rho = float(rng.uniform(1.0, 3.0))
    steps = int(rng.integers(steps_lo, steps_hi + 1))
    nd = int(rng.integers(1, 5))
    rmax = max(2.0, min(200.0, 0.25 * min(nx, ny)))
    rmin = min(20.0, 0.5 * rmax)
    disks = _seeded_disks(rng, nx, ny, nd, rmin, rmax, 0.5, 2.0)
    return Problem(nx, ny, 1.0, 1.0, c1, c2, rho, 0.5 / c1, steps, disks, 0.0, seed)


def batched_256(count: int = 256, seed: int = 4, side_lo: int = 128, side_hi: int = 2048,
                steps_lo: int = 200, steps_hi: int = 2000) -> List[Problem]:
    """The uneven batch: 256 independent FP32 solves."""
    rng = np.random.default_rng(seed)
    return [random_instance(rng, side_lo, side_hi, steps_lo, steps_hi, seed * 100003 + k)
            for k in range(count)]


@dataclasses.dataclass
class Request:
    arrival_s: float
    problem: Problem
    want: str  # "fields" or "receivers"


def serving_stream(rate: float, count: int, seed: int = 5, side_lo: int = 64,
                   side_hi: int = 4096, steps_lo: int = 100, steps_hi: int = 5000,
                   receivers_fraction: float = 0.5) -> List[Request]:
    """Poisson arrivals at `rate` per second; instances drawn as the batched workload."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(count):
        t += float(rng.exponential(1.0 / rate))
        p = random_instance(rng, side_lo, side_hi, steps_lo, steps_hi, seed * 1000003 + k)
        want = "receivers" if rng.uniform() < receivers_fraction else "fields"
        out.append(Request(t, p, want))
    return out

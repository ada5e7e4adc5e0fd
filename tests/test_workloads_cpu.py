"""The seeded synthetic workloads (le2d_b200/workloads.py) that bench.py and the GPU tests
run stand in for the benchmark configurations: the minimum slice (512^2, one disk, 200
steps), the 8192^2 single solve, the 4096^2 precision run, the 256-instance batched mix and
the Poisson serving stream.  Their shapes, parameters and value ranges are those configs',
and they are the same on every call (seeded)."""
import numpy as np

from le2d_b200 import workloads


def test_plain_512_is_the_minimum_slice():
    p = workloads.plain_512()
    assert (p.nx, p.ny, p.steps) == (512, 512, 200)
    assert (p.hx, p.hy, p.c1, p.c2, p.rho) == (1.0, 1.0, 2.0, 1.0, 1.0)
    assert p.dt == 0.5 * 1.0 / 2.0  # k1 = 0.5, k2 = 0.25
    assert p.disks == [(256.0, 256.0, 25.0, 1.0)]
    assert p.node_updates == 512 * 512 * 200


def _check_disks(p, count, rmin, rmax):
    assert len(p.disks) == count
    for cx, cy, r, s in p.disks:
        assert 0.1 * (p.nx - 1) <= cx <= 0.9 * (p.nx - 1) and 0.1 * (p.ny - 1) <= cy <= 0.9 * (p.ny - 1)
        assert rmin <= r <= rmax and 0.5 <= abs(s) <= 2.0


def test_single_8192_config():
    p = workloads.single_8192()
    assert (p.nx, p.ny, p.steps) == (8192, 8192, 1000)
    assert (p.c1, p.c2, p.rho) == (3.0, 1.7, 2.5) and p.dt == 0.5 / 3.0
    assert p.node_updates == 8192 * 8192 * 1000  # 6.71e10
    _check_disks(p, 8, 20.0, 200.0)
    assert p.disks == workloads.single_8192().disks  # seeded


def test_precision_4096_config():
    p = workloads.precision_4096()
    assert (p.nx, p.ny, p.steps) == (4096, 4096, 4000)
    assert (p.c1, p.c2, p.rho, p.dt) == (2.0, 1.0, 1.0, 0.25)
    _check_disks(p, 8, 20.0, 200.0)
    vx, vy = p.noise_fields(np.float64)
    assert vx.shape == (4096, 4096) and np.abs(vx).max() <= 1e-3 and np.abs(vy).max() <= 1e-3
    vx2, _ = p.noise_fields(np.float64)
    assert np.array_equal(vx, vx2)


def test_batched_256_mix():
    probs = workloads.batched_256()
    assert len(probs) == 256
    for p in probs:
        assert 128 <= p.nx <= 2048 and 128 <= p.ny <= 2048
        assert 1.0 <= p.c1 <= 4.0 and 0.3 <= p.c2 / p.c1 <= 0.6 and 1.0 <= p.rho <= 3.0
        assert p.dt == 0.5 / p.c1 and 200 <= p.steps <= 2000 and 1 <= len(p.disks) <= 4
    nu = sum(p.node_updates for p in probs)
    assert 1.0e11 < nu < 2.0e11  # about 1.4e11 node-updates in all
    # sides log-uniform: about as many below the geometric middle (512) as above it
    below = sum(p.nx < 512 for p in probs)
    assert 96 <= below <= 160
    again = workloads.batched_256()
    assert [(p.nx, p.ny, p.steps, p.disks) for p in again] == [(p.nx, p.ny, p.steps, p.disks) for p in probs]


def test_serving_stream():
    reqs = workloads.serving_stream(200.0, 48, seed=205)
    t = [r.arrival_s for r in reqs]
    assert len(reqs) == 48 and all(b > a for a, b in zip(t, t[1:]))
    assert 0.05 < t[-1] < 1.0  # 48 Poisson arrivals at 200 per second take about 0.24 s
    for r in reqs:
        assert 64 <= r.problem.nx <= 4096 and 64 <= r.problem.ny <= 4096 and 100 <= r.problem.steps <= 5000
        assert r.want in ("fields", "receivers")
    assert {r.want for r in reqs} == {"fields", "receivers"}
    assert [r.arrival_s for r in workloads.serving_stream(200.0, 48, seed=205)] == t

"""Batched solves (le2d_batch_*) through the C ABI.

The persistent batched kernel marches every tile with the same per-node operations
as the single-solve kernel, so each instance's result must equal, bit for bit, the
same instance solved alone with le_step; the single-solve path is itself checked
against the reference (test_parity_gpu.py), and instances are also checked against the
oracle and the reference here (FP32 <= 1e-5 relative L2 per field; FP64 <= 1e-12, and
equal value for value on the instances drawn from the uneven mix).
"""
import os

import numpy as np
import pytest

from le2d_b200 import capi, workloads
from oracle.oracle import ST_AOS, ST_SOA, Oracle, fields, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def libs():
    return {p: capi.Lib(p) for p in ("f", "d")}


def solve_alone(lib, p: workloads.Problem, stype, init=None, sample_row=-1, every=10):
    """The instance through the single-solve API; optionally samples (vx, vy) of one row."""
    mat = lib.le_init_material(p.c1, p.c2, p.rho)
    t = lib.le_init_task(p.dt, (p.hx, p.hy), mat, (p.nx, p.ny), stype)
    samples = []
    try:
        if init is not None:
            assert lib.upload(t, init) == 0
        else:
            for cx, cy, r, s in p.disks:
                lib.le_set_ball(t, (cx, cy), r, s)
        step = lib.le_step if stype == ST_AOS else lib.le_step_soa
        for k in range(p.steps):
            step(t)
            if sample_row >= 0 and (k + 1) % every == 0:
                g = np.zeros(5 * p.nx * p.ny, lib.dtype)
                assert lib.download(t, g) == 0
                f = fields(g, p.nx, p.ny, stype)
                samples.append(np.stack([f[0, sample_row], f[1, sample_row]]))
        out = np.zeros(5 * p.nx * p.ny, lib.dtype)
        assert lib.download(t, out) == 0
        assert lib.last_error(t) == 0
        return out, (np.stack(samples) if samples else None)
    finally:
        lib.le_free_task(t)


def small_set(seed, count, lo=5, hi=300, steps_lo=5, steps_hi=90):
    rng = np.random.default_rng(seed)
    return [workloads.random_instance(rng, lo, hi, steps_lo, steps_hi, seed * 1000 + k) for k in range(count)]


@pytest.mark.parametrize("prec", ["f", "d"])
def test_batch_equals_single_solves(libs, prec):
    lib = libs[prec]
    probs = small_set(21, 14)
    stypes = [ST_AOS if k % 3 else ST_SOA for k in range(len(probs))]
    with capi.Batch(lib, 1 << 30) as b:
        ids = [b.add(b.problem(p, st), disks=p.disks) for p, st in zip(probs, stypes)]
        assert all(i >= 0 for i in ids), ids
        rc, ms = b.run(window_steps=32)  # several windows, instances finishing at different times
        assert rc == 0, lib.strerror(rc)
        for i, p, st in zip(ids, probs, stypes):
            got = b.fields(i)
            want, _ = solve_alone(lib, p, st)
            assert got.tobytes() == want.tobytes(), (i, p.nx, p.ny, p.steps, st)


@pytest.mark.parametrize("prec", ["f", "d"])
def test_batch_against_oracle(libs, prec):
    lib = libs[prec]
    tol = 1e-5 if prec == "f" else 1e-12
    probs = small_set(22, 4, 40, 200, 20, 60)
    with capi.Batch(lib, 1 << 30) as b:
        ids = [b.add(b.problem(p), disks=p.disks) for p in probs]
        assert b.run(window_steps=1000)[0] == 0
        for i, p in zip(ids, probs):
            got = fields(b.fields(i), p.nx, p.ny, ST_AOS)
            o = Oracle(prec)
            g = np.zeros(5 * p.nx * p.ny, o.dtype)
            for d in p.disks:
                o.set_ball(g, p.nx, p.ny, p.hx, p.hy, ST_AOS, *d)
            o.run(g, p.nx, p.ny, p.dt, p.hx, p.hy, p.c1, p.c2, p.rho, ST_AOS, p.steps)
            err = rel_l2(got, fields(g, p.nx, p.ny, ST_AOS))
            assert np.all(err <= tol), (i, err)


@pytest.mark.parametrize("prec", ["f", "d"])
def test_batch_mix_subset_against_reference(libs, prec):
    """16 instances drawn (seeded) from the 256-instance uneven mix itself -- sizes, materials,
    disks and step counts as generated, among the instances of at most 5e7 node-updates so
    the CPU side stays short -- in one batched run (default tiles), against the reference
    solver run on the host (oracle/_ref: the reference's own simple/ build, OpenMP; else the
    C oracle, which reproduces it bit for bit).  FP64: equal value for value.  FP32: within
    1e-5 per field of the reference float and double builds, or 4x the float build's own
    distance from its double build where that is larger (small boxes with many reflections)."""
    from oracle.oracle import Reference
    from test_parity_gpu import check

    lib = libs[prec]
    mix = workloads.batched_256()
    small = [k for k, p in enumerate(mix) if p.node_updates <= 5e7]
    pick = sorted(np.random.default_rng(16).choice(small, size=min(16, len(small)), replace=False))
    threads = os.cpu_count() or 1
    lib.batch_autotune_reset()
    with capi.Batch(lib, 1 << 32) as b:
        ids = [b.add(b.problem(mix[k]), disks=mix[k].disks) for k in pick]
        assert b.run(window_steps=256)[0] == 0
        for i, k in zip(ids, pick):
            p = mix[k]
            got = b.fields(i)
            want = {}
            for q in ("f", "d") if prec == "f" else ("d",):
                o = Oracle(q)
                g = np.zeros(5 * p.nx * p.ny, o.dtype)
                for d in p.disks:
                    o.set_ball(g, p.nx, p.ny, p.hx, p.hy, ST_AOS, *d)
                if Reference.available(q):
                    Reference(q).run(g, p.nx, p.ny, p.dt, p.hx, p.hy, p.c1, p.c2, p.rho, ST_AOS, p.steps, threads)
                else:
                    o.run(g, p.nx, p.ny, p.dt, p.hx, p.hy, p.c1, p.c2, p.rho, ST_AOS, p.steps)
                want[q] = g
            if prec == "d":
                assert np.array_equal(got, want["d"]), (k, p.nx, p.ny, p.steps)
            else:
                check("f", got, want["f"], want["d"], p.nx, p.ny, ST_AOS,
                      f"mix[{k}] {p.nx}x{p.ny} x{p.steps}")


def test_batch_init_arrays_and_receivers(libs):
    lib = libs["f"]
    rng = np.random.default_rng(5)
    probs = small_set(23, 3, 30, 150, 30, 45)
    with capi.Batch(lib, 1 << 30) as b:
        inits, ids = [], []
        for p in probs:
            g = rng.uniform(-0.1, 0.1, 5 * p.nx * p.ny).astype(np.float32)
            inits.append(g)
            ids.append(b.add(b.problem(p, ST_AOS, receiver_row=p.ny // 4, receiver_every=10), init=g))
        assert b.run(window_steps=16)[0] == 0
        for i, p, g in zip(ids, probs, inits):
            want, samples = solve_alone(lib, p, ST_AOS, init=g, sample_row=p.ny // 4, every=10)
            assert b.fields(i).tobytes() == want.tobytes()
            rec = b.receivers(i)
            assert rec.shape == (p.steps // 10, 2, p.nx)
            assert rec.tobytes() == samples.astype(np.float32).tobytes()


def test_batch_diagnostics(libs):
    lib = libs["d"]
    p = small_set(24, 1, 60, 80, 10, 10)[0]
    with capi.Batch(lib, 1 << 28) as b:
        i = b.add(b.problem(p), disks=p.disks)
        assert b.run()[0] == 0
        rc, d = b.diagnostics(i)
        assert rc == 0
        g = b.fields(i)
        want = Oracle("d").diag(g, p.nx, p.ny, p.hx, p.hy, p.c1, p.c2, p.rho, ST_AOS)
        assert abs(d["energy"] - want[0]) <= 1e-12 * abs(want[0])


def test_batch_budget_and_validation(libs):
    lib = libs["f"]
    with capi.Batch(lib, 4 << 20) as b:  # 4 MiB of states
        ok = b.problem(workloads.Problem(100, 100, 1, 1, 2, 1, 1, 0.25, 5, []))
        assert b.add(ok) >= 0
        big = b.problem(workloads.Problem(1000, 1000, 1, 1, 2, 1, 1, 0.25, 5, []))
        assert b.add(big) == -capi.LE2D_EBUDGET
        bad = b.problem(workloads.Problem(2, 100, 1, 1, 2, 1, 1, 0.25, 5, []))
        assert b.add(bad) == -capi.LE2D_EINVAL
        cfl = b.problem(workloads.Problem(50, 50, 1, 1, 2, 1, 1, 0.75, 5, []))  # k1 = 1.5
        assert b.add(cfl) == -capi.LE2D_EINVAL
        assert b.run()[0] == 0


@pytest.mark.parametrize("prec", ["f", "d"])
def test_batch_bounded_wait_gives_up(libs, prec, monkeypatch):
    """A tile that never publishes its first step (test hook, first tile of the first
    window): the waits that depend on it run out after the wait limit and its instance
    fails alone -- le2d_batch_run reports LE2D_ETIMEOUT, the instance's results report
    LE2D_ETIMEOUT, the other instances' results equal their solves alone, and the device
    stays usable."""
    lib = libs[prec]
    victim = workloads.Problem(300, 200, 1, 1, 2, 1, 1, 0.25, 6, [(150.0, 100.0, 30.0, 1.0)])
    others = small_set(41, 3, 20, 200, 2, 5)  # fewer steps: ordered after the victim
    monkeypatch.setenv("LE2D_TEST_STALL_TILE", "0")
    with capi.Batch(lib, 1 << 28) as b:
        assert b.set_wait_limit(50_000_000) == 0  # 50 ms
        iv = b.add(b.problem(victim), disks=victim.disks)
        ids = [b.add(b.problem(p), disks=p.disks) for p in others]
        rc, _ = b.run(window_steps=6)
        assert rc == capi.LE2D_ETIMEOUT
        out = np.zeros(5 * victim.nx * victim.ny, lib.dtype)
        assert lib.lib.le2d_batch_fields(b.h, iv, out.ctypes.data) == capi.LE2D_ETIMEOUT
        for i, p in zip(ids, others):
            want, _ = solve_alone(lib, p, ST_AOS)
            assert b.fields(i).tobytes() == want.tobytes()
    monkeypatch.delenv("LE2D_TEST_STALL_TILE")
    with capi.Batch(lib, 1 << 28) as b:  # a normal run afterwards
        i = b.add(b.problem(victim), disks=victim.disks)
        assert b.run()[0] == 0
        want, _ = solve_alone(lib, victim, ST_AOS)
        assert b.fields(i).tobytes() == want.tobytes()


@pytest.mark.parametrize("prec", ["f", "d"])
def test_batch_odd_windows_and_receivers(libs, prec):
    """Odd window lengths (a two-step instance then ends a window with a one-step item) and
    samples every 3 steps (taken after the first step of a two-step item on the producer
    warp, after the second on the consumer, and after one-step items): fields and receiver
    lines bitwise equal to the instances solved alone."""
    lib = libs[prec]
    rng = np.random.default_rng(9)
    probs = small_set(24, 4, 20, 260, 17, 41)
    stypes = [ST_AOS, ST_AOS, ST_SOA, ST_AOS]
    with capi.Batch(lib, 1 << 30) as b:
        inits, ids = [], []
        for p, st in zip(probs, stypes):
            g = rng.uniform(-0.1, 0.1, 5 * p.nx * p.ny).astype(lib.dtype)
            inits.append(g)
            ids.append(b.add(b.problem(p, st, receiver_row=p.ny // 3, receiver_every=3), init=g))
        assert b.run(window_steps=7)[0] == 0
        for i, p, st, g in zip(ids, probs, stypes, inits):
            want, samples = solve_alone(lib, p, st, init=g, sample_row=p.ny // 3, every=3)
            assert b.fields(i).tobytes() == want.tobytes(), (i, st)
            rec = b.receivers(i)
            assert rec.shape == (p.steps // 3, 2, p.nx)
            assert rec.tobytes() == samples.astype(lib.dtype).tobytes(), (i, st)


def test_cli_batch_subcommand(capsys):
    """`python -m le2d_b200.cli batch n steps` (the driver the batched kernel's profile is
    taken with) runs the first n instances of the mix through the batched path."""
    from le2d_b200 import cli

    assert cli.main(["batch", "3", "6", "--window", "4"]) == 0
    out = capsys.readouterr().out.split()
    assert out[:4] == ["3", "instances", "6", "steps"] and float(out[-2]) > 0

"""The per-size-class autotuner (le2d_autotune): picks a compiled fused-kernel variant
and row-segment length, new tasks of the size class use it, and results do not depend
on the plan (every variant computes the same per-node operations)."""
import numpy as np
import pytest

from le2d_b200 import capi, workloads

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["f", "d"])
def test_autotune_applies_to_size_class(prec):
    lib = capi.Lib(prec)
    p = workloads.Problem(nx=300, ny=220, hx=1.0, hy=1.0, c1=2.0, c2=1.0, rho=1.0, dt=0.25, steps=40,
                          disks=[(150.0, 110.0, 30.0, 1.0)])

    def run():
        mat = lib.le_init_material(p.c1, p.c2, p.rho)
        t = lib.le_init_task(p.dt, (p.hx, p.hy), mat, (p.nx, p.ny), capi.ST_AOS)
        try:
            for d in p.disks:
                lib.le_set_ball(t, d[:2], d[2], d[3])
            assert lib.step_n(t, p.steps) == 0
            assert lib.sync_host(t) == 0
            return lib.get_plan(t), lib.grid_view(t).copy()
        finally:
            lib.le_free_task(t)

    lib.autotune_reset()
    plan0, out0 = run()
    tuned, nus = lib.autotune(p.nx, p.ny)
    assert nus > 0 and tuned["variant"] >= 0 and tuned["depth"] in (1, 2)
    plan1, out1 = run()  # same size class: 300 -> 512, 220 -> 256
    assert plan1["variant"] == tuned["variant"] and plan1["seg_len"] == tuned["seg_len"]
    assert plan1["depth"] == tuned["depth"]
    assert out0.tobytes() == out1.tobytes()
    lib.autotune_reset()
    plan2, _ = run()
    assert plan2 == plan0


def test_batch_autotune_size_class():
    """The batched-path autotuner picks a tile height and steps per work item for a size
    class; batches of that class use it, and results stay those of a single solve."""
    lib = capi.Lib("f")
    lib.batch_autotune_reset()
    plan, nus = lib.batch_autotune(300, 220)
    assert nus > 0 and plan["seg_len"] in (16, 32, 64, 128, 256) and plan["depth"] in (1, 2)
    p = workloads.Problem(nx=300, ny=220, hx=1.0, hy=1.0, c1=2.0, c2=1.0, rho=1.0, dt=0.25, steps=41,
                          disks=[(150.0, 110.0, 30.0, 1.0)])
    with capi.Batch(lib, 1 << 28) as b:
        i = b.add(b.problem(p), disks=p.disks)
        assert b.run()[0] == 0
        got = b.fields(i)
    mat = lib.le_init_material(p.c1, p.c2, p.rho)
    t = lib.le_init_task(p.dt, (p.hx, p.hy), mat, (p.nx, p.ny), capi.ST_AOS)
    try:
        for d in p.disks:
            lib.le_set_ball(t, d[:2], d[2], d[3])
        for _ in range(p.steps):
            lib.le_step(t)
        assert lib.sync_host(t) == 0
        want = lib.grid_view(t).copy()
    finally:
        lib.le_free_task(t)
    assert got.tobytes() == want.tobytes()
    lib.batch_autotune_reset()

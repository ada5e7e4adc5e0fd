"""Command-line solve through the C ABI, after the reference's driver (le2d simple/main.c).

    python -m le2d_b200.cli nx ny steps [--prec f|d] [--method fused|split]
                            [--workload plain|disks] [--save out.vtk]
                            [--variant K --seg ROWS] [--per-call]

Like simple/main.c:18-80: init material and task, set the initial condition, run
`steps` calls of le_step, print "nx ny steps seconds" (simple/main.c:68) and
optionally save the VTK.  The default initial condition is the reference driver's
(c1=2, c2=1, rho=1.5, dt=0.3, one disk r=10 at the centre, s=1); --workload disks
uses the seeded 8-disk material of the 8192x8192 workload scaled to the grid.
--variant / --seg pick a compiled fused-kernel variant and row-segment length
(le2d_set_variant) and print the plan, e.g. to profile one kernel variant.

    python -m le2d_b200.cli batch n steps [--window W] [--tune]

runs the first n instances of the seeded 256-instance mix (bench.py's batched workload:
sides 128-2048, their own materials and disks), `steps` steps each, through the batched
path (le2d_batch_*, windows of W steps; --tune: the batched autotuner's tiles per size
class, else the default tiles) and prints the launch rate, e.g. to profile the batched
kernel on a small case.
"""
from __future__ import annotations

import argparse
import sys
import time

from le2d_b200 import capi, workloads


def main_batch(argv) -> int:
    ap = argparse.ArgumentParser(prog="cli batch")
    ap.add_argument("n", type=int, help="instances: the first n of the 256-instance mix")
    ap.add_argument("steps", type=int, help="steps of every instance")
    ap.add_argument("--window", type=int, default=256, help="steps per persistent launch")
    ap.add_argument("--tune", action="store_true", help="batched autotuner's tiles per size class")
    a = ap.parse_args(argv)
    lib = capi.Lib("f")
    probs = [workloads.Problem(**{**p.__dict__, "steps": a.steps}) for p in workloads.batched_256()[:a.n]]
    budget = int(1.1 * sum(2 * 5 * 4 * (((p.nx + 31) // 32) * 32) * p.ny + 512 for p in probs)) + (64 << 20)
    if a.tune:
        lib.batch_autotune_reset()
        for p in probs:
            lib.batch_autotune(p.nx, p.ny)
    with capi.Batch(lib, budget) as b:
        for p in probs:
            if b.add(b.problem(p), disks=p.disks) < 0:
                print("le2d_batch_add failed", file=sys.stderr)
                return 1
        rc, ms = b.run(window_steps=a.window)
    if rc != 0:
        print(f"le2d error: {lib.strerror(rc)}", file=sys.stderr)
        return 1
    nu = sum(p.nx * p.ny for p in probs) * a.steps
    print(f"{len(probs)} instances {a.steps} steps {ms:.2f} ms {nu / (ms * 1e-3):.4g} nu/s")
    return 0


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if argv and argv[0] == "batch":
        return main_batch(argv[1:])
    ap = argparse.ArgumentParser()
    ap.add_argument("nx", type=int)
    ap.add_argument("ny", type=int)
    ap.add_argument("steps", type=int)
    ap.add_argument("--prec", default="f", choices=["f", "d"])
    ap.add_argument("--method", default="fused", choices=["fused", "split"])
    ap.add_argument("--workload", default="plain", choices=["plain", "disks"])
    ap.add_argument("--save", default=None)
    ap.add_argument("--per-call", action="store_true", help="one le_step call per step (default: le2d_step_n)")
    ap.add_argument("--variant", type=int, default=None, help="fused-kernel variant (le2d_set_variant)")
    ap.add_argument("--seg", type=int, default=0, help="row-segment length with --variant (0 = planner's)")
    a = ap.parse_args(argv)
    lib = capi.Lib(a.prec)
    if a.workload == "plain":
        c1, c2, rho, dt, disks = 2.0, 1.0, 1.5, 0.3, [(float(a.nx // 2), float(a.ny // 2), 10.0, 1.0)]
    else:
        p = workloads.single_8192(steps=a.steps, n=max(a.nx, a.ny))
        c1, c2, rho, dt, disks = p.c1, p.c2, p.rho, p.dt, p.disks
    mat = lib.le_init_material(c1, c2, rho)
    t = lib.le_init_task(dt, (1.0, 1.0), mat, (a.nx, a.ny), capi.ST_AOS)
    if not t.grid:
        print("le_init_task failed", file=sys.stderr)
        return 1
    try:
        lib.set_method(t, capi.LE2D_METHOD_FUSED if a.method == "fused" else capi.LE2D_METHOD_SPLIT)
        if a.variant is not None:
            if lib.set_variant(t, a.variant, a.seg) != 0:
                print(f"no fused-kernel variant {a.variant}", file=sys.stderr)
                return 1
            print("plan", lib.get_plan(t))
        for cx, cy, r, s in disks:
            lib.le_set_ball(t, (cx, cy), r, s)
        lib.wait(t)
        t0 = time.perf_counter()
        if a.per_call:
            for _ in range(a.steps):
                lib.le_step(t)
        else:
            lib.step_n(t, a.steps)
        lib.wait(t)
        secs = time.perf_counter() - t0
        print(f"{a.nx} {a.ny} {a.steps} {secs:f} ")
        if a.save:
            lib.le_save_task(t, a.save)
        err = lib.last_error(t)
        if err:
            print(f"le2d error: {lib.strerror(err)}", file=sys.stderr)
            return 1
        return 0
    finally:
        lib.le_free_task(t)


if __name__ == "__main__":
    sys.exit(main())

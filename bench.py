"""Benchmark of le2d's time step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: the 8192x8192 single solve (c1=3, c2=1.7, rho=2.5, h=1, dt=0.5*h/c1,
8 seeded pressure disks), 1000 time steps per solve.  A bench "step" is one such
solve (6.71e10 node-updates); the metric is node-updates/s (nu/s), one
node-update = one node advanced one full time step (x- and y-sweep).

Our arm (default) prints one JSON line with
  value     nu/s with the state resident in HBM (CUDA events on the task's stream),
  e2e       nu/s through the C ABI with host buffers: upload of the initial state
            from page-locked memory, 1000 steps, download of the final fields, one solve
            after the other (pipelined_value: two tasks alternating, so one solve's copies
            overlap the other's steps),
  roofline  the fused step kernel against the measured HBM copy bandwidth,
            40 algorithmic bytes per node-update in FP32 (read + write of 5 fields);
            a launch of temporal-block depth 2 advances every node two steps, so its
            algorithmic bytes are 2 x 40 B per node while it moves about half of that;
            an update of the grid launched in halves (launch_parts 3: the band around the
            middle row and the rows above and below it, overlapping) is timed as one launch,
            and gpu_launches counts its 3 kernel launches,
  cpu_baseline  the reference's own simple/ solver (oracle/_ref) on the host cores,
  fp64      the same measurement for the FP64 library (80 B per node-update),
  batched   256 uneven FP32 solves (sides 128-2048, steps 200-2000) in the persistent
            batched kernel against the plain one-instance-at-a-time le_step loop on the
            same GPU: solves/s of both, the speed-up, and the FP32 fields of every instance
            against the FP64 library's (which equals the reference double build),
  serving   Poisson request streams (10 and 200 requests/s) through the serving loop:
            solves/s and p50/p99 latency beside a one-at-a-time plain le_step server,
  precision 4096x4096 with disks and noise, 4000 steps: FP32 against FP64 (= the reference
            double build) per field every 500 steps, and the FP64 energy drift.
Under torchrun each rank solves its own instance (independent solves, weak scaling);
value is the total node-updates of all ranks over the slowest rank's time; the batched
and serving measurements run only in the one-process case.

--impl reference: the reference's own CPU solver (simple/ le_step, OpenMP over all
host threads) on a bounded sample of the same workload (one time step per bench
step); rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from le2d_b200 import capi, workloads  # noqa: E402

BYTES_PER_NU = {"f": 40, "d": 80}
SMI_FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per launch of the fused kernel from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as fh:
            return json.load(fh)
    return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={SMI_FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        if self.path and os.path.exists(self.path):
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def dist_init(world, local, backend):
    if world <= 1:
        return None
    import datetime

    import torch
    import torch.distributed as dist

    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
    return dist


def dist_max(dist, x: float, backend: str) -> float:
    if dist is None:
        return x
    import torch

    dev = f"cuda:{torch.cuda.current_device()}" if backend == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(dist):
    if dist is not None:
        dist.barrier()


def new_task(lib, p: workloads.Problem):
    mat = lib.le_init_material(p.c1, p.c2, p.rho)
    t = lib.le_init_task(p.dt, (p.hx, p.hy), mat, (p.nx, p.ny), capi.ST_AOS)
    if not t.grid or lib.last_error(t):
        raise RuntimeError(f"le_init_task failed: {lib.strerror(lib.last_error(t))}")
    return t


def initial_state(lib, p, t) -> np.ndarray:
    """The workload's initial state (disks through le_set_ball) as a page-locked host copy."""
    for cx, cy, r, s in p.disks:
        lib.le_set_ball(t, (cx, cy), r, s)
    assert lib.sync_host(t) == 0
    return lib.grid_view(t)  # task->grid is page-locked


def measure_ours(lib, prec, p, steps, warmup, dist, backend, device):
    """Device-resident timing of `steps` solves and end-to-end timing through the C ABI."""
    t = new_task(lib, p)
    e2e_t = new_task(lib, p)
    e2e_u = new_task(lib, p)
    host_out, free_out = lib.host_array(5 * p.nodes)  # page-locked result buffers
    host_out2, free_out2 = lib.host_array(5 * p.nodes)
    try:
        ic = initial_state(lib, p, t).copy()
        for tk in (e2e_t, e2e_u):
            lib.grid_view(tk)[:] = ic  # page-locked input buffer (task->grid)
        n = p.steps
        # --- device-resident: K solves of n steps, state in HBM ---
        for _ in range(warmup):
            assert lib.upload(t, ic) == 0
            rc, _ = lib.step_n_timed(t, n)
            assert rc == 0, lib.strerror(rc)
        assert lib.upload(t, ic) == 0 and lib.wait(t) == 0
        dist_barrier(dist)
        total_ms = 0.0
        with ClockSampler(device) as clk:
            for _ in range(steps):
                rc, ms = lib.step_n_timed(t, n)  # events on the launching stream, synchronised
                assert rc == 0, lib.strerror(rc)
                total_ms += ms
        dist_barrier(dist)
        clocks = clk.summary()
        slow_ms = dist_max(dist, total_ms, backend)
        # --- end to end: upload from page-locked host memory, n steps, download ---
        for _ in range(max(1, warmup // 2)):
            assert lib.sync_device(e2e_t) == 0
            assert lib.step_n(e2e_t, n) == 0 and lib.download(e2e_t, host_out) == 0
        dist_barrier(dist)
        t0 = time.perf_counter()
        for _ in range(steps):
            assert lib.sync_device(e2e_t) == 0       # H2D of task->grid (the initial state)
            assert lib.step_n(e2e_t, n) == 0         # n time steps
            assert lib.download(e2e_t, host_out) == 0  # D2H of the final fields, synchronised
        e2e_s = time.perf_counter() - t0
        dist_barrier(dist)
        e2e_serial = dist_max(dist, e2e_s, backend)
        assert np.isfinite(host_out).all()
        # --- end to end, two tasks alternating: solve k's upload and steps are queued before
        # solve k-1's result is read back, so the copies overlap the other solve's steps
        # (the same calls and bytes per solve; the copy engines are idle during steps) ---
        pair, outs = (e2e_t, e2e_u), (host_out, host_out2)
        dist_barrier(dist)
        t0 = time.perf_counter()
        for k in range(steps):
            tk = pair[k % 2]
            assert lib.sync_device(tk) == 0          # H2D of task->grid (the initial state)
            assert lib.step_n(tk, n) == 0            # n time steps
            if k > 0:                                # D2H of the previous solve's fields
                assert lib.download(pair[(k - 1) % 2], outs[(k - 1) % 2]) == 0
        assert lib.download(pair[(steps - 1) % 2], outs[(steps - 1) % 2]) == 0
        e2e_s = time.perf_counter() - t0
        dist_barrier(dist)
        e2e_slow = dist_max(dist, e2e_s, backend)
        assert np.isfinite(host_out2 if steps > 1 else host_out).all()
        return slow_ms, clocks, e2e_slow, e2e_serial, ic, {**lib.get_plan(t), "launch_parts": lib.launch_parts(t)}
    finally:
        lib.le_free_task(t)
        lib.le_free_task(e2e_t)
        lib.le_free_task(e2e_u)
        free_out()
        free_out2()


def cpu_reference_sample(p, budget_s=12.0):
    """The reference simple/ solver (oracle/_ref) or, if absent, the C oracle port, timed on
    all host threads over a bounded number of time steps of the same workload."""
    sys.path.insert(0, ROOT)
    from oracle.oracle import ST_AOS, Oracle, Reference, ReferencePthread

    threads = os.cpu_count() or 1
    g = np.zeros(5 * p.nx * p.ny, np.float32)
    o = Oracle("f")
    for cx, cy, r, s in p.disks:
        o.set_ball(g, p.nx, p.ny, p.hx, p.hy, ST_AOS, cx, cy, r, s)
    out = {}
    if Reference.available("f"):
        ref = Reference("f")
        t1 = ref.run(g.copy(), p.nx, p.ny, p.dt, p.hx, p.hy, p.c1, p.c2, p.rho, ST_AOS, 1, threads)
        k = max(1, min(20, int(budget_s / max(t1, 1e-3))))
        tk = ref.run(g.copy(), p.nx, p.ny, p.dt, p.hx, p.hy, p.c1, p.c2, p.rho, ST_AOS, k, threads)
        out["simple"] = {"value": p.nx * p.ny * k / tk, "unit": "node-updates/s", "cores": threads,
                         "kind": "reference",
                         "sample": f"reference simple/ le_step (gcc -O2 -fno-tree-vectorize, OpenMP), "
                                   f"FP32, {p.nx}x{p.ny}, {k} time steps"}
        if ReferencePthread.available("f"):
            pt = ReferencePthread("f")
            thr = max(1, min(threads, p.ny // 8))
            t1 = pt.run(None, p.nx, p.ny, p.dt, p.hx, p.hy, p.c1, p.c2, p.rho, 1, thr)
            k = max(1, min(20, int(budget_s / max(t1, 1e-3))))
            tk = pt.run(g.copy(), p.nx, p.ny, p.dt, p.hx, p.hy, p.c1, p.c2, p.rho, k, thr)
            out["pthread"] = {"value": p.nx * p.ny * k / tk, "unit": "node-updates/s", "cores": thr,
                              "kind": "reference",
                              "sample": f"reference pthread/ le_step (speed only), FP32, {p.nx}x{p.ny}, {k} steps"}
    else:
        t0 = time.perf_counter()
        o.run(g, p.nx, p.ny, p.dt, p.hx, p.hy, p.c1, p.c2, p.rho, ST_AOS, 1)
        t1 = time.perf_counter() - t0
        out["simple"] = {"value": p.nx * p.ny / t1, "unit": "node-updates/s", "cores": 1, "kind": "port",
                         "sample": f"C oracle port (single thread), FP32, {p.nx}x{p.ny}, 1 time step"}
    return out


def single_config(p, parallelism: str) -> dict:
    """The `config` of the single-solve workload (both arms)."""
    return {"workload": f"single_8192: {p.nx}x{p.ny} grid, c1={p.c1}, c2={p.c2}, rho={p.rho}, "
                        f"dt=0.5*h/c1, 8 seeded disks; one bench step = one solve of {p.steps} time steps",
            "nx": p.nx, "ny": p.ny, "time_steps_per_solve": p.steps,
            "l2": "state 1.34 GB (> 126 MB L2), no flush", "parallelism": parallelism}


def run_reference_arm(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    from oracle.oracle import ST_AOS, Oracle, Reference

    p = workloads.single_8192()
    threads = os.cpu_count() or 1
    g = np.zeros(5 * p.nx * p.ny, np.float32)
    o = Oracle("f")
    for cx, cy, r, s in p.disks:
        o.set_ball(g, p.nx, p.ny, p.hx, p.hy, ST_AOS, cx, cy, r, s)
    if Reference.available("f"):
        runner = Reference("f")
        kind = "reference"
        step = lambda: runner.run(g, p.nx, p.ny, p.dt, p.hx, p.hy, p.c1, p.c2, p.rho, ST_AOS, 1, threads)
        sample = (f"reference simple/ le_step (oracle/_ref, gcc -O2 -fno-tree-vectorize, OpenMP {threads} threads), "
                  f"FP32, one time step of {p.nx}x{p.ny} per bench step")
    else:
        kind = "port"
        threads = 1

        def step():
            t0 = time.perf_counter()
            o.run(g, p.nx, p.ny, p.dt, p.hx, p.hy, p.c1, p.c2, p.rho, ST_AOS, 1)
            return time.perf_counter() - t0

        sample = f"C oracle port (single thread), FP32, one time step of {p.nx}x{p.ny} per bench step"
    for _ in range(args.warmup):
        step()
    total = 0.0
    for _ in range(args.steps):
        total += step()
    value = p.nx * p.ny * args.steps / total
    line = {
        "impl": "reference", "metric": "node-updates/s", "value": value, "unit": "node-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {**single_config(p, f"host threads x{threads}"),
                   "sample": "each bench step times one of the solve's time steps (per-step cost is constant)"},
        "cpu_baseline": {"value": value, "unit": "node-updates/s", "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": "node-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def solve_plain(lib, p, per_call=True, stype=capi.ST_AOS, timing=None):
    """One solve through the single-solve API: le_init_task, le_set_ball, le_step x steps
    (or one le2d_step_n), download of the final fields.  Returns the fields; adds the
    seconds of the step loop alone (launches until the device is idle) to timing[0]."""
    mat = lib.le_init_material(p.c1, p.c2, p.rho)
    t = lib.le_init_task(p.dt, (p.hx, p.hy), mat, (p.nx, p.ny), stype)
    try:
        for cx, cy, r, s in p.disks:
            lib.le_set_ball(t, (cx, cy), r, s)
        assert lib.wait(t) == 0
        t0 = time.perf_counter()
        if per_call:
            step = lib.le_step if stype == capi.ST_AOS else lib.le_step_soa
            for _ in range(p.steps):
                step(t)
        else:
            assert lib.step_n(t, p.steps) == 0
        assert lib.wait(t) == 0
        if timing is not None:
            timing[0] += time.perf_counter() - t0
        assert lib.sync_host(t) == 0 and lib.last_error(t) == 0
        return lib.grid_view(t).copy()
    finally:
        lib.le_free_task(t)


def batched_measure(args, accuracy="all"):
    """256 uneven FP32 solves in the persistent batched kernel (autotuned, graph-captured
    windows) against the plain one-instance-at-a-time le_step loop on the same mix.

    accuracy="all": every instance's FP32 fields against the FP64 library's (the same mix
    through the FP64 batched path; the FP64 library equals the reference double build value
    for value), per field and relative to the whole state's norm, plus the reference's own
    float-vs-double error on the worst instance (the C oracle reproduces both builds bit for
    bit).  accuracy="smallest4" (the standalone mode): also the 4 smallest instances against
    the reference float and double builds."""
    from oracle.oracle import Oracle, fields, rel_l2

    probs = workloads.batched_256()
    lib = capi.Lib("f")
    nu = sum(p.node_updates for p in probs)

    def budget_of(itemsize):
        return int(1.1 * sum(2 * 5 * itemsize * (((p.nx + 31) // 32) * 32) * p.ny + 512 for p in probs)) + (64 << 20)

    def add_all(b, scale_steps=None):
        ids = []
        for p in probs:
            q = p if scale_steps is None else workloads.Problem(**{**p.__dict__, "steps": scale_steps})
            ids.append(b.add(b.problem(q), disks=q.disks))
        assert all(i >= 0 for i in ids)
        return ids

    # batched-path autotuner: tile height and steps per work item for every size class of the
    # mix (outside the timed region; the table then applies to the instances added below)
    tuned, tune_s = {}, 0.0
    if not args.no_tune:
        lib.batch_autotune_reset()
        t0 = time.perf_counter()
        for p in probs:
            key = (max(p.nx - 1, 1).bit_length(), max(p.ny - 1, 1).bit_length())
            if key not in tuned:
                plan, nus = lib.batch_autotune(p.nx, p.ny)
                tuned[key] = {**plan, "nu_s": nus}
        tune_s = time.perf_counter() - t0
    with capi.Batch(lib, budget_of(4)) as b:  # warm-up (kernels, allocations)
        add_all(b, scale_steps=8)
        assert b.run(window_steps=args.window)[0] == 0
    bf = capi.Batch(lib, budget_of(4))
    try:
        ids = add_all(bf)
        t0 = time.perf_counter()
        rc, ms = bf.run(window_steps=args.window)
        wall = time.perf_counter() - t0
        assert rc == 0, lib.strerror(rc)
        # the plain loop: every instance alone, one le_step call per step
        loop_only = [0.0]
        t0 = time.perf_counter()
        for p in probs:
            solve_plain(lib, p, per_call=True, timing=loop_only)
        plain_s = time.perf_counter() - t0
        out = {
            "metric": "solves/s", "value": len(probs) / (ms * 1e-3), "unit": "solves/s",
            "workload": "batched_256: 256 FP32 solves, sides log-uniform 128-2048, c1 U[1,4], c2/c1 U[0.3,0.6], "
                        "rho U[1,3], dt=0.5h/c1, 1-4 disks, steps U[200,2000]",
            "node_updates": nu, "batched_device_s": ms * 1e-3, "batched_wall_s": wall,
            "batched_nu_s": nu / (ms * 1e-3), "window_steps": args.window,
            "autotune": {"seconds": tune_s, "classes": {f"2^{a}x2^{b}": v for (a, b), v in sorted(tuned.items())}},
            "plain_le_step_loop_s": plain_s, "plain_le_step_solves_s": len(probs) / plain_s,
            "plain_le_step_loop_steps_only_s": loop_only[0],
            "speedup_vs_plain_le_step": plain_s / (ms * 1e-3),
            "speedup_vs_plain_le_step_steps_only": loop_only[0] / (ms * 1e-3),
            "plain": "each instance alone through le_init_task, le_set_ball, one le_step call per step, "
                     "download of the final fields (the reference's driver loop on the GPU library)",
        }
        if accuracy == "smallest4":
            loop_only_n = [0.0]
            t0 = time.perf_counter()
            for p in probs:
                solve_plain(lib, p, per_call=False, timing=loop_only_n)
            plain_n_s = time.perf_counter() - t0
            out.update({"plain_step_n_loop_s": plain_n_s, "plain_step_n_solves_s": len(probs) / plain_n_s,
                        "plain_step_n_loop_steps_only_s": loop_only_n[0],
                        "speedup_vs_plain_step_n": plain_n_s / (ms * 1e-3)})
        # accuracy over the whole mix: FP32 against the FP64 library, instance by instance
        libd = capi.Lib("d")
        with capi.Batch(libd, budget_of(8)) as bd:
            idd = add_all(bd)
            rcd, msd = bd.run(window_steps=args.window)
            assert rcd == 0, libd.strerror(rcd)
            per_field, state_rel, worst_k = [], [], 0
            for k, p in enumerate(probs):
                ours = fields(bf.fields(ids[k]), p.nx, p.ny, 1)
                ref = fields(bd.fields(idd[k]), p.nx, p.ny, 1)
                e = rel_l2(ours, ref)
                per_field.append(e)
                d = ours.astype(np.float64) - ref
                state_rel.append(float(np.sqrt((d * d).sum() / (ref * ref).sum())))
                if e.max() > per_field[worst_k].max():
                    worst_k = k
        per_field = np.array(per_field)
        acc = {"instances": len(probs), "fp64_batched_device_s": msd * 1e-3,
               "max_rel_l2_per_field": per_field.max(axis=0).tolist(),
               "median_rel_l2_per_field": np.median(per_field, axis=0).tolist(),
               "instances_over_1e-5_any_field": int((per_field.max(axis=1) > 1e-5).sum()),
               "max_state_rel_l2": max(state_rel), "median_state_rel_l2": float(np.median(state_rel)),
               "note": "the FP64 library equals the reference double build value for value, so these are "
                       "also the errors against the reference double build"}
        # the three worst instances beside the reference's own float build on them (the
        # reference simple/ builds from oracle/_ref on all host threads; else the C oracle,
        # single-threaded, on the instances small enough for it)
        from oracle.oracle import Reference

        worst = []
        threads = os.cpu_count() or 1
        for k in np.argsort(-per_field.max(axis=1))[:3]:
            wp = probs[int(k)]
            row = {"index": int(k), "nx": wp.nx, "ny": wp.ny, "steps": wp.steps,
                   "ours_fp32_vs_fp64_rel_l2": per_field[k].tolist(),
                   "ours_fp32_vs_fp64_state_rel_l2": state_rel[k]}
            use_ref = Reference.available("f") and Reference.available("d")
            if use_ref or wp.node_updates <= 6e7:
                refs = {}
                for prec in ("f", "d"):
                    o = Oracle(prec)
                    g = np.zeros(5 * wp.nx * wp.ny, o.dtype)
                    for dd in wp.disks:
                        o.set_ball(g, wp.nx, wp.ny, wp.hx, wp.hy, 1, *dd)
                    if use_ref:
                        Reference(prec).run(g, wp.nx, wp.ny, wp.dt, wp.hx, wp.hy, wp.c1, wp.c2, wp.rho, 1,
                                            wp.steps, threads)
                    else:
                        o.run(g, wp.nx, wp.ny, wp.dt, wp.hx, wp.hy, wp.c1, wp.c2, wp.rho, 1, wp.steps)
                    refs[prec] = fields(g, wp.nx, wp.ny, 1)
                d = refs["f"].astype(np.float64) - refs["d"]
                row["reference_float_vs_double_rel_l2"] = rel_l2(refs["f"], refs["d"]).tolist()
                row["reference_float_vs_double_state_rel_l2"] = float(np.sqrt((d * d).sum() /
                                                                              (refs["d"] ** 2).sum()))
            worst.append(row)
        acc["worst_instances"] = worst
        out["accuracy_fp32_vs_fp64"] = acc
        if accuracy == "smallest4":
            rows = []
            for k in sorted(range(len(probs)), key=lambda k: probs[k].node_updates)[:4]:
                p = probs[k]
                ours = fields(bf.fields(ids[k]), p.nx, p.ny, 1)
                refs = {}
                for prec in ("f", "d"):
                    o = Oracle(prec)
                    g = np.zeros(5 * p.nx * p.ny, o.dtype)
                    for dd in p.disks:
                        o.set_ball(g, p.nx, p.ny, p.hx, p.hy, 1, *dd)
                    o.run(g, p.nx, p.ny, p.dt, p.hx, p.hy, p.c1, p.c2, p.rho, 1, p.steps)
                    refs[prec] = fields(g, p.nx, p.ny, 1)
                rows.append({"instance": k, "nx": p.nx, "ny": p.ny, "steps": p.steps,
                             "ours_fp32_vs_reference_double_rel_l2": rel_l2(ours, refs["d"]).tolist(),
                             "ours_fp32_vs_reference_float_rel_l2": rel_l2(ours, refs["f"]).tolist(),
                             "reference_float_vs_double_rel_l2": rel_l2(refs["f"], refs["d"]).tolist()})
            out["accuracy_4_smallest"] = rows
    finally:
        bf.close()
    return out


def run_batched(args):
    """256 uneven FP32 solves in the persistent batched kernel vs the plain one-at-a-time loop."""
    line = batched_measure(args, accuracy="smallest4")
    line["n_gpus"] = 1
    print(json.dumps(line), flush=True)
    return 0


def serving_measure(args, rates):
    """Poisson request streams through the serving loop vs a one-at-a-time plain le_step server."""
    import threading

    lib = capi.Lib("f")
    out = {"metric": "serving", "workload": "serving_stream: Poisson arrivals, sides log-uniform 64-4096, "
                                            "materials/disks as the batched workload, steps U[100,5000], "
                                            "half fields / half receiver lines (vx,vy at row ny/4 every 10 steps)",
           "requests_per_rate": args.requests, "window_steps": args.window, "rates": []}
    for rate in rates:
        reqs = workloads.serving_stream(rate, args.requests, seed=5 + int(rate))
        nu = sum(r.problem.node_updates for r in reqs)
        with capi.Server(lib, args.budget << 30, window_steps=args.window) as srv:
            tickets = [None] * len(reqs)

            def submitter():
                t0 = srv.now()
                for k, r in enumerate(reqs):
                    delay = t0 + r.arrival_s - srv.now()
                    if delay > 0:
                        time.sleep(delay)
                    p = r.problem
                    want = capi.LE2D_WANT_RECEIVERS if r.want == "receivers" else capi.LE2D_WANT_FIELDS
                    prob = lib.le2d_problem(p.nx, p.ny, p.hx, p.hy, p.dt, p.c1, p.c2, p.rho, p.steps, capi.ST_AOS,
                                            p.ny // 4 if want else -1, 10)
                    tickets[k] = srv.submit(prob, disks=p.disks, want=want)

            th = threading.Thread(target=submitter)
            th.start()
            th.join()
            lat, spans = [], []
            for k, t in enumerate(tickets):
                assert t > 0 and srv.wait(t, 600.0) == 0
                s_, a, c = srv.times(t)
                lat.append(c - s_)
                spans.append((a, c))
                srv.release(t)
            st = srv.stats()
        first = min(a for a, _ in spans)
        last = max(c for _, c in spans)
        joined = sum(1 for b in spans if any(a[0] < b[0] < a[1] for a in spans if a is not b))
        # one-at-a-time plain le_step server on the same stream (FIFO, no overlap)
        plat, t0 = [], time.perf_counter()
        for r in reqs:
            now = time.perf_counter() - t0
            if now < r.arrival_s:
                time.sleep(r.arrival_s - now)
            solve_plain(lib, r.problem, per_call=True)
            plat.append(time.perf_counter() - t0 - r.arrival_s)
        plain_total = time.perf_counter() - t0 - reqs[0].arrival_s
        out["rates"].append({
            "rate_per_s": rate, "solves_s": len(reqs) / (last - first), "node_updates_s": nu / (last - first),
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "plain_solves_s": len(reqs) / plain_total, "plain_p50_s": float(np.percentile(plat, 50)),
            "plain_p99_s": float(np.percentile(plat, 99)), "windows": st["windows"],
            "admitted_while_others_ran": joined,
        })
        print(json.dumps(out["rates"][-1]), file=sys.stderr, flush=True)
    out["latency"] = "submission to completion (s); plain: arrival to completion"
    return out


def run_serving(args):
    print(json.dumps(serving_measure(args, [float(r) for r in args.rates.split(",")])), flush=True)
    return 0


def run_slabs(args):
    """The 8192^2 solve split into row slabs (le2d_slabs_*) over the visible devices,
    round-robin, against the same solve as one task: node-updates/s per slab count."""
    import ctypes

    rt = ctypes.CDLL("libcudart.so")
    nd = ctypes.c_int(0)
    ndev = max(1, nd.value) if rt.cudaGetDeviceCount(ctypes.byref(nd)) == 0 else 1
    lib = capi.Lib("f")
    p = workloads.single_8192() if args.time_steps is None else workloads.single_8192(args.time_steps)
    t = new_task(lib, p)
    rows = []
    try:
        ic = initial_state(lib, p, t).copy()
        for k in [1] + [int(x) for x in args.slabs.split(",")]:
            if k == 1:
                assert lib.upload(t, ic) == 0
                rc, _ = lib.step_n_timed(t, 8)
                assert lib.upload(t, ic) == 0 and lib.wait(t) == 0
                rc, ms = lib.step_n_timed(t, p.steps)
                assert rc == 0
                sec = ms * 1e-3
                devs = [0]
            else:
                devs = [j % ndev for j in range(k)]
                with capi.Slabs(lib, t, devs) as s:
                    assert s.upload(ic) == 0
                    assert s.step_n(8) == 0 and s.wait() == 0
                    assert s.upload(ic) == 0
                    t0 = time.perf_counter()
                    assert s.step_n(p.steps) == 0 and s.wait() == 0
                    sec = time.perf_counter() - t0
            rows.append({"slabs": k, "devices": devs, "node_updates_s": p.node_updates / sec, "seconds": sec})
    finally:
        lib.le_free_task(t)
    print(json.dumps({"metric": "slabs", "workload": f"single_8192: {p.nx}x{p.ny}, {p.steps} time steps",
                      "visible_devices": ndev, "rows": rows}), flush=True)
    return 0


def run_parity(args):
    """The 8192x8192 workload at its full length (1000 steps) through the library, FP32 and
    FP64, against the reference's own simple/ float and double builds (oracle/_ref, OpenMP;
    the two builds run side by side on half the host threads each): per-field relative L2
    and max-abs, and whether the FP64 result equals the reference double build's."""
    import threading

    from oracle.oracle import ST_AOS, Oracle, Reference, fields, max_abs, rel_l2

    p = workloads.single_8192() if args.time_steps is None else workloads.single_8192(args.time_steps)
    n = p.nx
    ours, t_gpu = {}, {}
    for prec in ("f", "d"):
        lib = capi.Lib(prec)
        t = new_task(lib, p)
        try:
            initial_state(lib, p, t)
            rc, ms = lib.step_n_timed(t, p.steps)
            assert rc == 0, lib.strerror(rc)
            g = np.zeros(5 * p.nodes, lib.dtype)
            assert lib.download(t, g) == 0 and lib.last_error(t) == 0
            ours[prec], t_gpu[prec] = g, ms * 1e-3
        finally:
            lib.le_free_task(t)
    threads = os.cpu_count() or 2
    refs, secs = {}, {}
    if Reference.available("d"):
        kind = "reference simple/ (oracle/_ref, gcc -O2 -fno-tree-vectorize, OpenMP)"

        def ref_run(prec, thr):
            o = Oracle(prec)
            g = np.zeros(5 * p.nodes, o.dtype)
            for cx, cy, r, s_ in p.disks:
                o.set_ball(g, n, n, p.hx, p.hy, ST_AOS, cx, cy, r, s_)
            secs[prec] = Reference(prec).run(g, n, n, p.dt, p.hx, p.hy, p.c1, p.c2, p.rho, ST_AOS, p.steps, thr)
            refs[prec] = g

        th = [threading.Thread(target=ref_run, args=(q, max(1, threads // 2))) for q in ("f", "d")]
        for x in th:
            x.start()
        for x in th:
            x.join()
    else:
        kind = "unavailable (oracle/_ref not built)"
    line = {"metric": "parity", "workload": f"single_8192: {n}x{n}, {p.steps} time steps, 8 seeded disks",
            "gpu_seconds": t_gpu, "reference": kind, "reference_threads_each": max(1, threads // 2),
            "reference_seconds": secs}
    if refs:
        fo = {q: fields(ours[q], n, n, ST_AOS) for q in ("f", "d")}
        fr = {q: fields(refs[q], n, n, ST_AOS) for q in ("f", "d")}
        line.update({
            "fp64_equal_to_reference_double": bool(np.array_equal(ours["d"], refs["d"])),
            "fp64_vs_reference_double_rel_l2": rel_l2(fo["d"], fr["d"]).tolist(),
            "fp64_vs_reference_double_max_abs": max_abs(fo["d"], fr["d"]).tolist(),
            "fp32_vs_reference_float_rel_l2": rel_l2(fo["f"], fr["f"]).tolist(),
            "fp32_vs_reference_double_rel_l2": rel_l2(fo["f"], fr["d"]).tolist(),
            "fp32_vs_reference_double_max_abs": max_abs(fo["f"], fr["d"]).tolist(),
            "reference_float_vs_double_rel_l2": rel_l2(fr["f"], fr["d"]).tolist(),
            "tolerances": {"fp64": 1e-12, "fp32": 1e-5},
        })
        # FP32: 1e-5 per field, or -- the tests' rule -- 4x the reference float build's own
        # distance from its double build where that is larger
        gap = np.array(line["reference_float_vs_double_rel_l2"])
        tol = np.maximum(1e-5, 4.0 * gap)
        line["pass_fp64"] = bool(max(line["fp64_vs_reference_double_rel_l2"]) <= 1e-12)
        line["pass_fp32_1e-5"] = bool(max(line["fp32_vs_reference_float_rel_l2"]) <= 1e-5 and
                                      max(line["fp32_vs_reference_double_rel_l2"]) <= 1e-5)
        line["pass_fp32_with_float_build_allowance"] = bool(
            np.all(np.array(line["fp32_vs_reference_float_rel_l2"]) <= tol) and
            np.all(np.array(line["fp32_vs_reference_double_rel_l2"]) <= tol))
    print(json.dumps(line), flush=True)
    return 0


def run_dist(args):
    """The 8192x8192 solve as ONE grid split into row slabs, one rank per GPU (torchrun):
    each rank steps its slab with the library and swaps the 4 owned rows beside each cut
    with its neighbours through NCCL send/recv after every two steps (le2d_b200.dist_slabs).
    Total work is fixed (strong scaling); value = the grid's node-updates / slowest rank."""
    import torch

    from le2d_b200.dist_slabs import GpuRankSlab

    world, rank, local = dist_setup()
    dist = dist_init(world, local, "nccl")
    torch.cuda.set_device(local)
    lib = capi.Lib("f")
    assert lib.set_device(local) == 0
    p = workloads.single_8192() if args.time_steps is None else workloads.single_8192(args.time_steps)
    t = new_task(lib, p)
    try:
        ic = initial_state(lib, p, t).copy()
    finally:
        lib.le_free_task(t)
    slab = GpuRankSlab(lib, dist, rank, world, p.nx, p.ny, p.dt, (p.hx, p.hy), p.c1, p.c2, p.rho)
    try:
        assert slab.upload(ic) == 0
        for _ in range(args.warmup):
            assert slab.step_n(8) == 0
        assert slab.upload(ic) == 0 and lib.wait(slab.task) == 0
        torch.cuda.synchronize()
        dist_barrier(dist)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            assert slab.step_n(p.steps) == 0
        assert lib.wait(slab.task) == 0
        torch.cuda.synchronize()
        sec = time.perf_counter() - t0
        dist_barrier(dist)
        slow = dist_max(dist, sec, "nccl")
        rows = slab.x.own
    finally:
        slab.close()
    if dist is not None:
        dist.destroy_process_group()
    if rank == 0:
        nu = p.node_updates * args.steps
        print(json.dumps({"metric": "node-updates/s", "value": nu / slow, "unit": "node-updates/s",
                          "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": 1e3 * slow / args.steps, "higher_is_better": True,
                          "scaling": "strong", "dtype": "f32", "data": "synthetic",
                          "config": {"workload": f"dist: one {p.nx}x{p.ny} grid in {world} row slabs "
                                                 f"(one per rank), {p.steps} time steps per bench step, "
                                                 "4 halo rows swapped by NCCL send/recv every 2 steps",
                                     "rows_rank0": rows},
                          "timing": "host clock between device synchronisations, max over ranks"}),
              flush=True)
    return 0


def precision_measure(args, with_reference=True):
    """4096x4096 precision study: FP32 vs FP64 library every 500 steps up to 4000 steps (the
    FP64 library equals the reference double build value for value, so this is also FP32 vs
    the reference double build), FP64 energy drift; with_reference: both builds against the
    reference's own CPU builds after 500 steps (~2 min of host time)."""
    from oracle.oracle import Reference, aos_to_soa, fields, max_abs, rel_l2

    p = workloads.precision_4096()
    n = p.nx
    libs = {"f": capi.Lib("f"), "d": capi.Lib("d")}
    tasks, ics = {}, {}
    for prec, lib in libs.items():
        mat = lib.le_init_material(p.c1, p.c2, p.rho)
        t = lib.le_init_task(p.dt, (p.hx, p.hy), mat, (n, n), capi.ST_AOS)
        for cx, cy, r, s in p.disks:
            lib.le_set_ball(t, (cx, cy), r, s)
        assert lib.sync_host(t) == 0
        g = lib.grid_view(t).reshape(n, n, 5)
        vx, vy = p.noise_fields(lib.dtype)
        g[:, :, 0] = vx
        g[:, :, 1] = vy
        ics[prec] = lib.grid_view(t).copy()
        assert lib.sync_device(t) == 0
        tasks[prec] = t
    e0 = libs["d"].diagnostics(tasks["d"])[1]["energy"]
    rows = []
    snap = {}
    for k in range(1, p.steps // 500 + 1):
        out = {}
        for prec, lib in libs.items():
            assert lib.step_n(tasks[prec], 500) == 0
            g = np.zeros(5 * n * n, lib.dtype)
            assert lib.download(tasks[prec], g) == 0
            out[prec] = fields(g, n, n, 1)
            if k == 1 and with_reference:
                snap[prec] = g
        ed = libs["d"].diagnostics(tasks["d"])[1]["energy"]
        ef = libs["f"].diagnostics(tasks["f"])[1]["energy"]
        rows.append({"step": 500 * k, "fp32_vs_fp64_rel_l2": rel_l2(out["f"], out["d"]).tolist(),
                     "fp32_vs_fp64_max_abs": max_abs(out["f"], out["d"]).tolist(),
                     "fp64_energy": ed, "fp64_energy_drift": (ed - e0) / e0,
                     "fp32_state_energy_drift": (ef - e0) / e0})
        print(json.dumps(rows[-1]), file=sys.stderr, flush=True)
    for prec, lib in libs.items():
        lib.le_free_task(tasks[prec])
    line = {"metric": "precision", "workload": "precision_4096: 4096x4096, c1=2, c2=1, rho=1, dt=0.5h/c1, "
                                              "8 seeded disks + U(+-1e-3) noise on vx, vy", "steps": p.steps,
            "every": 500, "rows": rows}
    # the reference's own CPU builds (simple/, OpenMP on all host cores) from the same initial
    # states for the first 500 steps, against the library's FP64 / FP32 results at step 500
    if Reference.available("d") and with_reference:
        threads = os.cpu_count() or 1
        for prec in ("d", "f"):
            ref = Reference(prec)
            g = ics[prec].copy()
            secs = ref.run(g, n, n, p.dt, p.hx, p.hy, p.c1, p.c2, p.rho, 1, 500, threads)
            fr = fields(g, n, n, 1)
            fl = fields(snap[prec], n, n, 1)
            line[f"step500_lib_{prec}_vs_reference_{prec}_rel_l2"] = rel_l2(fl, fr).tolist()
            line[f"step500_lib_{prec}_vs_reference_{prec}_max_abs"] = max_abs(fl, fr).tolist()
            line[f"reference_{prec}_cpu_seconds"] = secs
            if prec == "d":
                ref_d = fr
        line["step500_reference_f_vs_reference_d_rel_l2"] = rel_l2(fr, ref_d).tolist()
        line["reference_threads"] = threads
    return line


def run_precision(args):
    print(json.dumps(precision_measure(args, with_reference=not args.no_cpu)), flush=True)
    return 0


def run_precision_reference(args):
    """CPU only: the reference's own float and double builds (simple/, OpenMP on all host
    cores) on the 4096x4096 precision workload, relative L2 and max-abs of float against
    double every 500 steps up to 4000 -- the reference's own FP32 divergence curve beside
    which `--workload precision` reports the library's (takes ~1 h on 8 cores)."""
    from oracle.oracle import Oracle, Reference, fields, max_abs, rel_l2

    p = workloads.precision_4096(steps=args.time_steps or 4000)
    n = p.nx
    threads = os.cpu_count() or 1
    grids = {}
    for prec in ("f", "d"):
        o = Oracle(prec)
        g = np.zeros(5 * n * n, o.dtype)
        for cx, cy, r, s in p.disks:
            o.set_ball(g, n, n, p.hx, p.hy, 1, cx, cy, r, s)
        vx, vy = p.noise_fields(o.dtype)
        a = g.reshape(n, n, 5)
        a[:, :, 0] = vx
        a[:, :, 1] = vy
        grids[prec] = g
    refs = {prec: Reference(prec) for prec in ("f", "d")}
    rows = []
    for k in range(1, p.steps // 500 + 1):
        secs = {}
        for prec in ("f", "d"):
            secs[prec] = refs[prec].run(grids[prec], n, n, p.dt, p.hx, p.hy, p.c1, p.c2, p.rho, 1, 500, threads)
        ff, fd = fields(grids["f"], n, n, 1), fields(grids["d"], n, n, 1)
        rows.append({"step": 500 * k, "reference_f_vs_d_rel_l2": rel_l2(ff, fd).tolist(),
                     "reference_f_vs_d_max_abs": max_abs(ff, fd).tolist(), "seconds": secs})
        print(json.dumps(rows[-1]), file=sys.stderr, flush=True)
    print(json.dumps({"metric": "precision-reference", "threads": threads, "rows": rows}), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="single",
                    choices=["single", "batched", "serving", "precision", "precision-reference", "slabs",
                             "parity", "dist"])
    ap.add_argument("--slabs", default="2,4", help="slabs: slab counts besides the whole task")
    ap.add_argument("--window", type=int, default=256, help="steps per persistent launch (batched/serving)")
    ap.add_argument("--rates", default="10,50,200,2000", help="serving: request rates per second")
    ap.add_argument("--requests", type=int, default=48, help="serving: requests per rate")
    ap.add_argument("--budget", type=int, default=48, help="serving: HBM budget in GiB")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 leg")
    ap.add_argument("--no-tune", action="store_true", help="batched: skip the batched-path autotuner")
    ap.add_argument("--time-steps", type=int, default=None, help="time steps per solve (default 1000)")
    ap.add_argument("--no-extras", action="store_true",
                    help="single: skip the batched and serving measurements added to the line")
    ap.add_argument("--extra-rates", default="10,200", help="single: serving request rates in the line")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "batched":
        return run_batched(args)
    if args.workload == "serving":
        return run_serving(args)
    if args.workload == "precision":
        return run_precision(args)
    if args.workload == "precision-reference":
        return run_precision_reference(args)
    if args.workload == "slabs":
        return run_slabs(args)
    if args.workload == "parity":
        return run_parity(args)
    if args.workload == "dist":
        return run_dist(args)

    world, rank, local = dist_setup()
    backend = "nccl"
    dist = dist_init(world, local, backend)
    lib = capi.Lib("f")
    assert lib.set_device(local) == 0
    p = workloads.single_8192() if args.time_steps is None else workloads.single_8192(args.time_steps)
    peak, peak_kind = measured_peaks()

    slow_ms, clocks, e2e_s, e2e_serial, ic, plan = measure_ours(lib, "f", p, args.steps, args.warmup, dist,
                                                                backend, local)
    nu = p.node_updates * args.steps * world
    value = nu / (slow_ms * 1e-3)
    depth = plan["depth"]  # time steps per fused launch of the grid (temporal blocking)
    per_solve = p.steps // depth + p.steps % depth
    launches = args.steps * per_solve  # fused launches of the whole grid
    # a launch of the grid in halves is 3 kernel launches (band, upper and lower rows) that
    # overlap; its duration is that of the whole update
    parts = plan.get("launch_parts", 1)
    avg_launch_s = slow_ms * 1e-3 / launches
    # algorithmic bytes: one read + one write of the state per node-update, depth node-updates
    # per node and launch
    alg_bytes = BYTES_PER_NU["f"] * p.nodes * depth
    achieved = alg_bytes / avg_launch_s / 1e9
    kname = (f"{'fused_pair_kernel' if plan['warps_per_task'] == 2 else 'fused_step_kernel'}"
             f"<float, V={plan['lanes']}, depth={depth}>")
    traffic = profiled_traffic().get(f"fused_step_f32_8192_depth{depth}")
    line = {
        "metric": "node-updates/s", "value": value, "unit": "node-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": slow_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": single_config(p, f"independent solves x{world}"),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind,
                     "traffic": traffic.get("bytes_per_launch") if traffic else None,
                     "kernel": kname, "variant": plan["variant"], "seg_len": plan["seg_len"],
                     "launch_parts": parts, "algorithmic_bytes_per_launch": alg_bytes},
        "e2e": {"value": nu / e2e_serial, "unit": "node-updates/s",
                "h2d_bytes_per_step": int(ic.nbytes), "d2h_bytes_per_step": int(ic.nbytes),
                "how": "one task: upload, steps and read-back of each solve in turn",
                "pipelined_value": nu / e2e_s,
                "pipelined_how": "two tasks alternate: solve k's upload and steps are queued before solve "
                                 "k-1's fields are read back, so copies (and the launch tails of the two "
                                 "streams) overlap"},
        "gpu_launches": launches * parts,  # step-kernel launches in the timed region
        "clocks": clocks,
    }
    if not args.no_fp64:
        libd = capi.Lib("d")
        assert libd.set_device(local) == 0
        ksteps = min(args.steps, 2)
        d_ms, d_clk, d_e2e, _, d_ic, d_plan = measure_ours(libd, "d", p, ksteps, min(args.warmup, 3), dist,
                                                            backend, local)
        d_nu = p.node_updates * ksteps * world
        d_depth = d_plan["depth"]
        d_avg = d_ms * 1e-3 / (ksteps * (p.steps // d_depth + p.steps % d_depth))
        d_ach = BYTES_PER_NU["d"] * p.nodes * d_depth / d_avg / 1e9
        line["fp64"] = {"value": d_nu / (d_ms * 1e-3), "unit": "node-updates/s", "steps": ksteps,
                        "ms_per_step": d_ms / ksteps, "e2e": d_nu / d_e2e,
                        "roofline": {"bound": "hbm", "achieved": d_ach, "peak": peak, "unit": "GB/s",
                                     "frac": d_ach / peak,
                                     "kernel": (f"{'fused_pair_kernel' if d_plan['warps_per_task'] == 2 else 'fused_step_kernel'}"
                                                f"<double, V={d_plan['lanes']}, depth={d_depth}>"),
                                     "launch_parts": d_plan.get("launch_parts", 1)},
                        "clocks": d_clk}
    if world == 1 and not args.no_extras:
        # the batched and serving targets on the same GPU (one process; skipped under torchrun)
        line["batched"] = batched_measure(args)
        line["serving"] = serving_measure(args, [float(r) for r in args.extra_rates.split(",")])
        line["precision"] = precision_measure(args, with_reference=False)
    if rank == 0 and not args.no_cpu:
        cb = cpu_reference_sample(p)
        line["cpu_baseline"] = cb["simple"]
        if "pthread" in cb:
            line["cpu_baseline_pthread"] = cb["pthread"]
    if dist is not None:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())

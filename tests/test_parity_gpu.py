"""Parity of the CUDA path with the reference, through the C ABI.

Tolerances (per field, relative L2 = ||a-b|| / ||b||):
  * FP64 library vs the reference double build: <= 1e-12, and equal value for value (the
    FP64 kernels round every operation as the reference does; -0 and +0 count as equal)
  * FP32 library vs the reference float build:  <= 1e-5, and vs the double build too.
    Where a field's norm is tiny next to the others (e.g. noise-level vx beside unit
    stresses on a 3x7 grid) one float ulp of the large fields is already ~1e-4 of the
    small field's norm, and the reference's own float build sits up to 3e-5 from its
    double build; for such a field the bound is 4x the reference float build's own
    distance from its double build when that exceeds 1e-5/4.
Max-abs error of every result against the FP64 reference is printed (pytest -s).
"""
import hashlib

import numpy as np
import pytest

from golden_cases import arrays, cases, summary
from le2d_b200 import capi, workloads
from oracle.oracle import ST_AOS, ST_SOA, Oracle, aos_to_soa, fields, max_abs, rel_l2

pytestmark = pytest.mark.gpu

TOL = {"d": 1e-12, "f": 1e-5}
METHODS = {"fused": capi.LE2D_METHOD_FUSED, "split": capi.LE2D_METHOD_SPLIT}


@pytest.fixture(scope="module")
def libs():
    return {p: capi.Lib(p) for p in ("f", "d")}


def make_task(lib, c, method=capi.LE2D_METHOD_FUSED):
    mat = lib.le_init_material(c["c1"], c["c2"], c["rho"])
    t = lib.le_init_task(c["dt"], (c["hx"], c["hy"]), mat, (c["nx"], c["ny"]), c["stype"])
    assert t.grid
    assert lib.set_method(t, method) == 0
    return t


def run(lib, c, g0, steps, method=capi.LE2D_METHOD_FUSED, per_call=True):
    """Steps a copy of g0 through the library; returns the final grid (task layout)."""
    t = make_task(lib, c, method)
    try:
        assert lib.upload(t, np.ascontiguousarray(g0, dtype=lib.dtype)) == 0
        if per_call:
            step = lib.le_step if c["stype"] == ST_AOS else lib.le_step_soa
            for _ in range(steps):
                step(t)
        else:
            assert lib.step_n(t, steps) == 0
        out = np.zeros(5 * c["nx"] * c["ny"], lib.dtype)
        assert lib.download(t, out) == 0
        assert lib.last_error(t) == 0, lib.strerror(lib.last_error(t))
        return out
    finally:
        lib.le_free_task(t)


def fp32_tolerance(want_f, want_d):
    """Per-field FP32 bound: 1e-5, or 4x the reference float build's distance from its
    double build where that distance exceeds 1e-5/4."""
    gap = rel_l2(want_f, want_d)
    return np.maximum(TOL["f"], 4.0 * gap)


def check(prec, got, want, want_d, nx, ny, stype, label):
    g = fields(got, nx, ny, stype)
    w = fields(want, nx, ny, stype)
    wd = fields(want_d, nx, ny, stype)
    err = rel_l2(g, w)
    mab = max_abs(g, wd)
    print(f"\n{label}: rel_l2={np.array2string(err, precision=2)} max_abs_vs_fp64={np.array2string(mab, precision=2)}")
    if prec == "d":
        assert np.all(err <= TOL["d"]), (label, err)
        # the FP64 kernels round every operation as the reference double build does
        assert np.array_equal(g, w), (label, "FP64 not bitwise", int(np.sum(g != w)))
    else:
        tol = fp32_tolerance(w, wd)
        assert np.all(err <= tol), (label, err, tol)
        assert np.all(rel_l2(g, wd) <= tol), (label, rel_l2(g, wd), tol)


@pytest.mark.parametrize("method", sorted(METHODS))
@pytest.mark.parametrize("prec", ["f", "d"])
@pytest.mark.parametrize("name", sorted(cases()))
def test_golden_case(libs, name, prec, method):
    c = cases()[name]
    a, ad = arrays(prec), arrays("d")
    got = run(libs[prec], c, a[f"{name}__in"], c["steps"], METHODS[method])
    check(prec, got, a[f"{name}__out"], ad[f"{name}__out"], c["nx"], c["ny"], c["stype"],
          f"{name}/{prec}/{method}")


@pytest.mark.parametrize("prec", ["f", "d"])
def test_plain_512_full_length(libs, prec):
    """The reference driver's plain workload at its full length (512x512, c1=2, c2=1,
    rho=1, dt=0.25, disk r=25 at the centre with s=1, 200 steps, AoS): one le_step call
    per step as simple/main.c makes them.  FP64: the final grid hashes to the digest of the
    reference double build's own output (tests/golden/golden.json, plain_512); FP32: within
    1e-5 of the reference float and double builds (the C oracle, which reproduces both bit
    for bit), max-abs against the double build printed."""
    lib = libs[prec]
    nx = ny = 512
    c = dict(nx=nx, ny=ny, hx=1.0, hy=1.0, c1=2.0, c2=1.0, rho=1.0, dt=0.25, stype=ST_AOS)
    t = make_task(lib, c)
    try:
        lib.le_set_ball(t, (256.0, 256.0), 25.0, 1.0)
        for _ in range(200):
            lib.le_step(t)
        assert lib.sync_host(t) == 0 and lib.last_error(t) == 0
        got = lib.grid_view(t).copy()
    finally:
        lib.le_free_task(t)
    digest = summary()["plain_512"]
    if prec == "d":
        assert hashlib.sha256(got.tobytes()).hexdigest() == digest["d"]["sha256"]
        print(f"\nplain_512/d: bytes equal to the reference double build's output")
        return
    want = {}
    for q in ("f", "d"):
        o = Oracle(q)
        g = np.zeros(5 * nx * ny, o.dtype)
        o.set_ball(g, nx, ny, 1.0, 1.0, ST_AOS, 256.0, 256.0, 25.0, 1.0)
        o.run(g, nx, ny, 0.25, 1.0, 1.0, 2.0, 1.0, 1.0, ST_AOS, 200)
        assert hashlib.sha256(g.tobytes()).hexdigest() == digest[q]["sha256"]  # the reference's bytes
        want[q] = g
    check("f", got, want["f"], want["d"], nx, ny, ST_AOS, "plain_512/f")
    e = rel_l2(fields(got, nx, ny, ST_AOS), fields(want["d"], nx, ny, ST_AOS))
    assert np.all(e <= TOL["f"]), e


@pytest.mark.parametrize("prec", ["f", "d"])
def test_set_ball_device_bitwise(libs, prec):
    """le_set_ball on the device reproduces the reference initial condition bit for bit."""
    lib = libs[prec]
    o = Oracle(prec)
    for name in ("disks_noise_37x53", "strips_250x40", "soa_40x32"):
        c = cases()[name]
        t = make_task(lib, c)
        try:
            for cx, cy, r, s in c["disks"]:
                lib.le_set_ball(t, (cx, cy), r, s)
            assert lib.sync_host(t) == 0
            got = lib.grid_view(t).copy()
        finally:
            lib.le_free_task(t)
        want = np.zeros_like(got)
        for d in c["disks"]:
            o.set_ball(want, c["nx"], c["ny"], c["hx"], c["hy"], c["stype"], *d)
        assert got.tobytes() == want.tobytes(), name


def _medium(prec, stype, nx=300, ny=200, steps=150):
    rng = np.random.default_rng(7)
    p = dict(nx=nx, ny=ny, hx=1.0, hy=0.8, c1=2.5, c2=1.2, rho=1.7, stype=stype)
    p["dt"] = 0.45 * 0.8 / 2.5
    o = Oracle(prec)
    g0 = np.zeros(5 * nx * ny, o.dtype)
    for _ in range(5):
        o.set_ball(g0, nx, ny, 1.0, 0.8, stype, float(rng.uniform(0, nx)), float(rng.uniform(0, ny * 0.8)),
                   float(rng.uniform(5, 40)), float(rng.uniform(-2, 2)))
    g0 += rng.uniform(-1e-3, 1e-3, size=g0.shape).astype(o.dtype)
    return p, g0, steps


@pytest.mark.parametrize("method", sorted(METHODS))
@pytest.mark.parametrize("stype", [ST_AOS, ST_SOA])
@pytest.mark.parametrize("prec", ["f", "d"])
def test_oracle_medium(libs, prec, stype, method):
    """300x200, five disks + noise, 150 steps (waves cross every boundary), vs the oracle."""
    p, g0, steps = _medium(prec, stype)
    want = g0.copy()
    Oracle(prec).run(want, p["nx"], p["ny"], p["dt"], p["hx"], p["hy"], p["c1"], p["c2"], p["rho"], stype, steps)
    gd = g0.astype(np.float64)
    Oracle("d").run(gd, p["nx"], p["ny"], p["dt"], p["hx"], p["hy"], p["c1"], p["c2"], p["rho"], stype, steps)
    got = run(libs[prec], p, g0, steps, METHODS[method], per_call=False)
    check(prec, got, want, gd, p["nx"], p["ny"], stype, f"medium/{prec}/{stype}/{method}")


@pytest.mark.parametrize("prec", ["f", "d"])
def test_soa_far_end_differs_from_aos(libs, prec):
    """le_step_soa keeps the reference SoA step's far-end rows; le_step does not."""
    p, g0, steps = _medium(prec, ST_AOS, 64, 48, 60)
    aos = run(libs[prec], p, g0, steps)
    ps = dict(p, stype=ST_SOA)
    soa = run(libs[prec], ps, aos_to_soa(g0, 64, 48), steps)
    assert not np.allclose(aos_to_soa(aos, 64, 48), soa, rtol=0, atol=1e-9)


@pytest.mark.parametrize("prec", ["f", "d"])
def test_step_n_equals_single_steps(libs, prec):
    """The graph-replayed multi-step call is bitwise the same as one le_step per step."""
    p, g0, _ = _medium(prec, ST_AOS, 200, 150)
    a = run(libs[prec], p, g0, 200, per_call=True)
    b = run(libs[prec], p, g0, 200, per_call=False)
    assert a.tobytes() == b.tobytes()


def variants(lib):
    """Compiled fused-kernel variants with their temporal-block depth: {variant: depth}."""
    c = dict(nx=8, ny=8, hx=1.0, hy=1.0, c1=2.0, c2=1.0, rho=1.0, dt=0.25, stype=ST_AOS)
    t = make_task(lib, c)
    out = {}
    try:
        v = 0
        while lib.set_variant(t, v, 0) == 0:
            out[v] = lib.get_plan(t)["depth"]
            v += 1
    finally:
        lib.le_free_task(t)
    return out


@pytest.mark.parametrize("prec", ["f", "d"])
def test_variants_and_segments_bitwise_equal(libs, prec):
    """Every compiled variant and row-segment length computes the same per-node operations,
    so results are bitwise equal; also matches the oracle (AoS and SoA far end).  Variants
    of temporal-block depth 2 run two steps per launch (AoS; the SoA far end takes single
    steps), with the odd last step of 41 as a single step."""
    lib = libs[prec]
    vs = variants(lib)
    assert sorted(set(vs.values())) == [1, 2]
    for stype in (ST_AOS, ST_SOA):
        p, g0, steps = _medium(prec, stype, 263, 171, 41)
        outs = []
        for var in sorted(vs):
            for seg in (0, 7, 33, 171):
                t = make_task(lib, p)
                try:
                    assert lib.set_variant(t, var, seg) == 0
                    assert lib.upload(t, g0.copy()) == 0
                    assert lib.step_n(t, steps) == 0
                    o = np.zeros_like(g0)
                    assert lib.download(t, o) == 0
                    outs.append(((var, seg), o))
                finally:
                    lib.le_free_task(t)
        for key, o in outs[1:]:
            assert o.tobytes() == outs[0][1].tobytes(), key
        want = g0.copy()
        Oracle(prec).run(want, p["nx"], p["ny"], p["dt"], p["hx"], p["hy"], p["c1"], p["c2"], p["rho"], stype, steps)
        gd = g0.astype(np.float64)
        Oracle("d").run(gd, p["nx"], p["ny"], p["dt"], p["hx"], p["hy"], p["c1"], p["c2"], p["rho"], stype, steps)
        check(prec, outs[0][1], want, gd, p["nx"], p["ny"], stype, f"variants/{prec}/{stype}")


@pytest.mark.parametrize("prec", ["f", "d"])
def test_temporal_blocking_edges(libs, prec):
    """Two steps per launch on grids and segments that put the clamped ends everywhere a
    tile can meet them: widths around the strip width (one strip, two strips, a last strip
    of one column), heights below and around the segment length, segments of 1 and 3 rows.
    Bitwise equal to single steps, and to the oracle within tolerance."""
    lib = libs[prec]
    vs = variants(lib)
    two = [v for v, d in vs.items() if d == 2]
    one = [v for v, d in vs.items() if d == 1][0]
    rng = np.random.default_rng(11)
    for nx, ny in ((3, 3), (5, 4), (9, 7), (57, 3), (111, 20), (112, 33), (113, 17), (225, 9), (130, 64)):
        c = dict(nx=nx, ny=ny, hx=1.0, hy=0.9, c1=2.0, c2=1.1, rho=1.3, dt=0.2, stype=ST_AOS)
        o = Oracle(prec)
        g0 = rng.uniform(-1, 1, size=5 * nx * ny).astype(o.dtype)
        steps = 9
        want = g0.copy()
        o.run(want, nx, ny, c["dt"], c["hx"], c["hy"], c["c1"], c["c2"], c["rho"], ST_AOS, steps)
        gd = g0.astype(np.float64)
        Oracle("d").run(gd, nx, ny, c["dt"], c["hx"], c["hy"], c["c1"], c["c2"], c["rho"], ST_AOS, steps)
        ref = None
        for var, seg in [(one, 0)] + [(v, s) for v in two for s in (0, 1, 3, 5, 16)]:
            t = make_task(lib, c)
            try:
                assert lib.set_variant(t, var, seg) == 0
                assert lib.upload(t, g0.copy()) == 0
                assert lib.step_n(t, steps) == 0
                got = np.zeros_like(g0)
                assert lib.download(t, got) == 0
                assert lib.last_error(t) == 0
            finally:
                lib.le_free_task(t)
            if ref is None:
                ref = got
                check(prec, got, want, gd, nx, ny, ST_AOS, f"edges/{prec}/{nx}x{ny}")
            else:
                assert got.tobytes() == ref.tobytes(), (nx, ny, var, seg)


@pytest.mark.parametrize("prec", ["f", "d"])
def test_interior_tiles_lean_loops(libs, prec):
    """Grids wide and tall enough that most tiles are interior (strip inside the grid, 2 rows
    of margin per step above and below), which the lean loops take, with even and odd
    segment lengths: every variant, one or two steps per launch, bitwise equal to the first
    one-step variant."""
    lib = libs[prec]
    vs = variants(lib)
    one = [v for v, d in vs.items() if d == 1][0]
    rng = np.random.default_rng(23)
    for nx, ny, steps in ((517, 301, 10), (1000, 97, 7)):
        c = dict(nx=nx, ny=ny, hx=1.0, hy=0.9, c1=2.0, c2=1.1, rho=1.3, dt=0.2, stype=ST_AOS)
        g0 = rng.uniform(-1, 1, size=5 * nx * ny).astype(lib.dtype)
        ref = None
        for var, seg in [(one, 0)] + [(v, s) for v in sorted(vs) for s in (0, 8, 9, 40)]:
            t = make_task(lib, c)
            try:
                assert lib.set_variant(t, var, seg) == 0
                assert lib.upload(t, g0.copy()) == 0
                assert lib.step_n(t, steps) == 0
                got = np.zeros_like(g0)
                assert lib.download(t, got) == 0
                assert lib.last_error(t) == 0
            finally:
                lib.le_free_task(t)
            if ref is None:
                ref = got
            else:
                assert got.tobytes() == ref.tobytes(), (nx, ny, var, seg)


# Materials for the exact-tie states: one whose constants are dyadic (c1 = 2, c2 = 1,
# rho = 1, dt = 0.25, h = 1, so Courant numbers 0.5 / 0.25), where the fields stay small
# multiples of eps for several steps and ties recur; and a general one.
TIE_MATERIALS = {
    "dyadic": dict(hx=1.0, hy=1.0, c1=2.0, c2=1.0, rho=1.0, dt=0.25),
    "general": dict(hx=0.97, hy=1.03, c1=2.1, c2=1.13, rho=1.37, dt=0.21),
}


@pytest.mark.parametrize("mat", sorted(TIE_MATERIALS))
@pytest.mark.parametrize("prec", ["f", "d"])
def test_exact_ties(libs, prec, mat):
    """Velocity components whose neighbours differ by exactly +-eps (one component, or
    both), all else zero: P = D + eps or Q = eps - D is exactly 0 at many faces, in the
    x-sweep and -- after it -- in the y-sweep, so slope ratios x/0 and 0/0 reach the
    limiter and which faces tie depends on every rounding of the x-sweep.  Every variant
    and the plain method, one to three steps (two-step variants take the second and third
    on warp pairs / two-step tiles).
      FP64: equal value for value to the reference double build (the kernels round each
        operation as it does), which is what makes the ties fall on the same faces.
      FP32: within 1e-5 of the reference double build.  The reference float build adds
        eps in double (`r1 += TVD2_EPS`, a double literal), so its P is never 0 but the
        2.5e-15 remainder of the double eps over the float one, and its results here sit
        up to ~3e-2 from its own double build; the FP32 library's tie rule is the double
        build's (P = 0 exactly), and its result is compared with both under the usual
        allowance for the float build's own distance.  The plain method forms invariants
        and adds eps in float, like neither build, and is held to that allowance only."""
    lib = libs[prec]
    o = Oracle(prec)
    nx, ny = 260, 150
    c = dict(nx=nx, ny=ny, stype=ST_AOS, **TIE_MATERIALS[mat])
    eps = o.dtype(1e-6)
    rng = np.random.default_rng(31)
    for comps in (((0, 1),), ((1, -1),), ((0, 1), (1, -1))):  # vx in {0, eps}, vy in {0, -eps}
        g0 = np.zeros(5 * nx * ny, dtype=o.dtype)
        for field, sign in comps:
            g0[field::5] = sign * rng.integers(0, 2, size=nx * ny).astype(o.dtype) * eps
        for steps in (1, 2, 3):
            want = g0.copy()
            o.run(want, nx, ny, c["dt"], c["hx"], c["hy"], c["c1"], c["c2"], c["rho"], ST_AOS, steps)
            gd = g0.astype(np.float64)
            Oracle("d").run(gd, nx, ny, c["dt"], c["hx"], c["hy"], c["c1"], c["c2"], c["rho"], ST_AOS, steps)
            runs = [(f"v{var}", var, capi.LE2D_METHOD_FUSED) for var in sorted(variants(lib))]
            runs.append(("split", 0, capi.LE2D_METHOD_SPLIT))
            for name, var, method in runs:
                t = make_task(lib, c, method)
                try:
                    if method == capi.LE2D_METHOD_FUSED:
                        assert lib.set_variant(t, var, 16) == 0
                    assert lib.upload(t, g0.copy()) == 0
                    assert lib.step_n(t, steps) == 0
                    got = np.zeros_like(g0)
                    assert lib.download(t, got) == 0
                    assert lib.last_error(t) == 0
                finally:
                    lib.le_free_task(t)
                assert np.all(np.isfinite(got)), (comps, name, steps)
                label = f"ties/{prec}/{mat}/{len(comps)}c-f{comps[0][0]}/{name}/{steps}"
                check(prec, got, want, gd, nx, ny, ST_AOS, label)
                if prec == "f" and method == capi.LE2D_METHOD_FUSED:
                    e = rel_l2(fields(got, nx, ny, ST_AOS), fields(gd, nx, ny, ST_AOS))
                    assert np.all(e <= TOL["f"]), (label, e)


@pytest.mark.parametrize("prec", ["f", "d"])
def test_temporal_blocking_against_tiling_schedule(libs, prec):
    """The two-step (temporal-blocking) variants against the reference's own alternative
    schedule, tiling/ le_step_all2 (two buffers, a zero ring of two nodes around the grid,
    increments associated (v + d1) + d2), run from its sources (oracle/_ref): on the nodes
    that schedule's ends cannot reach after s steps (2 per step from each edge) the two are
    the same scheme with other roundings -- FP64 within 1e-12, FP32 within 1e-5."""
    from oracle.oracle import ReferenceTiling

    if not ReferenceTiling.available(prec):
        pytest.skip("oracle/_ref not built")
    lib = libs[prec]
    nx, ny, steps = 300, 190, 6
    c = dict(nx=nx, ny=ny, hx=1.0, hy=0.9, c1=2.3, c2=1.2, rho=1.6, dt=0.17, stype=ST_AOS)
    rng = np.random.default_rng(12)
    o = Oracle(prec)
    g0 = np.zeros(5 * nx * ny, o.dtype)
    for _ in range(4):
        o.set_ball(g0, nx, ny, 1.0, 0.9, ST_AOS, float(rng.uniform(30, 270)), float(rng.uniform(30, 140)),
                   float(rng.uniform(5, 25)), float(rng.uniform(-2, 2)))
    g0[0::5] += rng.uniform(-1e-3, 1e-3, nx * ny).astype(o.dtype)
    want = g0.copy()
    ReferenceTiling(prec).run(want, nx, ny, c["dt"], c["hx"], c["hy"], c["c1"], c["c2"], c["rho"], steps)
    m = 2 * steps
    fw = fields(want, nx, ny, ST_AOS)[:, m:ny - m, m:nx - m]
    two_step = [v for v, depth in sorted(variants(lib).items()) if depth == 2]
    assert two_step
    for var in two_step:
        t = make_task(lib, c)
        try:
            assert lib.set_variant(t, var, 0) == 0
            assert lib.upload(t, g0.copy()) == 0
            assert lib.step_n(t, steps) == 0
            got = np.zeros_like(g0)
            assert lib.download(t, got) == 0 and lib.last_error(t) == 0
        finally:
            lib.le_free_task(t)
        err = rel_l2(fields(got, nx, ny, ST_AOS)[:, m:ny - m, m:nx - m], fw)
        print(f"\ntiling/{prec}/v{var}: interior rel_l2={np.array2string(err, precision=2)}")
        assert np.all(err <= TOL[prec]), (var, err)


@pytest.mark.parametrize("prec", ["f", "d"])
def test_uniform_state_is_fixed_point(libs, prec):
    c = dict(nx=257, ny=131, hx=1.0, hy=1.0, c1=2.0, c2=1.0, rho=1.0, dt=0.25, stype=ST_AOS)
    g0 = np.tile(np.array([0.3, -0.2, 1.5, 0.25, -0.7], libs[prec].dtype), 257 * 131)
    got = run(libs[prec], c, g0, 50, per_call=False)
    assert got.tobytes() == g0.tobytes()


@pytest.mark.parametrize("prec", ["f", "d"])
def test_diagnostics_and_sim_time(libs, prec):
    lib = libs[prec]
    c = cases()["disks_noise_37x53"]
    g = arrays(prec)["disks_noise_37x53__out"]
    t = make_task(lib, c)
    try:
        assert lib.upload(t, g.copy()) == 0
        rc, d = lib.diagnostics(t)
        assert rc == 0
        # the library computes with the material as stored in `real` (e.g. float(1.7))
        m = [float(lib.dtype(c[k])) for k in ("hx", "hy", "c1", "c2", "rho")]
        want = Oracle(prec).diag(g, c["nx"], c["ny"], *m, c["stype"])
        assert abs(d["energy"] - want[0]) <= 1e-12 * abs(want[0])
        assert np.allclose(d["sumsq"], want[1:6], rtol=1e-12, atol=0)
        assert np.array_equal(d["maxabs"], want[6:11])
        assert lib.step_n(t, 137) == 0
        rc, tt, st = lib.sim_time(t)
        acc = 0.0
        for _ in range(137):
            acc += float(lib.dtype(c["dt"]))
        assert rc == 0 and st == 137 and tt == acc
    finally:
        lib.le_free_task(t)


@pytest.mark.parametrize("prec", ["f", "d"])
def test_upload_download_roundtrip(libs, prec):
    lib = libs[prec]
    for stype in (ST_AOS, ST_SOA):
        c = dict(nx=131, ny=77, hx=1.0, hy=1.0, c1=2.0, c2=1.0, rho=1.0, dt=0.25, stype=stype)
        g = np.random.default_rng(1).standard_normal(5 * 131 * 77).astype(lib.dtype)
        t = make_task(lib, c)
        try:
            assert lib.upload(t, g) == 0
            out = np.zeros_like(g)
            assert lib.download(t, out) == 0
            assert out.tobytes() == g.tobytes()
        finally:
            lib.le_free_task(t)


def _window_parity(lib, prec, p: workloads.Problem, steps, windows):
    """Full-size run; each window is checked against the oracle on a sub-grid that holds
    the window plus the domain of dependence (2 nodes per sweep per step)."""
    c = dict(nx=p.nx, ny=p.ny, hx=p.hx, hy=p.hy, c1=p.c1, c2=p.c2, rho=p.rho, dt=p.dt, stype=ST_AOS)
    t = make_task(lib, c)
    try:
        for cx, cy, r, s in p.disks:
            lib.le_set_ball(t, (cx, cy), r, s)
        assert lib.sync_host(t) == 0
        g0 = lib.grid_view(t).copy().reshape(p.ny, p.nx, 5)
        assert lib.step_n(t, steps) == 0
        assert lib.sync_host(t) == 0
        g1 = lib.grid_view(t).reshape(p.ny, p.nx, 5)
        m = 2 * steps
        for (x0, y0, w, h) in windows:
            sx0, sy0 = max(0, x0 - m), max(0, y0 - m)
            sx1, sy1 = min(p.nx, x0 + w + m), min(p.ny, y0 + h + m)
            sub = np.ascontiguousarray(g0[sy0:sy1, sx0:sx1]).reshape(-1)
            for po, subp in ((prec, sub), ("d", sub.astype(np.float64))):
                o = Oracle(po)
                ref = subp.copy()
                o.run(ref, sx1 - sx0, sy1 - sy0, p.dt, p.hx, p.hy, p.c1, p.c2, p.rho, ST_AOS, steps)
                ref = ref.reshape(sy1 - sy0, sx1 - sx0, 5)[y0 - sy0:y0 - sy0 + h, x0 - sx0:x0 - sx0 + w]
                got = g1[y0:y0 + h, x0:x0 + w]
                a = np.ascontiguousarray(got.transpose(2, 0, 1))
                b = np.ascontiguousarray(ref.transpose(2, 0, 1))
                if po == prec:
                    err = rel_l2(a, b)
                    assert np.all(err <= TOL[prec]), ((x0, y0), err)
                else:
                    print(f"\nwindow {(x0, y0)} {prec}: max_abs_vs_fp64={max_abs(a, b)}")
    finally:
        lib.le_free_task(t)


@pytest.mark.slow
@pytest.mark.parametrize("prec", ["f", "d"])
def test_full_size_8192_windows(libs, prec):
    """The 8192x8192 workload (8 seeded disks), 12 steps, windows at two disks, a corner and an edge."""
    p = workloads.single_8192()
    wins = []
    for cx, cy, r, s in p.disks[:3]:  # windows across the disk rims, where the waves are
        x0, y0 = int(cx + r) - 96, int(cy) - 96
        wins.append((min(max(0, x0), p.nx - 192), min(max(0, y0), p.ny - 192), 192, 192))
    wins += [(0, 0, 160, 160), (p.nx - 130, 4000, 130, 150), (3000, p.ny - 140, 170, 140)]
    _window_parity(libs[prec], prec, p, 12, wins)


def test_pair_bounded_wait_gives_up(libs, monkeypatch):
    """Two-step tiles on warp pairs: a producer warp that never hands its rows over (test
    hook LE2D_TEST_STALL_PAIR) makes its partner's bounded wait run out; the step reports
    LE2D_ETIMEOUT at the next synchronisation and the device stays usable."""
    lib = libs["f"]
    pair = [v for v in variants(lib) if v in (9, 10)]
    c = dict(nx=300, ny=200, hx=1.0, hy=1.0, c1=2.0, c2=1.0, rho=1.0, dt=0.25, stype=ST_AOS)
    rng = np.random.default_rng(5)
    g0 = rng.uniform(-1, 1, size=5 * 300 * 200).astype(lib.dtype)
    monkeypatch.setenv("LE2D_TEST_STALL_PAIR", "0")
    t = make_task(lib, c)
    try:
        assert lib.set_variant(t, pair[0], 0) == 0
        assert lib.get_plan(t)["warps_per_task"] == 2
        assert lib.upload(t, g0.copy()) == 0
        assert lib.step_n(t, 2) == 0
        assert lib.wait(t) == capi.LE2D_ETIMEOUT
        assert lib.last_error(t) == capi.LE2D_ETIMEOUT
    finally:
        lib.le_free_task(t)
    monkeypatch.delenv("LE2D_TEST_STALL_PAIR")
    outs = []
    for var in (pair[0], 2):
        t = make_task(lib, c)
        try:
            assert lib.set_variant(t, var, 0) == 0
            assert lib.upload(t, g0.copy()) == 0
            assert lib.step_n(t, 6) == 0
            o = np.zeros_like(g0)
            assert lib.download(t, o) == 0
            assert lib.last_error(t) == 0
            outs.append(o)
        finally:
            lib.le_free_task(t)
    assert outs[0].tobytes() == outs[1].tobytes()


@pytest.mark.parametrize("prec", ["f", "d"])
def test_save_task_from_device_bytes(libs, prec, tmp_path):
    """le_save_task forms |v| on the device (4 bytes per node cross to the host): the file is
    byte-identical to the reference writer's -- the golden file of the reference, and the
    oracle's writer on stepped states in both layouts."""
    lib = libs[prec]
    c = cases()["ball_64x48"]
    t = make_task(lib, c)
    try:
        assert lib.upload(t, arrays(prec)["ball_64x48__out"].copy()) == 0
        path = tmp_path / "golden.vtk"
        assert lib.le_save_task(t, str(path)) == 0
        assert path.read_bytes() == arrays(prec)["ball_64x48__vtk"].tobytes()
    finally:
        lib.le_free_task(t)
    for stype in (ST_AOS, ST_SOA):
        p, g0, steps = _medium(prec, stype, 131, 77, 9)
        t = make_task(lib, p)
        try:
            assert lib.upload(t, g0.copy()) == 0
            assert lib.step_n(t, steps) == 0
            path = tmp_path / f"dev{stype}.vtk"
            assert lib.le_save_task(t, str(path)) == 0
            state = np.zeros_like(g0)
            assert lib.download(t, state) == 0
        finally:
            lib.le_free_task(t)
        ref = tmp_path / f"oracle{stype}.vtk"
        assert Oracle(prec).save_vtk(state, p["nx"], p["ny"], p["hx"], p["hy"], stype, str(ref)) == 0
        assert path.read_bytes() == ref.read_bytes(), stype


def test_per_call_steps_pair_up(libs):
    """Under a two-step plan, consecutive le_step calls run as two-step launches; a step held
    back is queued by itself before anything else touches the state (set_ball, diagnostics,
    download, save, step_n), and a changed dt is not paired with the previous call's.  The
    results are bitwise those of a one-step plan through the same call sequence."""
    lib = libs["f"]
    vs = variants(lib)
    two = [v for v in vs if vs[v] == 2][-1]
    c = dict(nx=150, ny=97, hx=1.0, hy=1.0, c1=2.0, c2=1.0, rho=1.0, dt=0.25, stype=ST_AOS)

    def sequence(variant):
        t = make_task(lib, c)
        log = []
        try:
            assert lib.set_variant(t, variant, 0) == 0
            lib.le_set_ball(t, (75.0, 48.0), 20.0, 1.0)
            for _ in range(3):
                lib.le_step(t)
            lib.le_set_ball(t, (30.0, 30.0), 8.0, -0.5)
            lib.le_step(t)
            rc, dg = lib.diagnostics(t)
            assert rc == 0
            log.append(dg["energy"])
            for _ in range(2):
                lib.le_step(t)
            t.dt = 0.2  # the next call's constants differ from the held-back one's
            lib.le_step(t)
            lib.le_step(t)
            lib.le_step(t)
            assert lib.step_n(t, 5) == 0
            lib.le_step(t)
            g = np.zeros(5 * c["nx"] * c["ny"], lib.dtype)
            assert lib.download(t, g) == 0
            log.append(lib.sim_time(t))
            lib.le_step(t)
            assert lib.sync_host(t) == 0
            assert lib.last_error(t) == 0
            return g, lib.grid_view(t).copy(), log
        finally:
            lib.le_free_task(t)

    a = sequence(two)
    b = sequence(2)
    assert a[0].tobytes() == b[0].tobytes()
    assert a[1].tobytes() == b[1].tobytes()
    # the FP64 energy is a sum in atomic order (equal to ~1e-15), the simulated time exact
    assert abs(a[2][0] - b[2][0]) <= 1e-12 * abs(b[2][0])
    assert a[2][1] == b[2][1]

"""The CPU oracle (oracle/le2d_oracle.c) against the reference's own outputs.

Pins the restatement bit for bit to the golden fixtures produced by running the
reference's simple/ build (tests/golden/make_golden.py), and, when oracle/_ref
was built from the reference sources, against the reference run live.
"""
import hashlib
import os
import tempfile

import numpy as np
import pytest

from golden_cases import arrays, cases, summary
from oracle.oracle import ST_AOS, ST_SOA, Oracle, Reference, ReferenceTiling, aos_to_soa, fields, rel_l2

PRECS = ("f", "d")


@pytest.mark.parametrize("prec", PRECS)
def test_material_bitwise(prec):
    o = Oracle(prec)
    a = arrays(prec)
    for (c1, c2, rho), want in zip(a["materials_in"], a["materials_out"]):
        got = o.material(c1, c2, rho)
        assert got.tobytes() == want.tobytes()


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("name", sorted(cases()))
def test_initial_state_bitwise(prec, name):
    c = cases()[name]
    o = Oracle(prec)
    a = arrays(prec)
    g = np.zeros(5 * c["nx"] * c["ny"], o.dtype)
    for cx, cy, r, s in c["disks"]:
        o.set_ball(g, c["nx"], c["ny"], c["hx"], c["hy"], c["stype"], cx, cy, r, s)
    want = a[f"{name}__in"].copy()
    # the fixture adds noise to vx, vy after the disks; compare the stress planes
    fg = fields(g, c["nx"], c["ny"], c["stype"])
    fw = fields(want, c["nx"], c["ny"], c["stype"])
    assert fg[2:].tobytes() == fw[2:].tobytes()
    if c["noise"] == 0.0:
        assert fg.tobytes() == fw.tobytes()


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("name", sorted(cases()))
def test_step_bitwise(prec, name):
    c = cases()[name]
    o = Oracle(prec)
    a = arrays(prec)
    g = a[f"{name}__in"].copy()
    o.run(g, c["nx"], c["ny"], c["dt"], c["hx"], c["hy"], c["c1"], c["c2"], c["rho"], c["stype"], c["steps"])
    assert g.tobytes() == a[f"{name}__out"].tobytes()


@pytest.mark.parametrize("prec", PRECS)
def test_soa_equals_aos(prec):
    c = cases()["ball_64x48"]
    o = Oracle(prec)
    a = arrays(prec)
    g = a["ball_64x48__in"].copy()
    s = aos_to_soa(g, c["nx"], c["ny"])
    o.run(g, c["nx"], c["ny"], c["dt"], c["hx"], c["hy"], c["c1"], c["c2"], c["rho"], ST_AOS, 7)
    o.run(s, c["nx"], c["ny"], c["dt"], c["hx"], c["hy"], c["c1"], c["c2"], c["rho"], ST_SOA, 7)
    assert aos_to_soa(g, c["nx"], c["ny"]).tobytes() == s.tobytes()


@pytest.mark.parametrize("prec", PRECS)
def test_vtk_bytes(prec):
    c = cases()["ball_64x48"]
    o = Oracle(prec)
    a = arrays(prec)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "o.vtk")
        assert o.save_vtk(a["ball_64x48__out"], c["nx"], c["ny"], c["hx"], c["hy"], c["stype"], p) == 0
        assert open(p, "rb").read() == a["ball_64x48__vtk"].tobytes()


def test_float_vs_double_gap():
    """The reference's own float build sits ~5e-7 relative L2 from its double build."""
    c = cases()["ball_64x48"]
    f = arrays("f")["ball_64x48__out"]
    d = arrays("d")["ball_64x48__out"]
    err = rel_l2(fields(f, c["nx"], c["ny"], 1), fields(d, c["nx"], c["ny"], 1))
    assert np.all(err < 1e-5)


@pytest.mark.slow
@pytest.mark.parametrize("prec", PRECS)
def test_plain_512_digest(prec):
    """The full plain 512x512 x 200-step workload: oracle bytes hash to the reference's."""
    o = Oracle(prec)
    nx = ny = 512
    g = np.zeros(5 * nx * ny, o.dtype)
    o.set_ball(g, nx, ny, 1.0, 1.0, ST_AOS, 256.0, 256.0, 25.0, 1.0)
    o.run(g, nx, ny, 0.25, 1.0, 1.0, 2.0, 1.0, 1.0, ST_AOS, 200)
    assert hashlib.sha256(g.tobytes()).hexdigest() == summary()["plain_512"][prec]["sha256"]


@pytest.mark.skipif(not Reference.available("d"), reason="oracle/_ref not built")
@pytest.mark.parametrize("prec", PRECS)
def test_live_reference_random_cases(prec):
    """Random small cases against the reference run live (when oracle/_ref exists)."""
    o = Oracle(prec)
    ref = Reference(prec)
    rng = np.random.default_rng(123)
    for _ in range(6):
        nx, ny = int(rng.integers(3, 70)), int(rng.integers(3, 70))
        stype = int(rng.integers(0, 2))
        hx, hy = float(rng.uniform(0.5, 1.5)), float(rng.uniform(0.5, 1.5))
        c1 = float(rng.uniform(1, 4))
        c2 = c1 * float(rng.uniform(0.3, 0.6))
        rho = float(rng.uniform(1, 3))
        dt = 0.45 * min(hx, hy) / c1
        disks = [(float(rng.uniform(0, nx * hx)), float(rng.uniform(0, ny * hy)), float(rng.uniform(1, 10)),
                  float(rng.uniform(-2, 2))) for _ in range(3)]
        g0 = ref.initial_state(nx, ny, hx, hy, stype, disks)
        g1 = np.zeros_like(g0)
        for d in disks:
            o.set_ball(g1, nx, ny, hx, hy, stype, *d)
        assert g0.tobytes() == g1.tobytes()
        g0 += rng.uniform(-1e-3, 1e-3, size=g0.shape).astype(g0.dtype)
        g1 = g0.copy()
        steps = int(rng.integers(1, 30))
        ref.run(g0, nx, ny, dt, hx, hy, c1, c2, rho, stype, steps, threads=2)
        o.run(g1, nx, ny, dt, hx, hy, c1, c2, rho, stype, steps)
        assert g0.tobytes() == g1.tobytes()


@pytest.mark.skipif(not ReferenceTiling.available("d"), reason="oracle/_ref not built")
@pytest.mark.parametrize("prec", PRECS)
def test_tiling_schedule_matches_away_from_the_edges(prec):
    """The reference's two-buffer schedule (tiling/ le_step_all2: zero ring of two nodes
    around the grid, increments associated (v + d1) + d2) against the restatement of simple/
    on the nodes its ends cannot reach after s steps (2 per step from each edge): the same
    scheme with other roundings -- FP64 within 1e-12, FP32 within 1e-5 relative L2."""
    o, t = Oracle(prec), ReferenceTiling(prec)
    nx, ny, steps = 96, 80, 6
    rng = np.random.default_rng(11)
    g = np.zeros(5 * nx * ny, o.dtype)
    for _ in range(3):
        o.set_ball(g, nx, ny, 1.0, 0.9, ST_AOS, float(rng.uniform(20, 76)), float(rng.uniform(20, 60)),
                   float(rng.uniform(5, 15)), float(rng.uniform(-2, 2)))
    g[0::5] += rng.uniform(-1e-3, 1e-3, nx * ny).astype(o.dtype)
    a, b = g.copy(), g.copy()
    o.run(a, nx, ny, 0.17, 1.0, 0.9, 2.3, 1.2, 1.6, ST_AOS, steps)
    t.run(b, nx, ny, 0.17, 1.0, 0.9, 2.3, 1.2, 1.6, steps)
    m = 2 * steps
    fa = fields(a, nx, ny, ST_AOS)[:, m:ny - m, m:nx - m]
    fb = fields(b, nx, ny, ST_AOS)[:, m:ny - m, m:nx - m]
    err = rel_l2(fa, fb)
    assert np.all(err <= (1e-12 if prec == "d" else 1e-5)), err
    assert not np.array_equal(a, b)  # the ends differ (zero ring against clamped)

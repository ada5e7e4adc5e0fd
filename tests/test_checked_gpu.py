"""The bounds-checked build (le2d_b200/lib/checked/, compiled with LE2D_CHECK): every access
of the state by the step kernels checks that it stays inside the buffer it addresses, and
is skipped and counted when it does not.  Memory checkers cannot run on these machines; this
build stands in for one.  Grids of odd sizes around the strip width and the segment length,
every kernel variant with short segments, both storage layouts, batched instances with
receiver lines and row slabs run in it: no access may be refused, and every result must
equal, bit for bit, the normal build's."""
import numpy as np
import pytest

from le2d_b200 import capi, workloads
from oracle.oracle import ST_AOS, ST_SOA

from test_batch_gpu import small_set

pytestmark = pytest.mark.gpu

SIZES = ((3, 3), (5, 4), (9, 7), (57, 3), (111, 20), (113, 17), (130, 64), (225, 9), (301, 37))


def _run(lib, nx, ny, stype, var, seg, g0, steps):
    mat = lib.le_init_material(2.0, 1.1, 1.3)
    t = lib.le_init_task(0.2, (1.0, 0.9), mat, (nx, ny), stype)
    try:
        assert lib.set_variant(t, var, seg) == 0
        assert lib.upload(t, g0) == 0
        assert lib.step_n(t, steps) == 0
        out = np.zeros_like(g0)
        assert lib.download(t, out) == 0 and lib.last_error(t) == 0
        return out
    finally:
        lib.le_free_task(t)


@pytest.mark.parametrize("prec", ["f", "d"])
def test_checked_build_single_solves(prec):
    lib, chk = capi.Lib(prec), capi.Lib(prec, checked=True)
    assert lib.check_violations() == (False, 0)
    assert chk.check_violations()[0]
    rng = np.random.default_rng(21)
    nvar = 0
    while True:
        c = dict(nx=8, ny=8)
        mat = lib.le_init_material(2.0, 1.1, 1.3)
        t = lib.le_init_task(0.2, (1.0, 0.9), mat, (8, 8), ST_AOS)
        ok = lib.set_variant(t, nvar, 0) == 0
        lib.le_free_task(t)
        if not ok:
            break
        nvar += 1
    for nx, ny in SIZES:
        g0 = rng.uniform(-1, 1, 5 * nx * ny).astype(lib.dtype)
        for var in range(nvar):
            for seg in (0, 3):
                for stype in (ST_AOS, ST_SOA):
                    want = _run(lib, nx, ny, stype, var, seg, g0, 5)
                    got = _run(chk, nx, ny, stype, var, seg, g0, 5)
                    assert got.tobytes() == want.tobytes(), (prec, nx, ny, var, seg, stype)
        assert chk.check_violations() == (True, 0), (prec, nx, ny)


@pytest.mark.parametrize("prec", ["f", "d"])
def test_checked_build_batches_and_slabs(prec):
    lib, chk = capi.Lib(prec), capi.Lib(prec, checked=True)
    probs = small_set(44, 10, 5, 300, 5, 40)
    stypes = [ST_SOA if k % 3 == 0 else ST_AOS for k in range(len(probs))]
    res = {}
    for name, L in (("normal", lib), ("checked", chk)):
        with capi.Batch(L, 1 << 30) as b:
            ids = [b.add(b.problem(p, st, receiver_row=p.ny // 3, receiver_every=3), disks=p.disks)
                   for p, st in zip(probs, stypes)]
            assert b.run(window_steps=7)[0] == 0
            res[name] = [(b.fields(i).tobytes(), b.receivers(i).tobytes()) for i in ids]
    assert res["checked"] == res["normal"]
    assert chk.check_violations() == (True, 0)
    c = dict(nx=300, ny=90)
    g0 = np.random.default_rng(5).uniform(-1, 1, 5 * c["nx"] * c["ny"]).astype(lib.dtype)
    outs = {}
    for name, L in (("normal", lib), ("checked", chk)):
        mat = L.le_init_material(2.3, 1.2, 1.6)
        t = L.le_init_task(0.17, (1.0, 0.9), mat, (c["nx"], c["ny"]), ST_AOS)
        try:
            with capi.Slabs(L, t, [0, 0, 0]) as s:
                assert s.upload(g0) == 0 and s.step_n(9) == 0
                outs[name] = s.download()
        finally:
            L.le_free_task(t)
    assert outs["checked"].tobytes() == outs["normal"].tobytes()
    assert chk.check_violations() == (True, 0)

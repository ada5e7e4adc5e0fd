"""Fused launches in halves (le2d_api.cu, halves_launch): each launch cut into the band of
rows around the middle of the grid and the rows above and below it, on three streams that
wait for each other only where the stencils meet.  The results must be bitwise those of
whole launches.  The cut is chosen per process (LE2D_HALVES: 1 = on every grid of at least
16 rows, 0 = never), so each setting runs in a subprocess on the same seeded states."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CASES = [(64, 37, 5), (200, 300, 70), (513, 257, 131), (97, 1000, 2), (1000, 1000, 65), (300, 16, 9)]

SCRIPT = r"""
import json, sys
import numpy as np
from le2d_b200 import capi
out = {}
for prec in ("f", "d"):
    lib = capi.Lib(prec)
    for nx, ny, steps in json.loads(sys.argv[1]):
        rng = np.random.default_rng(nx * 7 + ny)
        g = (rng.standard_normal(5 * nx * ny) * rng.choice([0.0, 1e-3, 1.0], 5 * nx * ny)).astype(lib.dtype)
        mat = lib.le_init_material(2.1, 1.1, 1.3)
        t = lib.le_init_task(0.2, (1.0, 0.9), mat, (nx, ny), capi.ST_AOS)
        try:
            assert lib.upload(t, g) == 0
            assert lib.step_n(t, steps) == 0
            got = np.zeros_like(g)
            assert lib.download(t, got) == 0
            assert lib.last_error(t) == 0
        finally:
            lib.le_free_task(t)
        out[f"{prec}/{nx}x{ny}/{steps}"] = got.tobytes().hex()
print(json.dumps(out))
"""


def _run(halves: str) -> dict:
    env = dict(os.environ, LE2D_HALVES=halves, PYTHONPATH=ROOT)
    r = subprocess.run([sys.executable, "-c", SCRIPT, json.dumps(CASES)], env=env, cwd=ROOT,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_halves_equal_whole_launches():
    whole, halves = _run("0"), _run("1")
    assert whole.keys() == halves.keys()
    for key in whole:
        assert halves[key] == whole[key], key
    # the cases changed the state (the comparison is not of untouched inputs)
    k = f"f/{CASES[1][0]}x{CASES[1][1]}/{CASES[1][2]}"
    assert np.any(np.frombuffer(bytes.fromhex(whole[k]), np.float32) != 0)

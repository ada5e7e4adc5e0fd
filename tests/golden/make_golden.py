"""Generate the golden fixtures in tests/golden/ by running the reference solver itself.

Runs the reference's own ``simple/le_core.c`` (built unmodified into
``oracle/_ref/libref_simple_{f,d}.so`` by ``oracle/Makefile`` from the reference
sources) through its task API: ``le_init_material``, ``le_init_task``,
``le_set_ball``, ``le_step`` / ``le_step_soa`` and ``le_save_task``.  Each case stores
its parameters, the initial state the reference built, and the state after the
stated number of steps, for the float and the double build.

Usage (needs the reference sources, so it runs only where they are mounted):
    make -C oracle REF=/path/to/reference && python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import ST_AOS, ST_SOA, Reference  # noqa: E402

# name: (nx, ny, hx, hy, c1, c2, rho, dt, steps, stype, disks, noise, seed)
CASES = {
    "ball_64x48": (64, 48, 1.0, 1.0, 2.0, 1.0, 1.0, 0.25, 40, ST_AOS, [(32.0, 24.0, 10.0, 1.0)], 0.0, 11),
    "disks_noise_37x53": (37, 53, 1.0, 0.75, 3.0, 1.7, 2.5, 0.125, 25, ST_AOS,
                          [(10.0, 12.0, 6.0, 1.5), (25.0, 30.0, 9.0, -0.75), (18.0, 20.0, 4.0, 2.0)], 1e-3, 12),
    "tiny_3x3": (3, 3, 1.0, 1.0, 2.0, 1.0, 1.0, 0.25, 10, ST_AOS, [(1.0, 1.0, 1.5, 1.0)], 0.0, 13),
    "tiny_3x7": (3, 7, 1.0, 1.0, 2.0, 1.2, 1.5, 0.2, 12, ST_AOS, [(1.0, 3.0, 2.0, -1.0)], 1e-3, 14),
    "tiny_7x3": (7, 3, 1.0, 1.0, 2.0, 0.8, 1.5, 0.2, 12, ST_AOS, [(3.0, 1.0, 2.0, 1.0)], 1e-3, 15),
    "soa_40x32": (40, 32, 1.0, 1.0, 2.0, 1.0, 1.5, 0.3, 30, ST_SOA, [(20.0, 16.0, 7.0, 1.0)], 0.0, 16),
    "wide_129x17": (129, 17, 1.0, 1.0, 3.0, 1.7, 2.5, 0.5 / 3.0, 20, ST_AOS,
                    [(60.0, 8.0, 6.0, 1.0), (121.0, 9.0, 5.0, -2.0)], 1e-3, 17),
    "tall_17x300": (17, 300, 1.0, 1.0, 2.0, 1.0, 1.0, 0.25, 20, ST_AOS, [(8.0, 150.0, 6.0, 1.0)], 0.0, 18),
    "strips_250x40": (250, 40, 0.5, 1.0, 2.0, 1.1, 1.0, 0.125, 15, ST_AOS,
                      [(30.0, 10.0, 4.0, 1.0), (62.0, 30.0, 5.0, -1.0), (119.5, 20.0, 3.0, 0.6)], 1e-3, 19),
}

MATERIALS = [(2.0, 1.0, 1.0), (3.0, 1.7, 2.5), (2.0, 1.0, 1.5), (1.3, 0.5, 2.9), (4.0, 2.3, 1.1)]


def initial_state(ref: Reference, case) -> np.ndarray:
    nx, ny, hx, hy, c1, c2, rho, dt, steps, stype, disks, noise, seed = case
    g = ref.initial_state(nx, ny, hx, hy, stype, disks)
    if noise > 0.0:
        rng = np.random.default_rng(seed)
        vx = rng.uniform(-noise, noise, size=(ny, nx)).astype(ref.dtype)
        vy = rng.uniform(-noise, noise, size=(ny, nx)).astype(ref.dtype)
        if stype == ST_AOS:
            a = g.reshape(ny, nx, 5)
            a[:, :, 0] = vx
            a[:, :, 1] = vy
        else:
            a = g.reshape(5, ny, nx)
            a[0] = vx
            a[1] = vy
    return g


def main() -> None:
    summary = {"cases": {}, "materials": {}, "plain_512": {}}
    for prec in ("f", "d"):
        ref = Reference(prec)
        mats = np.stack([ref.material(*m) for m in MATERIALS])
        summary["materials"][prec] = mats.astype(np.float64).tolist()
        arrays = {"materials_in": np.asarray(MATERIALS, np.float64), "materials_out": mats}
        for name, case in CASES.items():
            nx, ny, hx, hy, c1, c2, rho, dt, steps, stype, disks, noise, seed = case
            g0 = initial_state(ref, case)
            g = g0.copy()
            ref.run(g, nx, ny, dt, hx, hy, c1, c2, rho, stype, steps, threads=1)
            arrays[f"{name}__in"] = g0
            arrays[f"{name}__out"] = g
            summary["cases"][name] = {
                "nx": nx, "ny": ny, "hx": hx, "hy": hy, "c1": c1, "c2": c2, "rho": rho, "dt": dt,
                "steps": steps, "stype": stype, "disks": disks, "noise": noise, "seed": seed,
            }
        # VTK bytes of the first case's final state (le_save_task).
        c = CASES["ball_64x48"]
        with tempfile.TemporaryDirectory() as td:
            p = os.path.join(td, "r.vtk")
            assert ref.save_vtk(arrays["ball_64x48__out"], c[0], c[1], c[2], c[3], c[9], p) == 0
            arrays["ball_64x48__vtk"] = np.frombuffer(open(p, "rb").read(), np.uint8)
        np.savez_compressed(os.path.join(HERE, f"golden_{prec}.npz"), **arrays)

        # The plain 512x512 workload, 200 steps: too large to store, so keep digests.
        nx = ny = 512
        g = ref.initial_state(nx, ny, 1.0, 1.0, ST_AOS, [(256.0, 256.0, 25.0, 1.0)])
        ref.run(g, nx, ny, 0.25, 1.0, 1.0, 2.0, 1.0, 1.0, ST_AOS, 200, threads=0)
        f = g.reshape(ny, nx, 5).astype(np.float64)
        summary["plain_512"][prec] = {
            "sha256": hashlib.sha256(g.tobytes()).hexdigest(),
            "sumsq": [float((f[:, :, k] ** 2).sum()) for k in range(5)],
            "sum": [float(f[:, :, k].sum()) for k in range(5)],
        }
    with open(os.path.join(HERE, "golden.json"), "w") as fh:
        json.dump(summary, fh, indent=1)
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    main()

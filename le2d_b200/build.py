"""Build lible2d_f.so and lible2d_d.so (sm_100a) in-tree with nvcc.

    python -m le2d_b200.build            # both precisions
    python -m le2d_b200.build --verbose  # also print ptxas register / spill reports

Objects go to le2d_b200/_build/, libraries to le2d_b200/lib/, and the bounds-checked build
(LE2D_CHECK: every state access of the step kernels checked and counted, for tests) to
le2d_b200/lib/checked/.  The host compiler
runs with -ffp-contract=off so the host-side material and initial-condition
arithmetic rounds like the reference build (x86-64 baseline, no FMA).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "lib")
INCLUDE = os.path.join(ROOT, "include")

SOURCES = ["le2d_api.cu", "step_fused.cu", "step_split.cu", "layout.cu", "diag.cu", "batch.cu", "engine.cu",
           "serve.cu", "diag_noalloc.cu", "slabs.cu", "selftest.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _flags(prec: str) -> list[str]:
    f = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
                "-I", INCLUDE, "-I", CSRC]
    if prec.startswith("d"):
        f += ["-DUSE_DOUBLE"]
    if prec.endswith("_check"):
        f += ["-DLE2D_CHECK"]
    return f


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return hs + [os.path.abspath(__file__)]


def _compile(prec: str, src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, prec, src.replace(".cu", ".o"))
    os.makedirs(os.path.dirname(obj), exist_ok=True)
    srcp = os.path.join(CSRC, src)
    if not _newer(obj, [srcp] + _deps()):
        return obj
    cmd = [nvcc(), "-c", srcp, "-o", obj] + _flags(prec)
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src} ({prec}):\n{r.stderr}")
    if verbose and r.stderr:
        sys.stderr.write(f"--- {src} [{prec}]\n{r.stderr}")
    return obj


def build(verbose: bool = False, precs=("f", "d"), checked: bool = True) -> list[str]:
    """The libraries of each precision; with `checked` also the bounds-checked build
    (LE2D_CHECK) under lib/checked/."""
    os.makedirs(LIBDIR, exist_ok=True)
    variants = list(precs) + ([p + "_check" for p in precs] if checked else [])
    out = []
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        futs = {(p, s): ex.submit(_compile, p, s, verbose) for p in variants for s in SOURCES}
        objs = {k: f.result() for k, f in futs.items()}
    for p in variants:
        if p.endswith("_check"):
            os.makedirs(os.path.join(LIBDIR, "checked"), exist_ok=True)
            lib = os.path.join(LIBDIR, "checked", f"lible2d_{p[:-6]}.so")
        else:
            lib = os.path.join(LIBDIR, f"lible2d_{p}.so")
        pobjs = [objs[(p, s)] for s in SOURCES]
        if _newer(lib, pobjs):
            cmd = [nvcc(), "-shared", "-o", lib] + pobjs + ARCH + ["-Xlinker", "-z,defs"]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"link failed ({p}):\n{r.stderr}")
        out.append(lib)
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    if a.force and os.path.exists(BUILD):
        shutil.rmtree(BUILD)
    for lib in build(a.verbose):
        print(lib)


if __name__ == "__main__":
    main()

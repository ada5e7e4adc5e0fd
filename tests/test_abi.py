"""The C-ABI boundary on the CPU: the libraries load, export every function the
headers declare, keep the reference's struct layouts, and a C host written against
the reference (its own simple/main.c) compiles and links against them unchanged."""
import ctypes
import os
import re
import subprocess
import tempfile

import pytest

from le2d_b200 import capi
from oracle.oracle import REFERENCE_ROOT

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")
REF = REFERENCE_ROOT


def header_functions():
    names = set()
    for h in os.listdir(INCLUDE):
        if not h.endswith(".h"):
            continue
        src = open(os.path.join(INCLUDE, h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"static __inline__[^{]*\{.*?\n\}", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(le\w+)\s*\([^;{]*\)\s*;", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_header_declares_reference_api():
    names = header_functions()
    for f in ["le_init_material", "le_init_task", "le_free_task", "le_set_ball", "le_save_task",
              "le_step", "le_step_soa"]:
        assert f in names
    assert "le_step_cf" not in names  # declared by the reference but defined nowhere
    assert names == set(capi.EXPORTS), names ^ set(capi.EXPORTS)


@pytest.mark.parametrize("prec", ["f", "d"])
def test_library_exports_every_declared_function(prec):
    path = capi.lib_path(prec)
    assert os.path.exists(path), "run python -m le2d_b200.build"
    lib = ctypes.CDLL(path)
    for name in header_functions():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert header_functions() <= exported


LAYOUT_PROBE = r"""
#include <stdio.h>
#include <stddef.h>
#include "le_core.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(le_task), sizeof(le_material),
         sizeof(le_vec2), sizeof(le_point2), sizeof(le_node), offsetof(le_task, h), offsetof(le_task, n),
         offsetof(le_task, mat), offsetof(le_task, stype), offsetof(le_task, grid));
  return 0;
}
"""


@pytest.mark.parametrize("double", [False, True])
def test_struct_layout_matches_reference(double):
    ours = _probe(INCLUDE, double)
    if os.path.exists(os.path.join(REF, "simple", "le_core.h")):
        assert ours == _probe(os.path.join(REF, "simple"), double)
    # independent of the reference: float  -> dt@0 h@4 n@12 mat@20 stype@52 grid@56, size 64
    #                                double -> dt@0 h@8 n@24 mat@32 stype@96 grid@104, size 112
    want = [64, 32, 8, 8, 20, 4, 12, 20, 52, 56] if not double else [112, 64, 16, 8, 40, 8, 24, 32, 96, 104]
    assert ours == want


def _probe(incdir, double):
    with tempfile.TemporaryDirectory() as td:
        c = os.path.join(td, "p.c")
        open(c, "w").write(LAYOUT_PROBE)
        exe = os.path.join(td, "p")
        cmd = ["gcc", "-I", incdir, c, "-o", exe] + (["-DUSE_DOUBLE"] if double else [])
        subprocess.run(cmd, check=True, capture_output=True)
        return [int(x) for x in subprocess.run([exe], capture_output=True, text=True).stdout.split()]


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "simple", "main.c")), reason="reference absent")
@pytest.mark.parametrize("prec", ["f", "d"])
def test_reference_driver_links_unchanged(prec):
    """The reference's own CLI driver compiles against include/le_core.h and links."""
    with tempfile.TemporaryDirectory() as td:
        exe = os.path.join(td, "simple_main")
        cmd = ["gcc", "-O2", "-fopenmp", "-I", INCLUDE, os.path.join(REF, "simple", "main.c"), "-o", exe,
               capi.lib_path(prec), "-lm", "-w"] + (["-DUSE_DOUBLE"] if prec == "d" else [])
        r = subprocess.run(cmd, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr

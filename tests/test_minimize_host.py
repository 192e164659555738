"""The product's minimiser (smmp-svn_b200/csrc/minimize.cpp: BFGS for
imin = 1, Polak-Ribiere+ conjugate gradients for imin = 2, the role of
minim.f:13) run on the CPU over the oracle's energy and gradient from the
README's Met-enkephalin start: both reach the published minimum
(README:482-513, total -12.43 kcal/mol and the listed dihedrals).  The GPU
test of smmp.minim runs the same minimiser over the GPU gradient."""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import DATA, ORACLE_SO, ROOT, Oracle

SRC = os.path.join(ROOT, "smmp-svn_b200", "csrc")
BUILD = os.path.join(ROOT, "tests", "_build")
HARNESS = os.path.join(BUILD, "minimize_host_check")
CRD = 57.2957795130823


@pytest.fixture(scope="module")
def harness():
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("g++ not found")
    Oracle.lib()
    os.makedirs(BUILD, exist_ok=True)
    odir = os.path.dirname(ORACLE_SO)
    subprocess.check_call(
        [gxx, "-std=c++17", "-O2", "-I" + SRC, os.path.join(ROOT, "tests", "minimize_host_check.cpp"),
         os.path.join(SRC, "minimize.cpp"), "-o", HARNESS, "-L" + odir, "-loracle_smmp",
         "-Wl,-rpath," + odir])
    return HARNESS


@pytest.mark.parametrize("imin", [1, 2])
def test_minimiser_reaches_the_published_minimum(harness, imin):
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        gold = json.load(f)["minim_enkefa"]
    out = subprocess.run([harness, DATA, DATA + "enkefa.seq", DATA + "enkefa.var", str(imin)],
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    lines = out.stdout.split("\n")
    calls, energy, grad2, converged = lines[0].split()
    assert int(converged) == 1 and int(calls) < 10000
    assert float(grad2) <= 1e-9
    assert abs(float(energy) - gold["total"]) <= 5e-3, energy
    v = np.array([float(x) for x in lines[1:] if x.strip()]) * CRD
    v = (v + 180.0) % 360.0 - 180.0
    want = np.array([w[2] for w in gold["variables"]])
    d = (v - want + 180.0) % 360.0 - 180.0
    assert np.all(np.abs(d) <= 0.051), np.c_[v, want]

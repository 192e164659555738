"""The analytic SASA kernel's per-atom arithmetic, compiled for the host, equals
the oracle's restatement of esolan.f bit for bit (CPU test: needs nvcc, no
GPU).  The harness is tests/esolan_host_check.cu; the GPU tests compare the
kernel's results on the device (tests/test_gpu_esolan.py)."""
import os
import shutil
import subprocess

import pytest

from conftest import DATA, ORACLE_SO, ROOT, Oracle, seqfile

HARNESS_SRC = os.path.join(ROOT, "tests", "esolan_host_check.cu")
BUILD = os.path.join(ROOT, "tests", "_build")
HARNESS = os.path.join(BUILD, "esolan_host_check")


@pytest.fixture(scope="module")
def harness():
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    Oracle.lib()   # builds the oracle library if needed
    os.makedirs(BUILD, exist_ok=True)
    oracle_dir = os.path.dirname(ORACLE_SO)
    subprocess.check_call([
        nvcc, "-std=c++17", "-O2", "-fmad=false", "-x", "cu",
        "-I" + os.path.join(ROOT, "smmp-svn_b200", "csrc"), "-I" + os.path.join(ROOT, "include"),
        "-I" + oracle_dir, HARNESS_SRC, "-o", HARNESS,
        "-L" + oracle_dir, "-loracle_smmp", "-Xlinker", "-rpath", "-Xlinker", oracle_dir])
    return HARNESS


def _run(harness, *args):
    out = subprocess.run([harness, DATA] + list(args), capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "OK deferred 0 mismatches 0" in out.stdout, out.stdout
    return out.stdout


def test_kernel_arithmetic_equals_oracle_enkefa(harness):
    _run(harness, DATA + "enkefa.seq", DATA + "enkefa.var")


def test_kernel_arithmetic_equals_oracle_protein60(harness, tmp_path):
    from smmp.sequences import natural_protein
    s = seqfile(tmp_path, natural_protein(60), "protein60")
    _run(harness, s)

"""The gradient arithmetic meant for the GPU (smmp-svn_b200/csrc/
gradient_core.cuh: atomic forces from the product's pair lists, derivatives
from sums over each variable's contiguous atom range), compiled for the host
over the product's own host topology, equals the oracle's gradient.f /
opeshe.f on the oracle's coordinates (CPU test: needs nvcc, no GPU).  The
harness is tests/gradient_host_check.cu."""
import os
import shutil
import subprocess

import pytest

from conftest import DATA, ORACLE_SO, ROOT, Oracle, seqfile

SRC = os.path.join(ROOT, "smmp-svn_b200", "csrc")
BUILD = os.path.join(ROOT, "tests", "_build")
HARNESS = os.path.join(BUILD, "gradient_host_check")


@pytest.fixture(scope="module")
def harness():
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not found")
    Oracle.lib()
    os.makedirs(BUILD, exist_ok=True)
    odir = os.path.dirname(ORACLE_SO)
    subprocess.check_call(
        [nvcc, "-std=c++17", "-O2", "-Xcompiler", "-ffp-contract=off", "-I" + SRC,
         "-I" + os.path.join(ROOT, "include"), "-x", "cu",
         os.path.join(ROOT, "tests", "gradient_host_check.cu"), "-x", "c++"] +
        [os.path.join(SRC, f) for f in ("molbuild.cpp", "ecepp.cpp", "topology.cpp")] +
        ["-o", HARNESS, "-L" + odir, "-loracle_smmp", "-Xlinker", "-rpath", "-Xlinker", odir])
    return HARNESS


def _run(harness, *args):
    out = subprocess.run([harness, DATA] + list(args), capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip().splitlines()[-1].startswith("OK"), out.stdout


def test_gradient_core_enkefa(harness):
    _run(harness, DATA + "enkefa.seq", DATA + "enkefa.var")


def test_gradient_core_ecepp2(harness):
    """ECEPP/2 tables and charges (lib.sh2)."""
    _run(harness, DATA + "enkefa.seq", DATA + "enkefa.var", "1", "0")


def test_gradient_core_sigmoidal_dielectric(harness):
    """The distance-dependent dielectric (gradient_pair's epsd branch)."""
    _run(harness, DATA + "enkefa.seq", DATA + "enkefa.var", "0", "1")


def test_gradient_core_protein60(harness, tmp_path):
    from smmp.sequences import natural_protein
    _run(harness, seqfile(tmp_path, natural_protein(60), "p60"))

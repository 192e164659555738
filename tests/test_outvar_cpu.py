"""outvar (outvar.f:12-121) on the CPU: the text of the final conformation of
the reference's annealing run (EXAMPLES/annealing.out:20-43) reproduced line
for line, and a round trip through the .var reader."""
import json
import os

import numpy as np

from conftest import DATA, ROOT

CRD = 57.2957795130823   # INCL.H:41


def _golden():
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        return json.load(f)["anneal_outvar"]


def _molecule(var=None):
    from smmp.ensemble import Molecule
    return Molecule(DATA + "enkefa.seq", var or DATA + "enkefa.ann", libdir=DATA, ff="ecepp2")


def test_outvar_reproduces_the_annealing_output():
    g = _golden()
    m = _molecule()
    deg = [float(line.split(":")[3].split()[0]) for line in g["lines"]]
    assert len(deg) == m.nvar
    text = m.outvar(np.array(deg) / CRD)
    assert text.splitlines() == g["lines"]


def test_outvar_text_reads_back(tmp_path):
    """The written variables, read by the .var reader (redvar), give the same
    values to the printed precision (angles in (-180, 180]: -180 reads back
    as 180) and the same fixed flags."""
    g = _golden()
    m = _molecule()
    deg = np.array([float(line.split(":")[3].split()[0]) for line in g["lines"]])
    p = tmp_path / "final.var"
    p.write_text(m.outvar(deg / CRD))
    back = _molecule(str(p))
    assert back.nvar == m.nvar and back.nvr == m.nvr
    assert np.array_equal(back.idvr, m.idvr)
    diff = (back.vlvr0 * CRD - deg + 180.0) % 360.0 - 180.0
    assert np.all(np.abs(diff) <= 5e-4)

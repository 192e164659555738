"""The CPU oracle against the reference's published numbers.

README:389-393 (Met-enkephalin energy and its terms) and
EXAMPLES/annealing.out:14-45 (an MT19937-driven annealing trajectory of
100,000 sweeps) pin the oracle's setup, lists, rebuild, ECEPP energy, random
numbers and Metropolis step.
"""
import json

import numpy as np
import pytest

from conftest import DATA, GOLDEN, Oracle


def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def sig(x, digits):
    return float("%.*e" % (digits - 1, x))


def test_enkefa_ecepp3_terms_match_readme():
    g = golden()["enkefa_ecepp3"]
    o = Oracle(DATA + "enkefa.seq", DATA + "enkefa.var")
    e, t = o.energy()
    assert o.natoms == 75 and o.nvr == 24
    # the README prints 5 significant digits for the total, 4 for the terms
    assert sig(e, 5) == pytest.approx(g["total"], rel=1e-12)
    assert sig(t[0], 4) == pytest.approx(g["coulomb"], rel=1e-12)
    assert sig(t[1], 4) == pytest.approx(g["lennard_jones"], rel=1e-12)
    assert sig(t[2], 4) == pytest.approx(g["hbond"], rel=1e-12)
    assert sig(t[3], 4) == pytest.approx(g["torsion"], rel=1e-12)


def _anneal(nswp):
    import ctypes
    o = Oracle(DATA + "enkefa.seq", DATA + "enkefa.ann", ff="ecepp2")
    o.sgrnd(81236)
    out = (ctypes.c_double * 6)()
    rc = o.lib().orc_anneal(o.h, 100, nswp, 1000.0, 100.0, 1, out)
    assert rc == 0
    return o, list(out)


def test_anneal_start_and_equilibration_match():
    g = golden()["anneal_ecepp2"]
    o, out = _anneal(10)
    assert o.nvr == 19                      # omega angles fixed by enkefa.ann
    assert sig(out[0], 5) == pytest.approx(g["start"], rel=1e-12)
    assert out[1] == pytest.approx(g["after_equilibration"], rel=1e-13)


@pytest.mark.slow
def test_anneal_full_trajectory_matches():
    """100,000 sweeps (1.9M proposals): identical acceptance count, same minimum."""
    g = golden()["anneal_ecepp2"]
    _, out = _anneal(100000)
    assert out[2] == pytest.approx(g["acceptance"], rel=1e-14)
    assert out[5] == g["lowest_sweep"]
    assert out[4] == pytest.approx(g["lowest"], rel=1e-11)
    assert out[3] == pytest.approx(g["last"], rel=1e-11)


def test_oracle_sasa_energy_is_finite_and_area_positive(tmp_path):
    from conftest import seqfile
    s = seqfile(tmp_path, ["ace"] + ["ala"] * 10 + ["nme"])
    o = Oracle(s, itysol=1)
    e, t = o.energy()
    assert np.isfinite(e) and t[4] != 0.0

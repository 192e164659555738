"""The oracle's restatement of minim.f / minqsn.f (quasi-Newton minimisation
with the analytic gradient) against the reference's published run
(README:389-514, EXAMPLES/minimization.f): Met-enkephalin from the deck's
conformation, ECEPP/3, eps 1e-9.  Every logged function call (energy and
squared gradient, E13.6) agrees up to step 82; in the last steps, at squared
gradients near 1e-11, round-off decides the final line search, so there the
energy still agrees and the gradient is converged.  The final energy terms
and free variables agree to the printed digits."""
import json
import math
import os

import numpy as np

from conftest import DATA, ROOT, Oracle

CRD = 57.2957795130823


def _e136(x):
    """Fortran E13.6 without the leading blanks (0.dddddd E+ee)."""
    if x == 0.0:
        return "0.000000E+00"
    e = math.floor(math.log10(abs(x))) + 1
    m = round(abs(x) / 10 ** e, 6)
    if m >= 1.0:
        m /= 10
        e += 1
    return ("-" if x < 0 else "") + "%.6fE%+03d" % (m, e)


def test_minimisation_reproduces_the_published_run():
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        g = json.load(f)["minim_enkefa"]
    o = Oracle(DATA + "enkefa.seq", DATA + "enkefa.var")
    nop, log = o.minim(1, 10000, 1e-9)
    steps = g["steps"]
    assert 85 <= nop <= 90 and len(log) == nop
    for k in range(82):
        assert [_e136(log[k][0]), _e136(log[k][1])] == steps[k], (k + 1, log[k], steps[k])
    for k in range(82, 85):
        assert _e136(log[k][0]) == steps[k][0]
    assert log[-1][1] < 1e-9
    e, t = o.energy()
    assert abs(e - g["total"]) <= 5e-3
    for key, idx in (("coulomb", 0), ("lennard_jones", 1), ("hbond", 2), ("torsion", 3)):
        assert abs(t[idx] - g[key]) <= 5e-3 * max(1.0, abs(g[key])), key
    v = o.vlvr()[o.idvr() - 1] * CRD
    want = np.array([w[2] for w in g["variables"]])
    d = (v - want + 180.0) % 360.0 - 180.0
    assert np.all(np.abs(d) <= 0.051), np.c_[v, want]


def test_conjugate_gradients_reach_the_same_minimum():
    """imin = 2 (mincjg.f) from the same start ends in the minimum the
    published quasi-Newton run found."""
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        g = json.load(f)["minim_enkefa"]
    o = Oracle(DATA + "enkefa.seq", DATA + "enkefa.var")
    nop, log = o.minim(2, 10000, 1e-9)
    assert nop < 10000 and log[-1][1] < 1e-6
    e, _ = o.energy()
    assert abs(e - g["total"]) <= 5e-3
    v = o.vlvr()[o.idvr() - 1] * CRD
    want = np.array([w[2] for w in g["variables"]])
    d = (v - want + 180.0) % 360.0 - 180.0
    assert np.all(np.abs(d) <= 0.051)

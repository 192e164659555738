"""The autotuner: it times the pair-work decompositions (pair lists, rows,
rows for molecules of 128+ atoms, rows with speculative windows of 2, 4 and 8
proposals) from a saved state, keeps the fastest, and
leaves the ensemble's state (variables, energies, random streams, counters)
exactly as it found it."""
import numpy as np
import pytest

from conftest import DATA, Oracle, seqfile

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [6, 40])
def test_autotune_leaves_no_trace_and_keeps_parity(tmp_path, n):
    from smmp.ensemble import Ensemble, Molecule, beta_of
    from smmp.sequences import polyala
    f = seqfile(tmp_path, polyala(n), "ala%d" % n)
    mol = Molecule(f, libdir=DATA)
    b = beta_of(300.0)
    ens = Ensemble([mol], [0] * 16, [40 + c for c in range(16)], [b] * 16, fp32=True)
    twin = Ensemble([mol], [0] * 16, [40 + c for c in range(16)], [b] * 16, fp32=True)
    for e in (ens, twin):
        e.random_start()
        e.sweeps(5)
    v0, e0 = ens.vlvr(), ens.energies()
    a0, p0 = ens.acceptance()
    form, ms = ens.autotune()
    assert np.array_equal(ens.vlvr(), v0) and np.array_equal(ens.energies(), e0)
    a1, p1 = ens.acceptance()
    assert np.array_equal(a0, a1) and np.array_equal(p0, p1)
    assert min(ms) > 0
    win, wms = ens.window()
    if win > 1:   # a speculative window on the row form beat every one-at-a-time form
        assert form == "rows" and wms[(2, 4, 8).index(win)] <= min(ms)
    else:
        assert form == Ensemble.AUTOTUNE_FORMS[int(np.argmin(ms))]
    # the random streams were restored: the next draws equal the twin's
    assert np.array_equal(ens.draw(3, 50), twin.draw(3, 50))
    ens.sweeps(5)
    assert not ens.errors().any()
    o = Oracle(f)
    V = ens.vlvr()
    E = ens.energies()
    for c in (0, 7, 15):
        o.set_vlvr(V[c, :o.ntlvr])
        e, _ = o.energy()
        assert abs(E[c] - e) <= max(1e-2, 1e-7 * abs(e))


def test_autotune_without_row_form_is_a_no_op():
    from smmp.ensemble import Ensemble, Molecule, beta_of
    mol = Molecule(DATA + "enkefa.seq", DATA + "enkefa.var", libdir=DATA)
    ens = Ensemble([mol], [0] * 4, [1, 2, 3, 4], [beta_of(300.0)] * 4, fp32=True)
    form, ms = ens.autotune()
    assert form in Ensemble.AUTOTUNE_FORMS

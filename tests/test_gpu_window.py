"""Speculative windows of the sweep: in the incremental mode (FP32 pair
terms, row-form pair work, relaxed states) k_sweep evaluates up to `window`
consecutive proposals at once from the same state and keeps the first
accepted one.  Each proposal draws the same numbers, is summed over the same
pairs by the same threads and decided with the same arithmetic as one at a
time, so a run with windows must leave exactly the same bits as a run
without: variables, energies, terms of the closing evaluation, acceptance
counts and the position of every chain's random stream."""
import numpy as np
import pytest

from conftest import DATA, seqfile

pytestmark = pytest.mark.gpu


def _ensemble(n, rndord=False):
    from smmp.ensemble import Ensemble, Molecule, beta_of
    mol = Molecule(DATA + "enkefa.seq", DATA + "enkefa.var", libdir=DATA)
    temps = 100.0 * 10.0 ** (np.arange(n) / max(n - 1, 1))
    ens = Ensemble([mol], [0] * n, [31433 + 1000 * k for k in range(n)],
                   [beta_of(t) for t in temps], fp32=True, rndord=rndord)
    ens.set_pair_work("rows")
    ens.set_window(1)
    ens.random_start()
    ens.sweeps(40)                 # out of the clash regime of the random start
    assert np.all(np.abs(ens.energies()) < 1e4)
    return ens


def _state(ens):
    a, p = ens.acceptance()
    draws = np.array([ens.draw(c, 3) for c in range(ens.nchains)])
    return ens.vlvr().copy(), ens.energies().copy(), ens.terms().copy(), a.copy(), p.copy(), draws


def _run(ens, blob, window, nsweeps, pt=False):
    ens.restore(blob)
    assert ens.set_window(window) == window
    if pt:
        ens.pt_sweeps(nsweeps)
    else:
        ens.sweeps(nsweeps)
    assert not ens.errors().any()
    assert ens.window()[0] == window
    return _state(ens)


def _same(a, b):
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("rndord", [False, True])
def test_windows_leave_the_same_bits(rndord):
    ens = _ensemble(8, rndord)
    blob = ens.checkpoint()
    ref = _run(ens, blob, 1, 12)
    assert 0 < ref[3].sum() < ref[4].sum()      # both accepted and rejected proposals
    for k in (2, 3, 4, 8):
        _same(_run(ens, blob, k, 12), ref)


def test_fused_parallel_tempering_with_windows():
    from smmp.ensemble import beta_of
    ens = _ensemble(16)
    temps = 100.0 * 10.0 ** (np.arange(16) / 15.0)
    ens.set_pt([beta_of(t) for t in temps], wrap=False, exchange_seed=4711)
    blob = ens.checkpoint()
    ref = _run(ens, blob, 1, 10, pt=True)
    assert ens.pt_fused_last()
    map_ref = ens.pt_map().copy()
    got = _run(ens, blob, 4, 10, pt=True)
    assert ens.pt_fused_last()
    _same(got, ref)
    assert np.array_equal(ens.pt_map(), map_ref)


def test_window_size_is_capped_for_large_molecules(tmp_path):
    from smmp.ensemble import Ensemble, Molecule, beta_of
    from smmp.sequences import natural_protein
    big = Molecule(seqfile(tmp_path, natural_protein(60), "p60"), None, libdir=DATA)
    ens = Ensemble([big], [0, 0], [1, 2], [beta_of(300.0)] * 2, fp32=True)
    assert ens.set_window(8) == 1            # 926 atoms: the buffers would not fit
    small = Molecule(DATA + "enkefa.seq", None, libdir=DATA)
    ens2 = Ensemble([small], [0, 0], [1, 2], [beta_of(300.0)] * 2, fp32=True)
    assert ens2.set_window(8) == 8
    solv = Molecule(DATA + "enkefa.seq", None, libdir=DATA, itysol=1)
    ens3 = Ensemble([solv], [0, 0], [1, 2], [beta_of(300.0)] * 2, fp32=True)
    assert ens3.set_window(4) == 1           # SASA sweeps take proposals one at a time

"""Cached pair terms (list-form molecules, FP32 pair terms): the sweep keeps
every pair's term of the state, and a proposal sums only the pairs its turn
changes (the crossing lists) against them.  The chain energies, which
accumulate these changes through a sweep, stay within 1e-3 kcal/mol of the
FP64 oracle's energy of the same conformations (the FP32 bar), every sweep's
closing consistency check passes, and the pair-term counter shows that the
proposals summed the crossing pairs only."""
import numpy as np
import pytest

from conftest import DATA, Oracle

pytestmark = pytest.mark.gpu

SEQ, VAR = DATA + "enkefa.seq", DATA + "enkefa.var"


def _crossing_total(mol):
    """Pairs whose distance turning each free variable changes (one atom in
    the atoms it moves, neither atom on its axis), summed over the free
    variables: computed here from the interaction lists and the tree."""
    pairs = mol.pairs()
    parent = mol.atoms()[0]
    prim = mol.variables()[:, 0]
    total = 0
    for v in mol.idvr:
        lo, hi = mol.var_lo[v], mol.var_hi[v]
        b = parent[prim[v]]
        a = parent[b]
        i, j = pairs[:, 0], pairs[:, 1]
        off_axis = (i != a) & (i != b) & (j != a) & (j != b)
        cross = ((i >= lo) & (i <= hi)) != ((j >= lo) & (j <= hi))
        total += int(np.sum(off_axis & cross))
    return total


def test_cached_terms_track_the_fp64_energy():
    from smmp.ensemble import Ensemble, Molecule, beta_of
    mol = Molecule(SEQ, VAR, libdir=DATA)
    n = 16
    ens = Ensemble([mol], [0] * n, [101 + 7 * k for k in range(n)], [beta_of(300.0)] * n,
                   fp32=True)
    ens.set_pair_work("pair lists")
    ens.set_window(1)
    ens.sweeps(200)                      # relax the README start (a clash of 900 kcal/mol)
    p0 = ens.pair_terms().astype(np.int64)
    nsw = 20
    ens.sweeps(nsw)
    p1 = ens.pair_terms().astype(np.int64)
    assert not np.any(ens.errors())
    E = ens.energies()
    V = ens.vlvr()
    o = Oracle(SEQ, VAR)
    for c in range(n):
        o.set_vlvr(V[c, :mol.nvar])
        eo = o.energy()[0]
        assert abs(E[c] - eo) <= 1e-3, (c, E[c], eo)
    # per sweep: the opening energy, the cache fill and one crossing list per
    # proposal (variables in order; at 300 K no accepted state holds a
    # guarded pair), and once the closing energy of the call
    npairs = len(mol.pairs())
    want = nsw * (2 * npairs + _crossing_total(mol)) + npairs
    assert np.all(p1 - p0 == want), (p1 - p0, want)
    assert want < 0.5 * nsw * (len(mol.idvr) + 1) * npairs

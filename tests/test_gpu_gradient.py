"""The GPU gradient (k_gradient: gradient.f / opeshe.f in the order-free
form, FP64) against the oracle's restatement of opeshe.f and against central
differences of the GPU's own FP64 energy; the minimiser over it (minim.f's
role) from the README's Met-enkephalin start reaches the published minimum
(README:482-513: total -12.43 kcal/mol and the listed dihedrals)."""
import json
import os

import numpy as np
import pytest

from conftest import DATA, ROOT, Oracle, seqfile

pytestmark = pytest.mark.gpu

SEQ, VAR = DATA + "enkefa.seq", DATA + "enkefa.var"
CRD = 57.2957795130823


def _ens(mol, V):
    from smmp.ensemble import Ensemble, beta_of
    n = len(V)
    ens = Ensemble([mol], [0] * n, list(range(1, n + 1)), [beta_of(300.0)] * n)
    W = np.zeros((n, ens.vstride))
    W[:, :mol.nvar] = V
    ens.set_vlvr(W)
    return ens


@pytest.mark.parametrize("case", ["enkefa", "enkefa-ecepp2", "enkefa-epsd", "protein60"])
def test_gradient_matches_the_oracle(case, tmp_path):
    from smmp.ensemble import Molecule
    from smmp.sequences import natural_protein
    ff, epsd, seq, var = "ecepp3", 0, SEQ, VAR
    if case == "enkefa-ecepp2":
        ff = "ecepp2"
    if case == "enkefa-epsd":
        epsd = 1
    if case == "protein60":
        seq, var = seqfile(tmp_path, natural_protein(60), "p60"), None
    mol = Molecule(seq, var, libdir=DATA, ff=ff, epsd=epsd)
    o = Oracle(seq, var, ff=ff, epsd=epsd)
    rng = np.random.default_rng(5)
    V = np.tile(mol.vlvr0, (4, 1))
    V[1:, mol.idvr] += rng.uniform(-0.15, 0.15, (3, len(mol.idvr)))
    g, e = _ens(mol, V).gradient()
    for c in range(4):
        o.set_vlvr(V[c])
        eo, go = o.gradient()
        scale = max(1.0, np.abs(go).max())
        assert np.abs(g[c, :mol.nvar] - go).max() <= 1e-9 * scale, (case, c)
        assert e[c] == pytest.approx(eo, rel=1e-10, abs=1e-9)


def test_gradient_equals_central_differences(tmp_path):
    """protein60, relaxed first: the residue-template start has clashing
    side chains (E ~ 3e8 kcal/mol), where the FP64 energy differences of a
    central difference are rounding noise."""
    import smmp
    from smmp.ensemble import Molecule
    from smmp.sequences import natural_protein
    seq = seqfile(tmp_path, natural_protein(60), "p60")
    smmp.reset()
    smmp.epar_l.sh2 = 0
    smmp.isolty.itysol = 0
    smmp.init_energy(DATA)
    smmp.init_molecule(1, "nh2", "cooh", seq)
    smmp.minim(1, 300, 1e-9)
    v0 = np.asarray(smmp.var_r.vlvr).copy()
    smmp.reset()
    mol = Molecule(seq, None, libdir=DATA)
    assert len(v0) == mol.nvar
    rng = np.random.default_rng(11)
    v0[mol.idvr] += rng.uniform(-0.02, 0.02, len(mol.idvr))
    g, e = _ens(mol, v0[None, :]).gradient()
    assert abs(e[0]) < 1e5, e[0]
    h = 1e-6
    picks = mol.idvr[rng.choice(len(mol.idvr), 12, replace=False)]
    V = np.tile(v0, (2 * len(picks), 1))
    for k, v in enumerate(picks):
        V[2 * k, v] += h
        V[2 * k + 1, v] -= h
    ens = _ens(mol, V)
    E = ens.energy()
    for k, v in enumerate(picks):
        fd = (E[2 * k] - E[2 * k + 1]) / (2 * h)
        assert abs(fd - g[0, v]) <= 1e-5 * max(1.0, abs(g[0, v])), (v, fd, g[0, v])


@pytest.mark.parametrize("imin", [1, 2])
def test_minim_reaches_the_published_minimum(imin):
    import smmp
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        gold = json.load(f)["minim_enkefa"]
    smmp.reset()
    smmp.epar_l.sh2 = 0
    smmp.isolty.itysol = 0
    smmp.init_energy(DATA)
    smmp.init_molecule(1, "nh2", "cooh", SEQ, VAR)
    e0, g0 = smmp.gradient()
    assert e0 == pytest.approx(1035.4, abs=0.05)               # README:391
    nop = smmp.minim(imin, 10000, 1e-9)
    e, g = smmp.gradient()
    v = np.asarray(smmp.var_r.vlvr)[np.asarray(smmp.var_i.idvr) - 1] * CRD
    smmp.reset()
    assert nop < 10000
    assert abs(e - gold["total"]) <= 5e-3, e
    assert float(np.sum(g ** 2)) < 1e-6
    want = np.array([w[2] for w in gold["variables"]])
    d = (v - want + 180.0) % 360.0 - 180.0
    assert np.all(np.abs(d) <= 0.051), np.c_[v, want]

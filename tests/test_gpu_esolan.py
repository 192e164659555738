"""The analytic SASA model (itysol < 0, esolan.f) on the GPU against the
oracle's restatement, through the C ABI: solvation term and total energy of
Met-enkephalin and of the 60-residue protein on several conformations; the
legacy layer's metropolis with this model (proposals on the host, every
energy() on the GPU) and batched sweeps of several chains (proposal, energy()
and decision launched across the chains) against the oracle's sweeps."""
import numpy as np
import pytest

from conftest import DATA, Oracle, seqfile

pytestmark = pytest.mark.gpu


def _confs(o, n, scale, seed):
    rng = np.random.default_rng(seed)
    idvr = o.idvr() - 1
    out = [o.vlvr().copy()]
    for _ in range(n - 1):
        v = o.vlvr().copy()
        v[idvr] = v[idvr] + rng.normal(0.0, scale, len(idvr))
        out.append(v)
    return out


def _gpu_energies(mol, confs):
    from smmp.ensemble import Ensemble
    n = len(confs)
    ens = Ensemble([mol], [0] * n, list(range(1, n + 1)), [1.0] * n)
    V = np.zeros((n, ens.vstride))
    for c, v in enumerate(confs):
        V[c, :len(v)] = v
    ens.set_vlvr(V)
    e = ens.energy()
    assert not ens.errors().any()
    return e, ens.terms(), ens


def _check(mol, o, confs):
    got, terms, ens = _gpu_energies(mol, confs)
    for g, t, v in zip(got, terms, confs):
        o.set_vlvr(v[:o.ntlvr])
        e, to = o.energy()
        assert t[4] == pytest.approx(to[4], rel=1e-10, abs=1e-8)   # eysl
        assert g == pytest.approx(e, rel=1e-10, abs=1e-8)
    return ens


def test_enkefa_analytic_solvation_matches_oracle():
    from smmp.ensemble import Molecule
    mol = Molecule(DATA + "enkefa.seq", DATA + "enkefa.var", libdir=DATA, itysol=-1)
    o = Oracle(DATA + "enkefa.seq", DATA + "enkefa.var", itysol=-1)
    _check(mol, o, _confs(o, 6, 0.3, 1))


def test_protein60_analytic_solvation_matches_oracle(tmp_path):
    from smmp.ensemble import Molecule
    from smmp.sequences import natural_protein
    s = seqfile(tmp_path, natural_protein(60), "protein60")
    mol = Molecule(s, libdir=DATA, itysol=-1)
    o = Oracle(s, itysol=-1)
    _check(mol, o, _confs(o, 3, 0.05, 2))


def test_legacy_metropolis_with_analytic_solvation_matches_oracle():
    import smmp
    smmp.reset()
    smmp.epar_l.sh2 = 0
    smmp.isolty.itysol = -1
    smmp.init_energy(DATA)
    smmp.init_molecule(1, "nh2", "cooh", DATA + "enkefa.seq", DATA + "enkefa.var")
    o = Oracle(DATA + "enkefa.seq", DATA + "enkefa.var", itysol=-1)
    e = smmp.energy()
    assert e == pytest.approx(o.energy()[0], rel=1e-10)
    smmp.sgrnd(4242)
    o.sgrnd(4242)
    smmp.bet.beta = 1.0 / (300 * 1.98773e-3)
    o.set_beta(smmp.bet.beta)
    eol, acz = e, 0.0
    for _ in range(3):
        eol, acz = smmp.metropolis(eol, acz, smmp.can_weight)
        oe, _ = o.sweeps(1)
        assert eol == pytest.approx(oe, rel=1e-10)
        assert np.array_equal(smmp.var_r.vlvr, o.vlvr())
    assert acz > 0
    smmp.reset()


def test_batched_sweeps_with_analytic_solvation_match_oracle():
    """Four chains, each on its own stream: every proposal's energy() runs the
    analytic SASA; after every sweep the variables equal the oracle's
    metropolis on each chain (bit for bit) and the energies agree to 1e-10."""
    from smmp.ensemble import Ensemble, Molecule, beta_of
    mol = Molecule(DATA + "enkefa.seq", DATA + "enkefa.var", libdir=DATA, itysol=-1)
    b = beta_of(300.0)
    seeds = [901, 902, 903, 904]
    ens = Ensemble([mol], [0] * 4, seeds, [b] * 4)
    oracles = []
    V = np.zeros((4, ens.vstride))
    for c, sd in enumerate(seeds):
        o = Oracle(DATA + "enkefa.seq", DATA + "enkefa.var", itysol=-1)
        o.sgrnd(sd)
        o.set_beta(b)
        oracles.append(o)
        V[c, :o.ntlvr] = o.vlvr()
    ens.set_vlvr(V)
    for k in range(3):
        ens.sweeps(1)
        V, E = ens.vlvr(), ens.energies()
        for c, o in enumerate(oracles):
            oe, _ = o.sweeps(1)
            assert np.array_equal(V[c, :o.ntlvr], o.vlvr()), (c, k)
            assert E[c] == pytest.approx(oe, rel=1e-10)
    assert not ens.errors().any()
    acc, prop = ens.acceptance()
    assert (prop == 3 * 24).all() and (acc > 0).all()


def test_pt_with_analytic_solvation_runs():
    from smmp.ensemble import Ensemble, Molecule, beta_of
    mol = Molecule(DATA + "enkefa.seq", DATA + "enkefa.var", libdir=DATA, itysol=-1)
    betas = [beta_of(t) for t in (300.0, 450.0, 700.0, 1000.0)]
    ens = Ensemble([mol], [0] * 4, [11, 12, 13, 14], betas)
    ens.set_pt(betas, wrap=False, exchange_seed=5)
    ens.pt_sweeps(2)
    assert not ens.errors().any()
    assert sorted(ens.pt_map().tolist()) == [0, 1, 2, 3]
    assert not ens.pt_fused_last()

"""GPU energy() against the CPU oracle, through the C ABI.

FP64 pair terms: agreement to ~1e-10 relative (the GPU sums in another order
and uses rsqrt).  FP32 pair terms (FP64 guard for pairs whose terms can exceed
1 kcal/mol, FP64 accumulation): within 1e-3 kcal/mol for conformations of
physical energy, 1e-7 relative for clashes.  SASA runs in FP64 with the
reference's operation order, so exposed-point counts are identical.
"""
import numpy as np
import pytest

from conftest import DATA, Oracle, seqfile

pytestmark = pytest.mark.gpu

TOL_FP32 = 1e-3       # kcal/mol, the required accuracy of FP32 pair terms


def ensemble(mol, n, fp32=False, seeds=None, betas=None):
    from smmp.ensemble import Ensemble
    seeds = seeds if seeds is not None else list(range(1, n + 1))
    betas = betas if betas is not None else [1.0] * n
    return Ensemble([mol], [0] * n, seeds, betas, fp32=fp32)


def relaxed_conformations(o, n, seed=7, sweeps=40, every=4, temp=300.0):
    """Low-energy conformations from short oracle Metropolis runs."""
    o.sgrnd(seed)
    o.random_start()
    o.set_beta(1.0 / (temp * 1.98773e-3))
    out = []
    while len(out) < n:
        o.sweeps(every)
        out.append(o.vlvr().copy())
    return out


def random_conformations(o, n, seed=3):
    rng = np.random.default_rng(seed)
    base = o.vlvr()
    idvr = o.idvr() - 1
    out = []
    for _ in range(n):
        v = base.copy()
        v[idvr] = rng.uniform(-np.pi, np.pi, len(idvr))
        out.append(v)
    return out


def compare(o, mol, confs, fp32):
    ens = ensemble(mol, len(confs), fp32=fp32)
    V = np.zeros((ens.nchains, ens.vstride))
    for c, v in enumerate(confs):
        V[c, :len(v)] = v
    ens.set_vlvr(V)
    got = ens.energy()
    terms = ens.terms()
    ref = []
    for v in confs:
        o.set_vlvr(v)
        e, t = o.energy()
        ref.append((e, t))
    assert not ens.errors().any()
    return got, terms, ref


def test_golden_enkefa_energy_and_terms():
    from smmp.ensemble import Molecule
    mol = Molecule(DATA + "enkefa.seq", DATA + "enkefa.var", libdir=DATA)
    o = Oracle(DATA + "enkefa.seq", DATA + "enkefa.var")
    got, terms, ref = compare(o, mol, [o.vlvr()], fp32=False)
    e, t = ref[0]
    assert got[0] == pytest.approx(e, rel=1e-12)
    assert round(got[0], 1) == 1035.4                      # README:391
    for k in range(4):
        assert terms[0, k] == pytest.approx(t[k], rel=1e-11, abs=1e-10)


@pytest.mark.parametrize("ff,epsd", [("ecepp3", 0), ("ecepp2", 0), ("ecepp3", 1)])
def test_relaxed_and_random_conformations_fp64(ff, epsd):
    from smmp.ensemble import Molecule
    mol = Molecule(DATA + "enkefa.seq", DATA + "enkefa.var", libdir=DATA, ff=ff, epsd=epsd)
    o = Oracle(DATA + "enkefa.seq", DATA + "enkefa.var", ff=ff, epsd=epsd)
    confs = relaxed_conformations(o.clone(), 24) + random_conformations(o, 40)
    got, _, ref = compare(o, mol, confs, fp32=False)
    for g, (e, _) in zip(got, ref):
        assert g == pytest.approx(e, rel=1e-10, abs=1e-8)


def test_fp32_pair_terms_within_1e_3():
    from smmp.ensemble import Molecule
    mol = Molecule(DATA + "enkefa.seq", DATA + "enkefa.var", libdir=DATA)
    o = Oracle(DATA + "enkefa.seq", DATA + "enkefa.var")
    relaxed = relaxed_conformations(o.clone(), 48)
    rnd = random_conformations(o, 48)
    got, _, ref = compare(o, mol, relaxed + rnd, fp32=True)
    errs = [abs(g - e) for g, (e, _) in zip(got[:48], ref[:48])]
    assert max(errs) <= TOL_FP32, max(errs)
    for g, (e, _) in zip(got[48:], ref[48:]):
        assert abs(g - e) <= max(TOL_FP32, 1e-7 * abs(e))


@pytest.mark.parametrize("n", [10, 25])
def test_polyalanine_with_sasa_fp64(tmp_path, n):
    from smmp.ensemble import Molecule
    s = seqfile(tmp_path, ["ace"] + ["ala"] * n + ["nme"])
    mol = Molecule(s, libdir=DATA, itysol=1)
    o = Oracle(s, itysol=1)
    assert mol.npairs == o.pair_count()
    confs = relaxed_conformations(o.clone(), 8, sweeps=8, every=2) + random_conformations(o, 16)
    got, terms, ref = compare(o, mol, confs, fp32=False)
    for g, tt, (e, t) in zip(got, terms, ref):
        assert g == pytest.approx(e, rel=1e-10, abs=1e-8)
        assert tt[4] == pytest.approx(t[4], rel=1e-11, abs=1e-9)   # eysl: same point counts


def test_polyalanine_with_sasa_fp32(tmp_path):
    from smmp.ensemble import Molecule
    s = seqfile(tmp_path, ["ace"] + ["ala"] * 20 + ["nme"])
    mol = Molecule(s, libdir=DATA, itysol=1)
    o = Oracle(s, itysol=1)
    confs = relaxed_conformations(o.clone(), 12, sweeps=6, every=2)
    got, _, ref = compare(o, mol, confs, fp32=True)
    assert max(abs(g - e) for g, (e, _) in zip(got, ref)) <= TOL_FP32


def test_nan_variable_sets_error_word():
    """Fault injection on the host: a NaN dihedral gives a NaN energy, which
    the kernel reports as an error word instead of trapping."""
    from smmp.ensemble import Molecule
    from smmp import SmmpError
    mol = Molecule(DATA + "enkefa.seq", DATA + "enkefa.var", libdir=DATA)
    ens = ensemble(mol, 2)
    V = ens.vlvr()
    V[1, 3] = np.nan
    ens.set_vlvr(V)
    with pytest.raises(SmmpError) as ei:
        ens.energy()
    assert ei.value.status == 4
    err = ens.errors()
    assert err[0] == 0 and err[1] == 1

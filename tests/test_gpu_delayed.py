"""Delayed acceptance: the surrogate screens proposals (stage 1) and the
exact ECEPP/3 energy decides every move that passes (stage 2).

* With a constant surrogate stage 1 passes everything and draws nothing, so
  the two-stage kernel must reproduce the plain sweep's trajectory exactly
  (FP64): this checks its proposal, rotation, exact energy, acceptance and
  random-stream bookkeeping.
* With a surrogate trained on the plain sampler's own parallel-tempering
  states, stage 1 filters most rejections: the exact energy is evaluated far
  fewer times per accepted move, the stationary energy distribution is the
  plain method's within statistical error, and the closing consistency check
  holds for every sweep.
"""
import numpy as np
import pytest

from conftest import DATA, Oracle

pytestmark = pytest.mark.gpu


def _mol():
    from smmp.ensemble import Molecule
    return Molecule(DATA + "enkefa.seq", DATA + "enkefa.var", libdir=DATA)


def test_plain_fallback_reproduces_plain_trajectory():
    """floor=1 with min_stage1=0 puts every chain on the fallback from the
    start: the two-stage kernel's plain path (one proposal at a time, exact
    energy, same uniforms in the same order) must give the plain sweep's
    trajectory bit for bit (FP64)."""
    from smmp.ensemble import Ensemble, beta_of
    from smmp.surrogate import Surrogate
    mol = _mol()
    n = 8
    seeds = [500 + c for c in range(n)]
    betas = [beta_of(t) for t in np.linspace(250.0, 600.0, n)]
    plain = Ensemble([mol], [0] * n, seeds, betas)
    da = Ensemble([mol], [0] * n, seeds, betas)
    plain.random_start()
    da.random_start()
    plain.sweeps(3)                       # leave the clash region first
    da.sweeps(3)
    sur = Surrogate(mol.nvr, seed=1)
    da.set_surrogate(sur, floor=1.0, min_stage1=0)
    for k in range(30):
        plain.sweeps(1)
        da.sweeps(1)
        assert np.array_equal(plain.vlvr(), da.vlvr()), k
    assert not da.errors().any()
    n1, n2 = da.da_stats()
    assert not n1.any() and not n2.any()
    np.testing.assert_allclose(plain.energies(), da.energies(), rtol=1e-12, atol=1e-9)


def test_constant_surrogate_keeps_the_energy_distribution():
    """A constant surrogate passes every proposal at stage 1, so the batched
    two-stage sweep is a plain Metropolis sweep with another use of the
    uniforms: same mean energy within statistical error."""
    from smmp.ensemble import Ensemble, beta_of
    from smmp.surrogate import Surrogate
    mol = _mol()
    n = 64
    b = beta_of(400.0)
    res = []
    for mode in (0, 1):
        ens = Ensemble([mol], [0] * n, [700 + c for c in range(n)], [b] * n, fp32=True)
        ens.random_start()
        ens.sweeps(100)
        if mode:
            sur = Surrogate(mol.nvr, seed=1)
            sur.set_params(np.zeros(sur.nparams, dtype=np.float32),
                           np.array([0.0, 1.0], np.float32))
            ens.set_surrogate(sur, floor=0.0, min_stage1=0)
        m = np.zeros(n)
        for _ in range(300):
            ens.sweeps(1)
            m += ens.energies()
        assert not ens.errors().any()
        if mode:
            n1, _ = ens.da_stats()
            assert np.all(n1 == 300 * mol.nvr)      # everything passes stage 1
        res.append(m / 300)
    se = np.sqrt(res[0].var(ddof=1) / n + res[1].var(ddof=1) / n)
    assert abs(res[0].mean() - res[1].mean()) < 4 * se


@pytest.fixture(scope="module")
def trained():
    """Surrogate trained on 64-replica PT states (100-1000 K) of the plain
    sampler, as the enkephalin surrogate configuration does (smaller)."""
    from smmp.ensemble import Ensemble, beta_of
    from smmp.surrogate import Surrogate, collect_samples
    mol = _mol()
    temps = [100.0 * 10 ** (k / 63) for k in range(64)]
    betas = [beta_of(t) for t in temps]
    ens = Ensemble([mol], [0] * 64, [31433 + 1000 * k for k in range(64)], betas, fp32=True)
    ens.random_start()
    ens.set_pt(betas, wrap=False)
    ens.pt_sweeps(100, graph_chunk=50)             # burn-in
    ang, e = collect_samples(ens, mol, 500)
    rng = np.random.default_rng(0)
    order = rng.permutation(len(e))
    ntest = len(e) // 10
    test, train = order[:ntest], order[ntest:]
    sur = Surrogate(mol.nvr, seed=2)
    sur.set_data(ang[train], e[train], clip=200.0)
    sur.train(40, batch=512, lr=1e-3)
    return mol, sur, ang[test], e[test], ens


def test_trained_surrogate_accuracy_against_fp64_oracle(trained):
    mol, sur, ang, e, _ = trained
    keep = e < 50.0                                   # the sampled low-energy region
    pred = sur.predict(ang[keep])
    o = Oracle(DATA + "enkefa.seq", DATA + "enkefa.var")
    v = o.vlvr()
    sub = np.flatnonzero(keep)[:200]
    ref = []
    for i in sub:
        v[mol.idvr] = ang[i]
        o.set_vlvr(v)
        ref.append(o.energy()[0])
    ref = np.array(ref)
    assert np.max(np.abs(e[sub] - ref)) < 2e-2        # the FP32 sampler's labels
    rmse = float(np.sqrt(np.mean((pred[:len(sub)] - ref) ** 2)))
    assert rmse < 0.25 * float(np.std(ref)), (rmse, np.std(ref))


def test_delayed_acceptance_gain_and_stationarity(trained):
    """300 K from the same states: DA evaluates the exact energy far fewer
    times per accepted move, and the mean energy matches the plain method's
    within statistical error."""
    from smmp.ensemble import Ensemble, beta_of
    mol, sur, _, _, src = trained
    n = 64
    start = src.vlvr()
    b = beta_of(300.0)
    res = {}
    for mode in ("plain", "da"):
        ens = Ensemble([mol], [0] * n, [900 + c for c in range(n)], [b] * n, fp32=True)
        ens.set_vlvr(start)
        if mode == "da":
            ens.set_surrogate(sur, floor=0.2, min_stage1=64)
        ens.sweeps(100)                               # equilibrate at 300 K
        acc0, prop0 = ens.acceptance()
        n10, n20 = ens.da_stats() if mode == "da" else (None, None)
        means = np.zeros(n)
        for k in range(300):
            ens.sweeps(1)
            means += ens.energies()
        means /= 300
        assert not ens.errors().any()
        acc, prop = ens.acceptance()
        accepted = float((acc - acc0).sum())
        if mode == "da":
            n1, n2 = ens.da_stats()
            exact = float((n1 - n10).sum())
        else:
            exact = float((prop - prop0).sum())
        res[mode] = (means, exact / accepted)
    mp, mda = res["plain"][0], res["da"][0]
    se = np.sqrt(mp.var(ddof=1) / n + mda.var(ddof=1) / n)
    assert abs(mp.mean() - mda.mean()) < 4 * se, (mp.mean(), mda.mean(), se)
    # exact energy evaluations per accepted move
    assert res["da"][1] < 0.5 * res["plain"][1], res

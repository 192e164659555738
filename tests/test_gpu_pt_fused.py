"""Several sweeps in one launch against one launch per sweep, and batched
parallel tempering as one cooperative launch (sweeps and exchanges separated
by grid barriers) against the graph path of separate sweep and exchange
launches: the whole ensemble state (variables, streams, energies, temperature
map, exchange statistics) is bit-identical after the same run."""
import numpy as np
import pytest

from conftest import DATA, seqfile

pytestmark = pytest.mark.gpu


def _ladder(n, t0=200.0, t1=1000.0):
    from smmp.ensemble import beta_of
    return [beta_of(t) for t in t0 * (t1 / t0) ** (np.arange(n) / (n - 1))]


def _run(mols, chain_mol, fp32, fused, nsweeps, chunks, wrap):
    from smmp.ensemble import Ensemble
    n = len(chain_mol)
    betas = _ladder(n)
    ens = Ensemble(mols, chain_mol, [5100 + 37 * c for c in range(n)], betas, fp32=fp32)
    ens.random_start()
    ens.sweeps(3)                      # off the random start's clashes
    ens.set_pt(betas, wrap=wrap, exchange_seed=2024)
    ens.set_pt_fused(fused)
    for k in chunks:
        ens.pt_sweeps(k, graph_chunk=4)
        assert ens.pt_fused_last() == fused
    assert sum(chunks) == nsweeps
    assert not ens.errors().any()
    return ens


def _enkefa():
    from smmp.ensemble import Molecule
    return Molecule(DATA + "enkefa.seq", DATA + "enkefa.var", libdir=DATA)


@pytest.mark.parametrize("fp32,wrap", [(False, True), (True, False)])
def test_fused_pt_equals_graph_path_enkefa(fp32, wrap):
    mol = _enkefa()
    chunks = [5, 1, 6]
    a = _run([mol], [0] * 16, fp32, True, 12, chunks, wrap)
    b = _run([mol], [0] * 16, fp32, False, 12, chunks, wrap)
    assert np.array_equal(a.vlvr(), b.vlvr())
    assert np.array_equal(a.energies(), b.energies())
    assert np.array_equal(a.pt_map(), b.pt_map())
    assert sorted(a.pt_map().tolist()) == list(range(16))
    assert a.checkpoint() == b.checkpoint()


def test_fused_pt_equals_graph_path_polyalanine_sasa(tmp_path):
    """Uneven chains (rows form, SASA, FP32 incremental pair sums)."""
    from smmp.ensemble import Molecule
    from smmp.sequences import polyala
    mols = [Molecule(seqfile(tmp_path, polyala(n), "ala%d" % n), libdir=DATA, itysol=1)
            for n in (12, 20)]
    chain_mol = [c % 2 for c in range(8)]
    a = _run(mols, chain_mol, True, True, 4, [4], True)
    b = _run(mols, chain_mol, True, False, 4, [4], True)
    assert np.array_equal(a.vlvr(), b.vlvr())
    assert np.array_equal(a.pt_map(), b.pt_map())
    assert a.checkpoint() == b.checkpoint()


@pytest.mark.parametrize("fp32", [False, True])
def test_multi_sweep_launch_equals_single_sweep_launches(fp32):
    """The opening energy() of every sweep follows one more setvar call, as
    the reference's energy() does (energy.f:47): with FP64 pair terms a launch
    of six sweeps leaves the same bits as six launches of one.  With FP32 pair
    terms only a launch's first sweep rebuilds the coordinates (later ones
    keep the rotated coordinates, equal up to FP64 rounding), so the runs
    agree to rounding."""
    from smmp.ensemble import Ensemble, beta_of
    mol = _enkefa()
    out = []
    for per_launch in (6, 1):
        ens = Ensemble([mol], [0] * 4, [77, 78, 79, 80], [beta_of(300.0)] * 4, fp32=fp32)
        ens.random_start()
        for _ in range(6 // per_launch):
            ens.sweeps(per_launch)
        assert not ens.errors().any()
        out.append((ens.vlvr(), ens.energies(), ens.terms(), ens.checkpoint()))
    if not fp32:
        assert np.array_equal(out[0][0], out[1][0])
        assert np.array_equal(out[0][1], out[1][1])
        assert np.array_equal(out[0][2], out[1][2])
        assert out[0][3] == out[1][3]
    else:
        np.testing.assert_allclose(out[0][0], out[1][0], rtol=0, atol=1e-12)
        np.testing.assert_allclose(out[0][1], out[1][1], rtol=1e-9, atol=1e-6)
        np.testing.assert_allclose(out[0][2], out[1][2], rtol=1e-9, atol=1e-6)


def test_more_chains_than_resident_blocks_take_the_graph_path():
    """One block of 512 threads per SM: 160 chains cannot all be resident on
    148 SMs, so the run falls back to separate launches (same results as an
    ensemble that asked for them)."""
    from smmp.ensemble import Ensemble
    mol = _enkefa()
    n = 160
    betas = _ladder(n)
    out = []
    for fused in (True, False):
        ens = Ensemble([mol], [0] * n, list(range(1, n + 1)), betas)
        ens.random_start()
        ens.set_pt(betas, exchange_seed=7)
        ens.set_pt_fused(fused)
        ens.pt_sweeps(2, graph_chunk=1)
        assert not ens.pt_fused_last()
        assert not ens.errors().any()
        out.append(ens.checkpoint())
    assert out[0] == out[1]


def test_grid_barrier_wait_is_bounded():
    """A barrier that never opens (it waits for one arrival more than the
    launch has blocks): every chain gives up after the timeout with error
    code 4, the call reports it, and the context stays usable."""
    from smmp._lib import SmmpError
    from smmp.ensemble import Ensemble
    mol = _enkefa()
    betas = _ladder(8)
    ens = Ensemble([mol], [0] * 8, list(range(1, 9)), betas)
    ens.random_start()
    ens.set_pt(betas)
    ens.set_pt_fused(True, timeout_s=0.05, barrier_extra=1)
    with pytest.raises(SmmpError):
        ens.pt_sweeps(3)
    assert ens.pt_fused_last()
    assert (ens.errors() == 4).all()
    ok = _run([mol], [0] * 8, False, True, 2, [2], True)   # a new ensemble runs
    assert not ok.errors().any()

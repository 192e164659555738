"""GPU sweeps against the oracle: RNG streams, accept/reject trajectories,
parallel tempering, checkpoints."""
import numpy as np
import pytest

from conftest import DATA, Oracle, seqfile

pytestmark = pytest.mark.gpu


def mol_enkefa(ff="ecepp3", var="enkefa.var"):
    from smmp.ensemble import Molecule
    return Molecule(DATA + "enkefa.seq", DATA + var if var else None, libdir=DATA, ff=ff)


@pytest.mark.parametrize("seed", [4357, 31433, 81236])
def test_device_stream_equals_oracle_stream(seed):
    from smmp.ensemble import Ensemble
    ens = Ensemble([mol_enkefa()], [0, 0], [seed, seed + 1], [1.0, 1.0])
    o = Oracle(DATA + "enkefa.seq")
    o.sgrnd(seed)
    want = np.array([o.grnd() for _ in range(3000)])
    got = ens.draw(0, 3000)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("fp32", [False, True])
def test_canonical_trajectory_matches_oracle(fp32):
    """Seeded random start + 300 sweeps at 300 K: the variables after every
    sweep are bit-identical, i.e. the same proposals were accepted."""
    from smmp.ensemble import Ensemble, beta_of
    b = beta_of(300.0)
    ens = Ensemble([mol_enkefa()], [0], [31433], [b], fp32=fp32)
    ens.random_start()
    o = Oracle(DATA + "enkefa.seq", DATA + "enkefa.var")
    o.sgrnd(31433)
    o.random_start()
    o.set_beta(b)
    first_diff = None
    for k in range(300):
        ens.sweeps(1)
        o.sweeps(1)
        if not np.array_equal(ens.vlvr()[0, :o.ntlvr], o.vlvr()):
            first_diff = k
            break
    assert not ens.errors().any()
    if not fp32:
        assert first_diff is None
    else:   # FP32 energies may flip a decision only at an exact threshold tie
        assert first_diff is None or first_diff > 100


def test_annealing_golden_on_gpu():
    """EXAMPLES/annealing.out: 100,000 sweeps, same acceptance rate to the
    last printed digit and the same lowest-energy sweep."""
    import json
    import smmp
    from conftest import GOLDEN
    g = json.load(open(GOLDEN))["anneal_ecepp2"]
    smmp.reset()
    smmp.epar_l.sh2 = 1
    smmp.isolty.itysol = 0
    smmp.init_energy(DATA)
    smmp.init_molecule(1, "nh2", "cooh", DATA + "enkefa.seq", DATA + "enkefa.ann")
    smmp.sgrnd(81236)
    out = smmp.anneal(100, 100000, 1000, 1000.0, 100.0, 1)
    smmp.reset()
    assert out[0] == pytest.approx(7.59205812552858e8, rel=1e-12)
    assert out[1] == pytest.approx(g["after_equilibration"], rel=1e-12)
    assert out[2] == pytest.approx(g["acceptance"], rel=1e-14)
    assert out[5] == g["lowest_sweep"]
    assert out[4] == pytest.approx(g["lowest"], rel=1e-9)


def test_legacy_api_energy_and_metropolis():
    import smmp
    smmp.reset()
    smmp.epar_l.sh2 = 0
    smmp.init_energy(DATA)
    smmp.init_molecule(1, "nh2", "cooh", DATA + "enkefa.seq", DATA + "enkefa.var")
    e = smmp.energy()
    assert round(e, 1) == 1035.4
    assert smmp.mol_par.nvr == 24
    smmp.sgrnd(31433)
    smmp.bet.beta = 1.0 / (300 * 1.98773e-3)
    o = Oracle(DATA + "enkefa.seq", DATA + "enkefa.var")
    o.sgrnd(31433)
    o.set_beta(smmp.bet.beta)
    eol, acz = e, 0.0
    for _ in range(5):
        eol, acz = smmp.metropolis(eol, acz, smmp.can_weight)
        oe, _ = o.sweeps(1)
        assert eol == pytest.approx(oe, rel=1e-10)
    assert np.array_equal(smmp.var_r.vlvr, o.vlvr())
    # a Python weight goes through the host callback path, same stream
    eol2, acz2 = smmp.metropolis(eol, acz, lambda x: x * smmp.bet.beta)
    oe, _ = o.sweeps(1)
    assert eol2 == pytest.approx(oe, rel=1e-10)
    # writing into the COMMON view is seen by the next call
    v = smmp.var_r.vlvr
    v[3] = 0.5
    o.set_vlvr(np.asarray(v))
    assert smmp.energy() == pytest.approx(o.energy()[0], rel=1e-10)
    smmp.reset()


def test_serial_pt_matches_partem_s():
    """shared_stream + serial schedule reproduces partem_s.f (newsta, switch=1):
    same final energies, variables and temperature map."""
    import ctypes
    from smmp.ensemble import Ensemble
    temps = [1000.0, 600.0, 400.0, 300.0]
    betas = [1.0 / (t * 0.00198773) for t in temps]
    n, nequi, nswp = len(temps), 2, 12
    o = Oracle(DATA + "enkefa.seq", DATA + "enkefa.var")
    o.sgrnd(4242)
    eo = np.zeros(n)
    ipo = np.zeros(n, dtype=np.int32)
    vl = np.zeros(n * o.nvr)
    b = (ctypes.c_double * n)(*betas)
    rc = o.lib().orc_partem(o.h, n, b, nequi, nswp, eo.ctypes.data_as(ctypes.c_void_p),
                            ipo.ctypes.data_as(ctypes.c_void_p),
                            vl.ctypes.data_as(ctypes.c_void_p))
    assert rc == 0
    g = Ensemble([mol_enkefa()], [0] * n, [4242], betas, shared_stream=True)
    g.random_start()
    g.set_pt(betas, wrap=True)
    g.equilibrate(nequi)          # partem_s.f:134-162, replica by replica
    g.pt_sweeps(nswp, serial=True)
    assert np.allclose(g.energies(), eo, rtol=1e-10, atol=1e-8)
    assert np.array_equal(g.pt_map(), ipo - 1)
    idvr = o.idvr() - 1
    assert np.array_equal(g.vlvr()[:, idvr], vl.reshape(n, -1))


def test_batched_pt_runs_and_checkpoint_restores_bit_identically():
    from smmp.ensemble import Ensemble, beta_of
    n = 16
    temps = 100.0 * 10 ** (np.arange(n) / (n - 1))
    betas = [beta_of(t) for t in temps]
    ens = Ensemble([mol_enkefa()], [0] * n, [31433 + 1000 * k for k in range(n)], betas)
    ens.random_start()
    ens.set_pt(betas, wrap=False, exchange_seed=99)
    ens.pt_sweeps(10, graph_chunk=5)
    blob = ens.checkpoint()
    ens.pt_sweeps(7, graph_chunk=1)
    a_v, a_e, a_m = ens.vlvr(), ens.energies(), ens.pt_map()
    ens.restore(blob)
    ens.pt_sweeps(7, graph_chunk=1)
    assert np.array_equal(ens.vlvr(), a_v)
    assert np.array_equal(ens.energies(), a_e)
    assert np.array_equal(ens.pt_map(), a_m)
    assert sorted(a_m.tolist()) == list(range(n))
    assert not ens.errors().any()
    acc, prop = ens.acceptance()
    assert (prop == 17 * 24).all() and (acc > 0).all()


def test_uneven_chains_in_one_launch(tmp_path):
    from smmp.ensemble import Ensemble, Molecule, beta_of
    mols, oracles = [], []
    for n in (3, 7, 12):
        s = seqfile(tmp_path, ["ace"] + ["ala"] * n + ["nme"], name="ala%d" % n)
        mols.append(Molecule(s, libdir=DATA))
        oracles.append(Oracle(s))
    chain_mol = [0, 1, 2, 2, 1, 0]
    b = beta_of(300.0)
    ens = Ensemble(mols, chain_mol, [11, 12, 13, 14, 15, 16], [b] * 6)
    ens.random_start()
    ens.sweeps(20)
    assert not ens.errors().any()
    for c, m in enumerate(chain_mol):
        o = oracles[m].clone()
        o.sgrnd(11 + c)
        o.random_start()
        o.set_beta(b)
        o.sweeps(20)
        assert np.array_equal(ens.vlvr()[c, :o.ntlvr], o.vlvr())

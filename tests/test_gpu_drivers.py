"""The reference-facing drivers on the GPU against the oracle's restatements,
FP64 pair terms (the legacy layer), same seeds: canon (canon.f:12-132), sweeps
with the multicanonical weights muca_weight / muca_weight2 looked up on the
device (mulcan_par_mod.f90:380-410), the whole mulcan_par weight iteration
(mulcan_par_mod.f90:23-190), and enysol (enysol.f:13)."""
import ctypes

import numpy as np
import pytest

from conftest import DATA, Oracle

pytestmark = pytest.mark.gpu

SEQ, VAR = DATA + "enkefa.seq", DATA + "enkefa.var"


def _legacy(itysol=0, seed=31433):
    import smmp
    smmp.reset()
    smmp.epar_l.sh2 = 0
    smmp.isolty.itysol = itysol
    smmp.init_energy(DATA)
    smmp.init_molecule(1, "nh2", "cooh", SEQ, VAR)
    smmp.sgrnd(seed)
    return smmp


def test_canon_matches_the_oracle():
    smmp = _legacy()
    trace, equi, acc, last = smmp.canon(5, 40, 10, 300.0, 1)
    smmp.reset()
    o = Oracle(SEQ, VAR)
    o.sgrnd(31433)
    t = np.zeros(5)
    out = np.zeros(3)
    L = o.lib()
    L.orc_canon.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                            ctypes.c_double, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    assert L.orc_canon(o.h, 5, 40, 10, 300.0, 1, t.ctypes.data, out.ctypes.data) == 0
    np.testing.assert_allclose(trace, t, rtol=1e-10, atol=1e-8)
    assert equi == pytest.approx(out[0], rel=1e-10, abs=1e-8)
    assert acc == out[1]
    assert last == pytest.approx(out[2], rel=1e-10, abs=1e-8)


@pytest.mark.parametrize("kind", [1, 2])
def test_multicanonical_weights_on_the_device(kind):
    """Sweeps whose acceptance uses a muca table looked up on the GPU give the
    oracle's trajectory (variables after every sweep, energies)."""
    from smmp.ensemble import Ensemble, Molecule, beta_of
    import smmp
    kmin, kmax, ebin = -10, 40, 1.0
    rng = np.random.default_rng(kind)
    b = rng.uniform(-0.2, 0.3, kmax - kmin + 1)
    alpha = rng.uniform(-2.0, 2.0, kmax - kmin + 1)
    w = smmp.MucaWeight(b, alpha, kmin, kmax, ebin, kind=kind)
    beta = beta_of(500.0)
    mol = Molecule(SEQ, VAR, libdir=DATA)
    ens = Ensemble([mol], [0], [4242], [beta])
    ens.random_start()
    o = Oracle(SEQ, VAR)
    o.sgrnd(4242)
    o.random_start()
    o.set_beta(beta)
    L = o.lib()
    L.orc_sweeps_muca.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.c_void_p, ctypes.c_void_p]
    eol, acz = ctypes.c_double(0.0), ctypes.c_double(0.0)
    bb, aa = np.ascontiguousarray(b), np.ascontiguousarray(alpha)
    for k in range(30):
        ens.sweeps(1, weight=w)
        assert L.orc_sweeps_muca(o.h, 1, kind, kmin, kmax, ebin, bb.ctypes.data, aa.ctypes.data,
                                 ctypes.byref(eol), ctypes.byref(acz)) == 0
        assert np.array_equal(ens.vlvr()[0, :o.ntlvr], o.vlvr()), k
    assert not ens.errors().any()
    assert ens.energies()[0] == pytest.approx(eol.value, rel=1e-10, abs=1e-8)
    a, p = ens.acceptance()
    assert 0 < a[0] < p[0] and a[0] == acz.value


def test_mulcan_par_matches_the_oracle(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    smmp = _legacy(seed=777)
    kmin, kmax, ebin = -12, 30, 1.0
    st = smmp.mulcan_par(60, 20, 1000.0, kmin, kmax, ebin)
    smmp.reset()
    o = Oracle(SEQ, VAR)
    o.sgrnd(777)
    nb = kmax - kmin + 1
    b, alpha, out = np.zeros(nb), np.zeros(nb), np.zeros(2)
    L = o.lib()
    L.orc_mulcan_par.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                 ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_void_p,
                                 ctypes.c_void_p, ctypes.c_void_p]
    assert L.orc_mulcan_par(o.h, 60, 20, 1000.0, kmin, kmax, ebin, b.ctypes.data,
                            alpha.ctypes.data, out.ctypes.data) == 0
    assert st.acceptance == out[0]
    assert st.last_energy == pytest.approx(out[1], rel=1e-10, abs=1e-8)
    np.testing.assert_allclose(st.b, b, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(st.alpha, alpha, rtol=1e-12, atol=1e-12)
    assert (tmp_path / "muca.d").exists() and (tmp_path / "mpar_full.d").exists()


def test_enysol_matches_the_oracle():
    smmp = _legacy(itysol=1)
    v = np.asarray(smmp.var_r.vlvr).copy()
    e = smmp.enysol(0)
    smmp.reset()
    o = Oracle(SEQ, VAR, itysol=1)
    o.set_vlvr(v)
    o.energy()
    got = ctypes.c_double()
    L = o.lib()
    L.orc_enysol.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    assert L.orc_enysol(o.h, 0, ctypes.byref(got)) == 0
    assert e == pytest.approx(got.value, rel=1e-11, abs=1e-11)
    smmp = _legacy(itysol=0)
    with pytest.raises(smmp.SmmpError):
        smmp.enysol(0)
    smmp.reset()

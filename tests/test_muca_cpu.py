"""The multicanonical weight recursion of mulcan_par (mulcan_par_mod.f90:
93-145 every nup sweeps, 163-168 at the end) in the product's host code
against the oracle's restatement, bit for bit, over several updates of
synthetic histograms (CPU; the sweeps that fill the histograms are the GPU's
tested multicanonical Metropolis)."""
import ctypes

import numpy as np

from conftest import Oracle


def _oracle_update(kmin, kmax, ebin, beta, ihist, arrs):
    L = Oracle.lib()
    L.orc_muca_update.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double] + \
        [ctypes.c_void_p] * 6
    assert L.orc_muca_update(kmin, kmax, ebin, beta, ihist.ctypes.data_as(ctypes.c_void_p),
                             *(a.ctypes.data_as(ctypes.c_void_p) for a in arrs)) == 0


def test_weight_recursion_matches_oracle():
    import smmp
    kmin, kmax, ebin = -12, 20, 1.0
    beta = 1.0 / (300 * 1.98773e-3)
    st = smmp.MucaState(kmin, kmax, ebin)
    n = kmax - kmin + 1
    ref = [np.zeros(n) for _ in range(5)]   # xhist, g1, b, alpha, ent
    rng = np.random.default_rng(9)
    centre = 12.0
    for rnd in range(6):
        # a histogram drifting towards low energies, some bins empty or single
        e = rng.normal(centre - 3.0 * rnd, 4.0, 400)
        k = np.clip(np.trunc(e / ebin + np.copysign(0.5, e)), kmin, kmax).astype(int)
        h = np.bincount(k - kmin, minlength=n).astype(np.int32)
        h[rng.integers(0, n, 4)] = 1
        h1, h2 = h.copy(), h.copy()
        st.update(h1, beta)
        _oracle_update(kmin, kmax, ebin, beta, h2, ref)
        assert not h1.any() and not h2.any()
        for got, want in zip((st.xhist, st.g1, st.b, st.alpha, st.ent), ref):
            assert np.array_equal(got, want), rnd
    assert np.abs(st.b).max() > 0.0
    L = Oracle.lib()
    L.orc_muca_finish.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_void_p, ctypes.c_void_p]
    st.finish(beta)
    assert L.orc_muca_finish(kmin, kmax, ebin, beta, ref[2].ctypes.data_as(ctypes.c_void_p),
                             ref[3].ctypes.data_as(ctypes.c_void_p)) == 0
    assert np.array_equal(st.b, ref[2]) and np.array_equal(st.alpha, ref[3])


def test_addang_wraps_like_the_reference():
    import smmp
    pi = np.pi
    for a, b in [(pi, 0.5), (pi, -0.5), (pi, pi), (-pi, -0.1), (3.0, 3.0), (0.1, 0.2)]:
        d = np.fmod(a + b, 2 * pi)
        want = d if abs(d) <= pi else d - np.copysign(2 * pi, d)
        assert smmp._addang(a, b) == want


def test_mulcan_par_driver_logic(tmp_path, monkeypatch):
    """The driver's host logic with the GPU calls replaced by a seeded fake
    walk: energies binned as mulcan_par_mod.f90:118 bins them, the weights
    updated every nup sweeps from exactly those histograms (checked by
    replaying the recursion), mpar_full.d and muca.d written, and the
    acceptance normalised by (nsweep+1)*nvr as the Fortran loop leaves it."""
    import smmp
    rng = np.random.default_rng(2)
    energies = list(rng.normal(5.0, 6.0, 64))
    calls = {"metropolis": 0}

    class FakeVar:
        vlvr = np.zeros(10)
        axvr = np.full(10, 2 * np.pi)

    def fake_metropolis(eol, acz, w):
        calls["metropolis"] += 1
        assert isinstance(w, smmp.MucaWeight) and w.kind == 1
        return energies[calls["metropolis"] - 1], acz + 3.0

    monkeypatch.chdir(tmp_path)
    monkeypatch.setattr(smmp, "metropolis", fake_metropolis)
    monkeypatch.setattr(smmp, "energy", lambda: 0.0)
    monkeypatch.setattr(smmp, "outpdb", lambda nml, f: None)
    monkeypatch.setattr(smmp, "grnd", lambda: 0.25)
    monkeypatch.setattr(smmp, "var_r", FakeVar())
    monkeypatch.setattr(smmp, "var_i", type("I", (), {"idvr": np.array([1, 2, 3])})())
    monkeypatch.setattr(smmp, "mol_par", type("M", (), {"nvr": 3})())
    monkeypatch.setattr(smmp, "bet", type("B", (), {"beta": 0.0})())
    kmin, kmax, ebin, nup, nsweep = -8, 16, 1.0, 16, 64
    st = smmp.mulcan_par(nsweep, nup, 300.0, kmin, kmax, ebin)
    assert calls["metropolis"] == nsweep
    beta = 1.0 / (300.0 * 1.98773e-3)
    ref = smmp.MucaState(kmin, kmax, ebin)
    h = np.zeros(kmax - kmin + 1, dtype=np.int32)
    for n, e in enumerate(energies, start=1):
        k = int(min(float(kmax), max(float(kmin), e / ebin + np.copysign(0.5, e))))
        h[k - kmin] += 1
        if n % nup == 0:
            ref.update(h, beta)
    ref.finish(beta)
    assert np.array_equal(st.b, ref.b) and np.array_equal(st.alpha, ref.alpha)
    assert np.array_equal(st.xhist, ref.xhist)
    assert st.acceptance == 3.0 * nsweep / ((nsweep + 1) * 3)
    rows = np.loadtxt(tmp_path / "mpar_full.d")
    assert rows.shape == (kmax - kmin + 1, 6) and rows[0, 0] == kmax
    muca = np.loadtxt(tmp_path / "muca.d")
    assert np.allclose(muca[:, 1], st.b) and np.allclose(muca[:, 2], st.alpha)

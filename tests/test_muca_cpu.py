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

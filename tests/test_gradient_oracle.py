"""The oracle's restatement of gradient.f / opeshe.f (energy derivatives with
respect to the dihedrals, the recursive force and torque sums) and of
opesol.f with esolan.f's area derivatives (the analytic solvation term): the
energy is the oracle's energy() and the derivatives equal central finite
differences of that energy, for ECEPP/3, ECEPP/2, the sigmoidal dielectric
and the analytic SASA model."""
import numpy as np
import pytest

from conftest import DATA, Oracle


def _check(o, v, h=1e-5):
    o.set_vlvr(v)
    e, g = o.gradient()
    e0, _ = o.energy()
    assert e == pytest.approx(e0, rel=1e-13, abs=1e-10)
    num = np.zeros(len(v))
    for k in range(len(v)):
        vp = v.copy()
        vp[k] += h
        o.set_vlvr(vp)
        ep, _ = o.energy()
        vm = v.copy()
        vm[k] -= h
        o.set_vlvr(vm)
        em, _ = o.energy()
        num[k] = (ep - em) / (2 * h)
    o.set_vlvr(v)
    # central differences: truncation ~h^2, cancellation ~1e-16 * (largest
    # term) / h, which the largest derivative bounds
    tol = 1e-5 * np.maximum(1.0, np.abs(num)) + 1e-8 * np.abs(num).max()
    assert np.all(np.abs(g - num) <= tol), np.c_[g, num]


@pytest.mark.parametrize("ff,epsd", [("ecepp3", 0), ("ecepp2", 0), ("ecepp3", 1)])
def test_gradient_equals_finite_differences(ff, epsd):
    o = Oracle(DATA + "enkefa.seq", DATA + "enkefa.var", ff=ff, epsd=epsd)
    v0 = o.vlvr().copy()
    _check(o, v0)
    rng = np.random.default_rng(11)
    idvr = o.idvr() - 1
    for _ in range(2):
        v = v0.copy()
        v[idvr] = v[idvr] + rng.normal(0.0, 0.05, len(idvr))
        _check(o, v)


@pytest.mark.parametrize("ff,epsd", [("ecepp3", 0), ("ecepp2", 0), ("ecepp3", 1)])
def test_order_free_sums_equal_the_recursion(ff, epsd):
    """Total atomic forces from all pairs, then each variable's force and
    torque sums over the atoms it moves (the form a parallel gradient kernel
    computes) give opeshe's derivatives to rounding."""
    import ctypes
    o = Oracle(DATA + "enkefa.seq", DATA + "enkefa.var", ff=ff, epsd=epsd)
    lib = o.lib()
    lib.orc_gradient_by_sums.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    rng = np.random.default_rng(3)
    idvr = o.idvr() - 1
    for k in range(3):
        v = o.vlvr().copy()
        if k:
            v[idvr] = v[idvr] + rng.normal(0.0, 0.05, len(idvr))
        o.set_vlvr(v)
        _, g = o.gradient()
        g2 = np.zeros(o.ntlvr)
        assert lib.orc_gradient_by_sums(o.h, g2.ctypes.data_as(ctypes.c_void_p)) == 0
        assert np.abs(g - g2).max() <= 1e-12 * np.abs(g).max()


def test_solvation_gradient_equals_finite_differences():
    """itysol = -1: the gradient minus the vacuum gradient is the derivative
    of eysl alone (opesol.f, esolan.f:547-569, 718-899, 998-1042)."""
    an = Oracle(DATA + "enkefa.seq", DATA + "enkefa.var", itysol=-1)
    va = Oracle(DATA + "enkefa.seq", DATA + "enkefa.var")
    v0 = an.vlvr().copy()
    rng = np.random.default_rng(5)
    idvr = an.idvr() - 1
    for k in range(3):
        v = v0.copy()
        if k:
            v[idvr] = v[idvr] + rng.normal(0.0, 0.05, len(idvr))
        an.set_vlvr(v)
        va.set_vlvr(v)
        ea, ga = an.gradient()
        e0, t = an.energy()
        assert ea == pytest.approx(e0, rel=1e-13, abs=1e-10)
        _, gv = va.gradient()
        gs = ga - gv
        h = 1e-5
        num = np.zeros(len(v))
        for j in range(len(v)):
            vp = v.copy()
            vp[j] += h
            an.set_vlvr(vp)
            _, tp = an.energy()
            vm = v.copy()
            vm[j] -= h
            an.set_vlvr(vm)
            _, tm = an.energy()
            num[j] = (tp[4] - tm[4]) / (2 * h)
        an.set_vlvr(v)
        assert np.abs(num).max() > 1.0   # the solvation term does depend on the dihedrals
        assert np.all(np.abs(gs - num) <= 1e-6 * np.maximum(1.0, np.abs(num))), np.c_[gs, num]


def test_gradient_refuses_numerical_solvation():
    o = Oracle(DATA + "enkefa.seq", DATA + "enkefa.var", itysol=1)
    lib = o.lib()
    import ctypes
    e = ctypes.c_double()
    g = np.zeros(o.ntlvr)
    assert lib.orc_gradient(o.h, ctypes.byref(e), g.ctypes.data_as(ctypes.c_void_p)) != 0

"""The oracle's restatement of esolan.f (analytic SASA, itysol < 0) on the CPU.

The reference publishes no output of esolan, so the restatement is pinned by
geometry instead: the closed-form area of two intersecting spheres (also when
the north point of a sphere lies on its neighbour, which sends esolan.f
through its random re-orientation), and clusters of spheres against a fine
numerical quadrature of the exposed surface.  On Met-enkephalin the analytic
solvation energy agrees with the numerical one of enysol.f (itysol > 0) to
within the point-set quadrature error of the latter."""
import math

import numpy as np
import pytest

from conftest import DATA, Oracle


def _two_sphere_areas(c1, r1, c2, r2):
    d = float(np.linalg.norm(np.subtract(c2, c1)))
    h1 = r1 - (d * d + r1 * r1 - r2 * r2) / (2 * d)
    h2 = r2 - (d * d + r2 * r2 - r1 * r1) / (2 * d)
    return 4 * math.pi * r1 * r1 - 2 * math.pi * r1 * h1, \
        4 * math.pi * r2 * r2 - 2 * math.pi * r2 * h2


def _fibonacci_sphere(n):
    k = np.arange(n) + 0.5
    z = 1 - 2 * k / n
    phi = k * math.pi * (3 - math.sqrt(5))
    s = np.sqrt(1 - z * z)
    return np.stack([s * np.cos(phi), s * np.sin(phi), z], axis=1)


def _quadrature_areas(xyz, r, npts=200_000):
    u = _fibonacci_sphere(npts)
    out = np.zeros(len(r))
    for i in range(len(r)):
        p = xyz[i] + r[i] * u
        free = np.ones(npts, dtype=bool)
        for j in range(len(r)):
            if j != i:
                free &= np.sum((p - xyz[j]) ** 2, axis=1) > r[j] * r[j]
        out[i] = 4 * math.pi * r[i] * r[i] * free.mean()
    return out


@pytest.mark.parametrize("seed", range(6))
def test_two_spheres_closed_form(seed):
    rng = np.random.default_rng(seed)
    r1, r2 = rng.uniform(1.2, 3.2, 2)
    d = rng.uniform(abs(r1 - r2) + 0.05, r1 + r2 - 0.05)
    v = rng.normal(size=3)
    c2 = d * v / np.linalg.norm(v)
    a, total = Oracle.esolan_spheres([[0, 0, 0], c2], [r1, r2])
    w1, w2 = _two_sphere_areas([0, 0, 0], r1, c2, r2)
    assert a[0] == pytest.approx(w1, rel=1e-12)
    assert a[1] == pytest.approx(w2, rel=1e-12)
    assert total == pytest.approx(w1 + w2, rel=1e-12)


def test_isolated_enclosed_and_disjoint_spheres():
    a, _ = Oracle.esolan_spheres([[0, 0, 0], [9, 0, 0]], [1.0, 2.0])
    assert a == pytest.approx([4 * math.pi, 16 * math.pi], rel=1e-15)
    a, _ = Oracle.esolan_spheres([[0, 0, 0], [0.2, 0.1, 0]], [3.0, 1.0])
    assert a[1] == 0.0 and a[0] == pytest.approx(36 * math.pi, rel=1e-15)


@pytest.mark.parametrize("seed", [1, 7, 4711])
def test_north_point_on_a_neighbour_takes_the_random_reorientation(seed):
    """The north point (0, 0, R) of sphere 1 lies on sphere 2 (|a| = 0 <
    1e-6): esolan.f re-orients the neighbours by two random angles; the
    area is the closed form whatever the draws."""
    R, r = 1.5, 1.0
    c2 = [1.0, 0.0, 1.5]   # |(0, 0, R) - c2| = 1.0 = r
    a, _ = Oracle.esolan_spheres([[0, 0, 0], c2], [R, r], seed=seed)
    w1, w2 = _two_sphere_areas([0, 0, 0], R, c2, r)
    assert a[0] == pytest.approx(w1, rel=1e-10)
    assert a[1] == pytest.approx(w2, rel=1e-10)


@pytest.mark.parametrize("seed", range(4))
def test_sphere_clusters_against_quadrature(seed):
    """Eight overlapping spheres (atomic radii plus the 1.4 A probe) in a
    small box, 1.5-70 % of each surface exposed: every sphere's area within
    0.05 % of its full area of a 200,000-point quadrature of the exposed
    surface (the agreement seen is 2e-5 to 8e-5)."""
    rng = np.random.default_rng(100 + seed)
    n = 8
    r = rng.uniform(2.6, 3.4, n)
    xyz = rng.uniform(0.0, 6.0, (n, 3))
    a, total = Oracle.esolan_spheres(xyz, r)
    q = _quadrature_areas(xyz, r)
    full = 4 * math.pi * r * r
    assert np.all(np.abs(a - q) <= 5e-4 * full), np.c_[a, q, full]
    assert total == pytest.approx(a.sum(), rel=1e-12)


def test_enkefa_analytic_and_numerical_solvation_agree():
    """Met-enkephalin with the OONS set: energy() with itysol = -1 (esolan)
    and itysol = 1 (enysol, 122-point quadrature) on the same conformations;
    the other terms are identical."""
    an = Oracle(DATA + "enkefa.seq", DATA + "enkefa.var", itysol=-1)
    nu = Oracle(DATA + "enkefa.seq", DATA + "enkefa.var", itysol=1)
    rng = np.random.default_rng(3)
    idvr = an.idvr() - 1
    confs = [an.vlvr().copy()]
    for _ in range(3):
        v = an.vlvr().copy()
        v[idvr] = v[idvr] + rng.normal(0.0, 0.15, len(idvr))
        confs.append(v)
    for v in confs:
        an.set_vlvr(v)
        nu.set_vlvr(v)
        ea, ta = an.energy()
        en, tn = nu.energy()
        assert np.array_equal(ta[:4], tn[:4])
        areas, _ = an.esolan_atoms()
        assert np.all(areas >= -1e-9)
        # numerical quadrature error of enysol: a few percent of the term
        assert abs(ta[4] - tn[4]) <= 0.03 * abs(tn[4]) + 0.2, (ta[4], tn[4])
        assert ea == pytest.approx(sum(ta[:4]) + ta[4], rel=1e-12)

"""Hand-computable pins of the numerical SASA (enysol.f:13-339).

enysol scales the npnt unit-sphere points of tes.dat (tessel, enysol.f:341-365)
onto every atom sphere and counts the points outside all neighbour spheres
(enysol.f:254-306); the area is 4 pi r^2 * count / npnt.  So:

* an isolated sphere keeps every point: area 4 pi r^2;
* of two spheres, each keeps the points outside the other, a count read off
  tes.dat directly, and as the spheres part the count rises to npnt;
* on a molecule the counts are those of the same point test over all
  neighbour pairs without the box decomposition.

The point sets here are parsed from tes.dat by this file, independently of
the oracle's reader.  The last test ties the oracle's sphere-set form to its
per-molecule enysol, which the GPU tests compare with the product."""
import ctypes
import math

import numpy as np
import pytest

from conftest import DATA, Oracle

TES = DATA + "tes.dat"


def _points():
    lines = [ln for ln in open(TES).read().splitlines() if not ln.startswith("!")]
    n = int(lines[0][:5])
    pts = np.array([[float(ln[20 * k:20 * k + 20]) for k in range(3)] for ln in lines[1:1 + n]])
    assert pts.shape == (n, 3)
    return pts


def _spheres(xyz, r, sigma=None):
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    r = np.ascontiguousarray(r, dtype=np.float64)
    n = len(r)
    sg = np.ascontiguousarray(np.ones(n) if sigma is None else sigma, dtype=np.float64)
    counts = np.zeros(n, dtype=np.int32)
    areas = np.zeros(n)
    eysl, asa = ctypes.c_double(), ctypes.c_double()
    L = Oracle.lib()
    L.orc_enysol_spheres.argtypes = [ctypes.c_int] + [ctypes.c_void_p] * 3 + [
        ctypes.c_char_p] + [ctypes.c_void_p] * 4
    rc = L.orc_enysol_spheres(n, xyz.ctypes.data, r.ctypes.data, sg.ctypes.data, TES.encode(),
                              counts.ctypes.data, areas.ctypes.data, ctypes.byref(eysl),
                              ctypes.byref(asa))
    assert rc == 0, L.orc_last_error()
    return counts, areas, eysl.value, asa.value


def _exposed(pts, ci, ri, others):
    """Points of sphere (ci, ri) outside every sphere of others [(c, r)], by
    the reference's scaled test: |(ci - c)/ri + p|^2 > (r/ri)^2."""
    keep = np.ones(len(pts), dtype=bool)
    for c, r in others:
        d = (np.asarray(ci, dtype=np.float64) - np.asarray(c, dtype=np.float64)) / ri
        dd = d[0] * d[0] + d[1] * d[1] + d[2] * d[2]
        ak = r / ri
        if not dd <= (1.0 + ak) * (1.0 + ak):
            continue   # not a neighbour
        t = d[None, :] + pts
        sdd = t[:, 0] * t[:, 0] + t[:, 1] * t[:, 1] + t[:, 2] * t[:, 2]
        keep &= ~(sdd <= ak * ak)
    return int(keep.sum())


def test_tes_points_lie_on_the_unit_sphere():
    pts = _points()
    assert len(pts) == 122
    assert np.allclose(np.linalg.norm(pts, axis=1), 1.0, atol=1e-8)


@pytest.mark.parametrize("r", [1.2, 1.7, 3.4])
def test_isolated_sphere_has_the_full_area(r):
    pts = _points()
    counts, areas, eysl, asa = _spheres([0.3, -1.1, 2.0], [r], [0.25])
    assert counts[0] == len(pts)
    assert areas[0] == pytest.approx(4.0 * math.pi * r * r, rel=1e-15)
    assert eysl == pytest.approx(0.25 * 4.0 * math.pi * r * r, rel=1e-15)
    assert asa == areas[0]


def test_far_apart_spheres_are_isolated():
    pts = _points()
    xyz = [[0, 0, 0], [10, 0, 0], [0, 10, 0], [0, 0, 10], [10, 10, 10]]
    r = [1.5, 2.0, 1.0, 1.8, 2.5]
    counts, areas, _, asa = _spheres(xyz, r)
    assert list(counts) == [len(pts)] * 5
    assert asa == pytest.approx(sum(4.0 * math.pi * q * q for q in r), rel=1e-14)


def test_zero_radius_spheres_take_no_part():
    counts, areas, _, _ = _spheres([[0, 0, 0], [0.5, 0, 0]], [1.5, 0.0])
    assert counts[1] == -1 and areas[1] == 0.0
    assert counts[0] == len(_points())


@pytest.mark.parametrize("r1,r2", [(1.5, 1.5), (1.2, 2.0), (2.0, 1.0)])
def test_two_spheres_count_from_tes_dat(r1, r2):
    pts = _points()
    npnt = len(pts)
    prev = -1
    for d in np.linspace(0.05, r1 + r2 + 0.2, 41):
        c1, c2 = np.array([0.1, 0.2, 0.3]), np.array([0.1 + d, 0.2 + 0.3 * d, 0.3 - 0.2 * d])
        dist = float(np.linalg.norm(c2 - c1))
        counts, areas, _, _ = _spheres([c1, c2], [r1, r2])
        want1 = _exposed(pts, c1, r1, [(c2, r2)])
        want2 = _exposed(pts, c2, r2, [(c1, r1)])
        assert (counts[0], counts[1]) == (want1, want2), d
        assert areas[0] == pytest.approx(4 * math.pi * r1 * r1 * want1 / npnt, rel=1e-15)
        # the exposed part of the smaller sphere grows as the spheres part ...
        if r1 <= r2:
            assert counts[0] >= prev
        prev = counts[0]
        # ... and follows the spherical cap it loses to sphere 2 (122 points
        # resolve the area to a few percent of the sphere)
        if dist >= r1 + r2:
            assert counts[0] == npnt
        elif dist + r1 <= r2:
            assert counts[0] == 0
        elif dist + r2 < r1:   # sphere 2 inside sphere 1
            assert counts[0] == npnt
        elif dist > abs(r1 - r2):
            h = (r2 * r2 - (dist - r1) ** 2) / (2.0 * dist)   # cap height on sphere 1
            assert counts[0] / npnt == pytest.approx(1.0 - h / (2.0 * r1), abs=0.06)
    assert prev == npnt


@pytest.mark.parametrize("seed", [None, 7, 19])
def test_molecule_counts_match_the_brute_force_test(seed):
    """Every heavy atom of Met-enkephalin: the box-sorted search finds the
    same neighbours and counts as the all-pairs point test."""
    o = Oracle(DATA + "enkefa.seq", DATA + "enkefa.var", itysol=1)
    if seed is not None:
        o.sgrnd(seed)
        o.random_start()
    o.energy()
    xyz = o.coords()
    rv, sg = np.zeros(o.natoms), np.zeros(o.natoms)
    L = o.lib()
    L.orc_get_solvation(o.h, rv.ctypes.data_as(ctypes.c_void_p), sg.ctypes.data_as(ctypes.c_void_p))
    counts, areas, eysl, _ = _spheres(xyz, rv, sg)
    pts = _points()
    heavy = np.nonzero(rv > 0)[0]
    assert len(heavy) > 30
    for i in heavy:
        others = [(xyz[j], rv[j]) for j in heavy if j != i]
        assert counts[i] == _exposed(pts, xyz[i], rv[i], others), i
    want = sum(sg[i] * 4 * math.pi * rv[i] ** 2 * counts[i] / len(pts) for i in heavy)
    assert eysl == pytest.approx(want, rel=1e-12)
    # the per-molecule enysol of the oracle is the same sum in the same order
    got = ctypes.c_double()
    L.orc_enysol.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    assert L.orc_enysol(o.h, 0, ctypes.byref(got)) == 0
    assert got.value == eysl

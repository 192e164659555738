"""Host-side assembly and flattening of the product library against the
oracle, on CPU (no GPU needed to build a molecule): atom, variable and pair
counts, and the free-variable order, for the molecules of every workload."""
import numpy as np
import pytest

from conftest import DATA, Oracle, seqfile


def _cases(tmp_path):
    from smmp.sequences import natural_protein, polyala
    yield "enkefa", DATA + "enkefa.seq", DATA + "enkefa.var", "ecepp3", 0
    yield "enkefa-ecepp2", DATA + "enkefa.seq", DATA + "enkefa.var", "ecepp2", 0
    for n in (10, 25, 40):
        yield "ala%d" % n, seqfile(tmp_path, polyala(n), "ala%d" % n), None, "ecepp3", 1
    yield "protein60", seqfile(tmp_path, natural_protein(60), "p60"), None, "ecepp3", 1


def test_host_topology_matches_oracle(tmp_path):
    from smmp.ensemble import Molecule
    for name, seq, var, ff, ity in _cases(tmp_path):
        m = Molecule(seq, var, libdir=DATA, ff=ff, itysol=ity)
        o = Oracle(seq, var, ff=ff, itysol=ity)
        assert m.natoms == o.natoms, name
        assert m.nvar == o.ntlvr, name
        assert m.nvr == o.nvr, name
        assert m.npairs == o.pair_count(), name
        assert np.array_equal(m.idvr, o.idvr() - 1), name


def test_sequences_are_seeded_and_valid():
    from smmp.sequences import NATURAL_COMPOSITION, natural_protein, polyala, polyala_lengths
    assert natural_protein(60) == natural_protein(60)
    p = natural_protein(60)
    assert len(p) == 60 and p[0] != "pro" and set(p) <= set(NATURAL_COMPOSITION)
    L = polyala_lengths(256)
    assert L == polyala_lengths(256) and min(L) >= 10 and max(L) <= 40 and len(L) == 256
    assert polyala(3) == ["ace", "ala", "ala", "ala", "nme"]
    assert abs(sum(NATURAL_COMPOSITION.values()) - 100.0) < 0.2   # rounded percentages


def test_moved_atoms_are_the_contiguous_variable_ranges(tmp_path):
    """The atoms a variable moves in the reference (its moving sets and,
    recursively, those of the variables added to it; setmvs.f) are exactly
    the contiguous range [var_lo, var_hi] the product rotates, so derivative
    sums over them are prefix-sum differences over atoms."""
    import ctypes
    from smmp.ensemble import Molecule
    for name, seq, var, ff, ity in _cases(tmp_path):
        m = Molecule(seq, var, libdir=DATA, ff=ff, itysol=ity)
        o = Oracle(seq, var, ff=ff, itysol=ity)
        lib = o.lib()
        lib.orc_moved_atoms.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int]
        cap = 2_000_000
        off = np.zeros(o.ntlvr + 1, np.int32)
        at = np.zeros(cap, np.int32)
        assert lib.orc_moved_atoms(o.h, off.ctypes.data_as(ctypes.c_void_p),
                                   at.ctypes.data_as(ctypes.c_void_p), cap) == 0
        for v in range(o.ntlvr):
            got = np.sort(at[off[v]:off[v + 1]]) - 1
            assert np.array_equal(got, np.arange(m.var_lo[v], m.var_hi[v] + 1)), (name, v)

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

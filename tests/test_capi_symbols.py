"""The C-ABI library loads without a GPU and exports every declared symbol."""
import ctypes
import os
import re

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "smmp_b200.h")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(smmp_[a-z0-9_]+)\s*\(", text)) - {"smmp_weight_fn"})


def test_header_declares_entry_points():
    names = declared()
    assert "smmp_energy" in names and "smmp_metropolis" in names and "smmp_ens_create" in names


def test_library_exports_every_declared_symbol():
    from smmp import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from smmp import _lib
    assert sorted(declared()) == sorted(_lib.EXPORTED)


def test_mol_build_runs_on_host():
    """Assembly is host work: building a molecule needs no GPU."""
    from smmp.ensemble import Molecule
    from conftest import DATA, Oracle
    m = Molecule(DATA + "enkefa.seq", DATA + "enkefa.var", libdir=DATA)
    o = Oracle(DATA + "enkefa.seq", DATA + "enkefa.var")
    assert (m.natoms, m.nvar, m.nvr) == (75, 24, 24)
    assert m.npairs == o.pair_count()

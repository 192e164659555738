"""outpdb (outpdb.f:12-185) on the CPU.  The reference ships no outpdb output,
so the text is checked against its FORMAT statements (outpdb.f:181-183) read
by PDB columns: 80-column lines, one ATOM/HETATM record per atom in atom order
with the oracle's coordinates, residue names and numbers, the hydrogen naming
rule, TER, and CONECT records that hold every bond of the build tree."""
import numpy as np

from conftest import DATA, Oracle, seqfile


def _pdb(seq, var=None):
    from smmp.ensemble import Molecule
    m = Molecule(seq, var, libdir=DATA)
    o = Oracle(seq, var)
    o.energy()   # setvar + bldmol
    xyz = o.coords().reshape(-1, 3)
    return m, o, xyz, m.outpdb(xyz)


def test_outpdb_columns_and_coordinates():
    m, o, xyz, text = _pdb(DATA + "enkefa.seq", DATA + "enkefa.var")
    lines = text.split("\n")[:-1]
    assert all(len(line) == 80 for line in lines)
    atoms = [line for line in lines if line[:6] in ("ATOM  ", "HETATM")]
    assert len(atoms) == m.natoms
    for k, line in enumerate(atoms):
        assert int(line[6:11]) == k + 1
        got = [float(line[30:38]), float(line[38:46]), float(line[46:54])]
        assert np.allclose(got, xyz[k], atol=5e-4)
        assert line[54:60] == "  1.00" and line[60:66] == "  0.00"
        assert line[21] == " " and line[26] == " "
    # nh2/cooh end groups: every residue of the deck is an ATOM record
    assert atoms[0][:6] == "ATOM  " and atoms[0][17:20] == "TYR"
    assert int(atoms[-1][22:26]) == 5 and atoms[-1][17:20] == "MET"
    ter = [line for line in lines if line.startswith("TER")]
    assert len(ter) == 1 and int(ter[0][6:11]) == m.natoms + 1 and ter[0][17:20] == "MET"
    assert lines[-1].rstrip() == "END"
    # hydrogens: a trailing digit of the name moves to column 13
    names = [line[12:16] for line in atoms]
    for nm in names:
        assert nm == nm.upper()
        if nm[0].isdigit():
            assert nm[1] == "H"


def test_outpdb_conect_is_the_oracle_bond_table():
    """CONECT lists, for every atom with bonds, its bonded partners after it
    (outpdb.f:137-176), taken here from the oracle's atom table."""
    m, o, xyz, text = _pdb(DATA + "enkefa.seq", DATA + "enkefa.var")
    got = {}
    for line in text.split("\n"):
        if line.startswith("CONECT"):
            i = int(line[6:11])
            got[i] = [int(line[k:k + 5]) for k in range(11, 31, 5) if line[k:k + 5].strip()]
    ai = o.atom_table()
    want = {}
    for i in range(1, m.natoms + 1):
        iow, nbd, b1, b2, b3 = ai[i - 1, 1], ai[i - 1, 2], ai[i - 1, 3], ai[i - 1, 4], ai[i - 1, 5]
        if nbd <= 0:
            continue
        ibd = [iow, b1, b2, b3] if i == 1 else [b1, b2, b3]
        js = [j for j in ibd if j > i]
        if js:
            want[i] = js
    assert got == want
    for i, js in got.items():   # bonded atoms are 0.9-2.0 A apart
        for j in js:
            d = np.linalg.norm(xyz[i - 1] - xyz[j - 1])
            assert 0.9 < d < 2.0, (i, j, d)


def test_outpdb_caps_are_hetatm(tmp_path):
    """ace and nme residues are HETATM records (outpdb.f:92-96)."""
    from smmp.sequences import polyala
    m, o, xyz, text = _pdb(seqfile(tmp_path, polyala(3), "ala3"))
    recs = [(line[:6], line[17:20]) for line in text.split("\n")
            if line[:6] in ("ATOM  ", "HETATM")]
    assert {r for t, r in recs if t == "HETATM"} == {"ACE", "NME"}
    assert {r for t, r in recs if t == "ATOM  "} == {"ALA"}

"""The product's molecule builder (smmp-svn_b200/csrc/molbuild.cpp) against
the oracle's restatement of getmol/addend/setmvs/mklist/redvar, field by
field, and its pair set against an independent geometric classification
(CPU only; building a molecule needs no GPU).

For every molecule: the tree (parents), classes, charges, bond lengths,
valence angles and the dihedral state the variable file leaves; the variables
(primary atoms, classes, fixed flags, free order, values); the interaction
lists pair for pair, normal and 1-4 separately, each under the same listing
atom as mklist.f; and both lists against brute force: turning each variable
alone on the oracle's own rebuild, a pair whose distance some variable
changes is an interaction pair, and every 1-4 pair is one that exactly one
variable changes.
"""
import numpy as np
import pytest

from conftest import DATA, Oracle, seqfile


def _write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def _cases(tmp_path):
    """(name, seq, var, ff, itysol, grpn, grpc): every workload molecule plus
    every terminal-group rule and each residue type of the library."""
    from smmp.sequences import natural_protein, polyala
    yield "enkefa", DATA + "enkefa.seq", DATA + "enkefa.var", "ecepp3", 0, "nh2", "cooh"
    yield "enkefa-ecepp2", DATA + "enkefa.seq", DATA + "enkefa.var", "ecepp2", 0, "nh2", "cooh"
    yield "enkefa-ann", DATA + "enkefa.seq", DATA + "enkefa.ann", "ecepp2", 0, "nh2", "cooh"
    for n in (10, 25, 40):
        yield "ala%d" % n, seqfile(tmp_path, polyala(n), "ala%d" % n), None, "ecepp3", 1, "nh2", "cooh"
    yield "protein60", seqfile(tmp_path, natural_protein(60), "p60"), None, "ecepp3", 1, "nh2", "cooh"
    # charged ends, glycine and proline at the ends, a single residue
    yield "gly-ends", seqfile(tmp_path, ["gly", "ala", "gly"], "g"), None, "ecepp3", 0, "nh3+", "coo-"
    yield "gly-ends-cooh", seqfile(tmp_path, ["gly", "ser", "gly"], "g2"), None, "ecepp3", 0, "nh2", "cooh"
    yield "gly-ecepp2", seqfile(tmp_path, ["gly", "ala", "gly"], "g3"), None, "ecepp2", 0, "nh2", "coo-"
    yield "hyp-ecepp2", seqfile(tmp_path, ["hyp", "ala", "prom"], "h2"), None, "ecepp2", 0, "nh2", "cooh"
    yield "pro-first", seqfile(tmp_path, ["pro", "ala", "pro", "gly"], "pf"), None, "ecepp3", 0, "nh2", "cooh"
    yield "pro-first-nh3", seqfile(tmp_path, ["pro", "trp", "his"], "pn"), None, "ecepp3", 0, "nh3+", "coo-"
    yield "single", seqfile(tmp_path, ["ala"], "one"), None, "ecepp3", 0, "nh2", "cooh"
    # every other residue of lib.sh3, charged forms included
    every = ["arg", "arg+", "asn", "asp", "asp-", "cys", "cyss", "gln", "glu", "glu-", "his",
             "hise", "his+", "hyp", "ile", "leu", "lys", "lys+", "met", "phe", "ser", "thr", "trp",
             "tyr", "val", "cpro", "cpru", "prou"]
    yield "every", seqfile(tmp_path, ["ace"] + every + ["nme"], "every"), None, "ecepp3", 1, "nh2", "cooh"
    # variable-file grammar: global parameters, zones, wildcards, fixing
    var = _write(tmp_path, "g.var",
                 "@ 1.5, -2.0, 0.25, 30.0, -20.0, 100.0\n"
                 "1-2 : phi,psi : -65 ; 3- : x* : 60\n"
                 "  : om* : 175.5 &\n"
                 "4 : 1 : 45\n"
                 "Phe : x2 : -90\n")
    yield "varfile", DATA + "enkefa.seq", var, "ecepp3", 0, "nh2", "cooh"


def _oracle_pairs(o):
    ai, ad, vi, ms, vw, l14 = o.topology()
    normal = set()
    for j1, j2, i in vw:
        for j in range(j1, j2 + 1):
            normal.add((i - 1, j - 1))
    one4 = {(i - 1, j - 1) for j, i in l14}
    return normal, one4


def _product_pairs(m):
    p = m.pairs()
    normal = {(int(i), int(j)) for i, j, k in p if k == 0}
    one4 = {(int(i), int(j)) for i, j, k in p if k == 1}
    return normal, one4


def _wrap(a):
    return (a + np.pi) % (2 * np.pi) - np.pi


@pytest.fixture(scope="module")
def built(tmp_path_factory):
    from smmp.ensemble import Molecule
    tmp = tmp_path_factory.mktemp("mb")
    out = []
    for name, seq, var, ff, ity, gn, gc in _cases(tmp):
        m = Molecule(seq, var, libdir=DATA, ff=ff, itysol=ity, grpn=gn, grpc=gc)
        o = Oracle(seq, var, ff=ff, itysol=ity, grpn=gn, grpc=gc)
        out.append((name, m, o))
    return out


def test_atoms_match_the_oracle(built):
    for name, m, o in built:
        assert m.natoms == o.natoms, name
        ai, ad, vi, _, _, _ = o.topology()
        par, typ, chg, geom = m.atoms()
        assert par[0] == -1, name
        assert np.array_equal(par[1:], ai[1:, 1] - 1), name          # iowat
        assert np.array_equal(typ, ai[:, 0]), name                   # ityat
        assert np.array_equal(chg, ad[:, 0]), name                   # cgat, bit for bit
        assert np.array_equal(geom[:, 0], ad[:, 1]), name            # blat, bit for bit
        # baat (the first atom's is never used) and the dihedral state
        np.testing.assert_allclose(geom[1:, 1], ad[1:, 2], rtol=0, atol=1e-13, err_msg=name)
        np.testing.assert_allclose(_wrap(geom[:, 2] - ad[:, 3]), 0.0, atol=1e-13, err_msg=name)


def test_variables_match_the_oracle(built):
    for name, m, o in built:
        ai, ad, vi, _, _, _ = o.topology()
        assert m.nvar == o.ntlvr and m.nvr == o.nvr, name
        v = m.variables()
        assert np.array_equal(v[:, 0], vi[:, 0] - 1), name     # iatvr
        assert np.array_equal(v[:, 1], vi[:, 2]), name         # iclvr
        assert np.array_equal(v[:, 2], vi[:, 8]), name         # fxvr
        assert np.array_equal(m.idvr, o.idvr() - 1), name
        np.testing.assert_allclose(_wrap(m.vlvr0 - o.vlvr()), 0.0, atol=1e-13, err_msg=name)


def test_pair_lists_match_mklist(built):
    """Pair for pair, each under the atom mklist.f lists it, 1-4 separately."""
    for name, m, o in built:
        n_o, f_o = _oracle_pairs(o)
        n_p, f_p = _product_pairs(m)
        assert len(n_p) + len(f_p) == m.npairs, name             # no pair twice
        assert f_p == f_o, (name, sorted(f_p ^ f_o)[:10])
        assert n_p == n_o, (name, sorted(n_p ^ n_o)[:10])
        assert m.npairs == o.pair_count(), name


def _brute_force(o, seed=7):
    """Unordered pairs whose distance changes when each variable turns alone
    (oracle rebuild, valence angles perturbed by up to 0.1 rad so that no
    atom sits on a rotation axis it is not bonded along), with the number of
    variables that change each."""
    import ctypes
    o.lib().orc_perturb_valence.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_double]
    o.lib().orc_perturb_valence(o.h, seed, 0.1)
    rng = np.random.default_rng(seed)
    v0 = o.vlvr() + rng.uniform(-0.3, 0.3, o.ntlvr)   # a generic conformation
    o.set_vlvr(v0)
    o.energy()
    x0 = o.coords()
    d0 = np.linalg.norm(x0[:, None, :] - x0[None, :, :], axis=-1)
    count = np.zeros(d0.shape, np.int32)
    for k in range(o.ntlvr):
        v = v0.copy()
        v[k] += 1.1
        o.set_vlvr(v)
        o.energy()
        x = o.coords()
        d = np.linalg.norm(x[:, None, :] - x[None, :, :], axis=-1)
        count += (np.abs(d - d0) > 1e-7).astype(np.int32)
    o.set_vlvr(v0)
    iu = np.triu_indices(len(x0), 1)
    c = count[iu]
    pairs = {(int(i), int(j)) for i, j in zip(iu[0][c > 0], iu[1][c > 0])}
    one4 = {(int(i), int(j)) for i, j in zip(iu[0][c == 1], iu[1][c == 1])}
    return pairs, one4


def test_pair_set_equals_geometric_classification(built):
    """Interaction pairs = pairs whose distance some variable changes (so no
    bonded or 1-3 pair, whose distances are fixed); every 1-4 pair is one
    that exactly one variable changes (the reference's 1-4 set is the part
    of those around the turning bond, mklist.f:96-207)."""
    for name, m, o in built:
        if name == "every":
            continue   # covered residue by residue in the lists test; brute force is slow here
        n_p, f_p = _product_pairs(m)
        und = lambda s: {(min(a), max(a)) for a in s}
        allp, one4 = _brute_force(o.clone())
        assert und(n_p) | und(f_p) == allp, name
        assert und(f_p) <= one4, name


def test_moving_ranges_match_setmvs(built):
    """The atoms each variable moves (setmvs.f moving sets plus those of its
    added variables) are the contiguous range the product rotates."""
    import ctypes
    for name, m, o in built:
        lib = o.lib()
        lib.orc_moved_atoms.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int]
        cap = 4_000_000
        off = np.zeros(o.ntlvr + 1, np.int32)
        at = np.zeros(cap, np.int32)
        assert lib.orc_moved_atoms(o.h, off.ctypes.data_as(ctypes.c_void_p),
                                   at.ctypes.data_as(ctypes.c_void_p), cap) == 0
        for v in range(o.ntlvr):
            got = np.sort(at[off[v]:off[v + 1]]) - 1
            assert np.array_equal(got, np.arange(m.var_lo[v], m.var_hi[v] + 1)), (name, v)


def test_builder_rejects_bad_input(tmp_path):
    from smmp import SmmpError
    from smmp.ensemble import Molecule
    bad = [
        (["ala", "ace", "ala"], "nh2", "cooh", "allowed at N-terminus only"),
        (["nme", "ala"], "nh2", "cooh", "allowed at C-terminus only"),
        (["ala", "xyz"], "nh2", "cooh", "NOT FOUND"),
        (["ala"], "ace", "cooh", "SEQUENCE file"),
        (["ala"], "nh4", "cooh", "nh2 or nh3+"),
        (["ala"], "nh2", "cooo", "cooh or coo-"),
        (["hyp", "ala"], "nh2", "cooh", "Hyp"),
    ]
    for k, (res, gn, gc, msg) in enumerate(bad):
        with pytest.raises(SmmpError) as ei:
            Molecule(seqfile(tmp_path, res, "bad%d" % k), None, libdir=DATA, grpn=gn, grpc=gc)
        assert msg in str(ei.value), (res, str(ei.value))
    var = _write(tmp_path, "bad.var", "1 : phi : abc\n")
    with pytest.raises(SmmpError) as ei:
        Molecule(DATA + "enkefa.seq", var, libdir=DATA)
    assert "Cannot read value" in str(ei.value)
    var = _write(tmp_path, "bad2.var", "9 : phi : 10\n")
    with pytest.raises(SmmpError) as ei:
        Molecule(DATA + "enkefa.seq", var, libdir=DATA)
    assert "Error in identifier" in str(ei.value)

"""Shared fixtures: paths, the CPU oracle (checker) and the product package.

The oracle under oracle/ is test infrastructure: tests load it through ctypes
to check the product's results; the product never loads it.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "smmp-svn_b200")
DATA = os.path.join(ROOT, "tests", "golden", "smmp_data") + "/"
GOLDEN = os.path.join(ROOT, "tests", "golden", "golden.json")
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle_smmp.so")

if PKG not in sys.path:
    sys.path.insert(0, PKG)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "slow: runs for more than a few seconds")


def _have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAVE_GPU = _have_gpu()


def pytest_collection_modifyitems(config, items):
    if HAVE_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA GPU in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


# ------------------------------------------------------------------ oracle
def _build_oracle():
    if not os.path.exists(ORACLE_SO):
        subprocess.check_call(["make", "-C", os.path.join(ROOT, "oracle")])


class Oracle:
    """ctypes wrapper over oracle/liboracle_smmp.so (one system per object)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            _build_oracle()
            L = ctypes.CDLL(ORACLE_SO)
            L.orc_create.restype = ctypes.c_void_p
            L.orc_create.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
            L.orc_clone.restype = ctypes.c_void_p
            L.orc_clone.argtypes = [ctypes.c_void_p]
            L.orc_last_error.restype = ctypes.c_char_p
            L.orc_grnd.restype = ctypes.c_double
            L.orc_grnd.argtypes = [ctypes.c_void_p]
            L.orc_set_beta.argtypes = [ctypes.c_void_p, ctypes.c_double]
            L.orc_anneal.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
            L.orc_bench_chains.restype = ctypes.c_double
            L.orc_bench_chains.argtypes = [ctypes.c_void_p, ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_int),
                                           ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                                           ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
            for f in ["orc_init_molecule", "orc_energy", "orc_sizes", "orc_sweeps",
                      "orc_sgrnd", "orc_random_start", "orc_get_vlvr", "orc_set_vlvr",
                      "orc_get_idvr", "orc_get_coords", "orc_get_topology", "orc_partem",
                      "orc_get_mt", "orc_destroy", "orc_get_toat", "orc_set_rndord",
                      "orc_get_axvr", "orc_get_names"]:
                getattr(L, f).argtypes = None
            L.orc_esolan_spheres.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
            L.orc_esolan_atoms.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
            L.orc_gradient.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
            L.orc_minim.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                    ctypes.c_void_p]
            cls._lib = L
        return cls._lib

    def gradient(self):
        """gradient.f: (energy, dE/dvlvr of every variable)."""
        e = ctypes.c_double()
        g = np.zeros(self.ntlvr)
        rc = self.lib().orc_gradient(self.h, ctypes.byref(e), g.ctypes.data_as(ctypes.c_void_p))
        assert rc == 0, self.lib().orc_last_error()
        return e.value, g

    def minim(self, imin=1, maxit=10000, eps=1e-9):
        """minim.f: (function calls, [(energy, |grad|^2) of every call])."""
        nop, nlog = ctypes.c_int(), ctypes.c_int()
        cap = 100000
        log = np.zeros(2 * cap)
        rc = self.lib().orc_minim(self.h, int(imin), int(maxit), float(eps), ctypes.byref(nop),
                                  log.ctypes.data_as(ctypes.c_void_p), cap, ctypes.byref(nlog))
        assert rc == 0, self.lib().orc_last_error()
        return nop.value, log[:2 * min(nlog.value, cap)].reshape(-1, 2)

    @classmethod
    def esolan_spheres(cls, xyz, radii, seed=1):
        """esolan.f area arithmetic on free spheres: (areas, total)."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        r = np.ascontiguousarray(radii, dtype=np.float64)
        a = np.zeros(len(r))
        t = ctypes.c_double()
        rc = cls.lib().orc_esolan_spheres(len(r), xyz.ctypes.data, r.ctypes.data, int(seed),
                                          a.ctypes.data, ctypes.byref(t))
        assert rc == 0, cls.lib().orc_last_error()
        return a, t.value

    def esolan_atoms(self):
        """Analytic SASA of every atom of the current conformation."""
        a = np.zeros(self.natoms)
        t = ctypes.c_double()
        rc = self.lib().orc_esolan_atoms(self.h, a.ctypes.data, ctypes.byref(t))
        assert rc == 0, self.lib().orc_last_error()
        return a, t.value

    def __init__(self, seq, var=None, ff="ecepp3", itysol=0, epsd=0, grpn="nh2", grpc="cooh",
                 _handle=None):
        L = self.lib()
        if _handle is not None:
            self.h = ctypes.c_void_p(_handle)
        else:
            h = L.orc_create(DATA.encode(), 1 if ff == "ecepp2" else 0, int(epsd), int(itysol))
            assert h, L.orc_last_error()
            self.h = ctypes.c_void_p(h)
            rc = L.orc_init_molecule(self.h, seq.encode(), (var or " ").encode(), grpn.encode(),
                                     grpc.encode())
            assert rc == 0, L.orc_last_error()
        sz = (ctypes.c_int * 7)()
        L.orc_sizes(self.h, sz)
        self.natoms, self.ntlvr, self.nvr = sz[0], sz[1], sz[2]
        self.sizes = list(sz)

    def clone(self):
        return Oracle(None, _handle=self.lib().orc_clone(self.h))

    def energy(self):
        e = ctypes.c_double()
        t = (ctypes.c_double * 6)()
        rc = self.lib().orc_energy(self.h, ctypes.byref(e), t)
        assert rc == 0, self.lib().orc_last_error()
        return e.value, list(t)

    def vlvr(self):
        a = np.zeros(self.ntlvr)
        self.lib().orc_get_vlvr(self.h, a.ctypes.data_as(ctypes.c_void_p))
        return a

    def set_vlvr(self, v):
        a = np.ascontiguousarray(v, dtype=np.float64)
        self.lib().orc_set_vlvr(self.h, a.ctypes.data_as(ctypes.c_void_p))

    def idvr(self):
        a = np.zeros(self.nvr, dtype=np.int32)
        self.lib().orc_get_idvr(self.h, a.ctypes.data_as(ctypes.c_void_p))
        return a

    def toat(self):
        a = np.zeros(self.natoms)
        self.lib().orc_get_toat(self.h, a.ctypes.data_as(ctypes.c_void_p))
        return a

    def coords(self):
        a = np.zeros(3 * self.natoms)
        self.lib().orc_get_coords(self.h, a.ctypes.data_as(ctypes.c_void_p))
        return a.reshape(-1, 3)

    def sgrnd(self, seed):
        self.lib().orc_sgrnd(self.h, ctypes.c_int(seed))

    def grnd(self):
        return self.lib().orc_grnd(self.h)

    def set_beta(self, b):
        self.lib().orc_set_beta(self.h, b)

    def random_start(self):
        self.lib().orc_random_start(self.h)

    def sweeps(self, n, log=None):
        eol, acz = ctypes.c_double(), ctypes.c_double()
        ptr = log.ctypes.data_as(ctypes.c_void_p) if log is not None else None
        rc = self.lib().orc_sweeps(self.h, ctypes.c_int(n), ctypes.byref(eol), ctypes.byref(acz),
                                   ptr)
        assert rc == 0, self.lib().orc_last_error()
        return eol.value, acz.value

    def atom_table(self):
        """Per atom (1-based atom numbers): ityat, iowat, nbdat, ibdat(1..3), ..."""
        na, nv = self.natoms, self.ntlvr
        ai = np.zeros((na, 11), np.int32)
        ad = np.zeros((na, 4))
        vi = np.zeros((nv, 9), np.int32)
        ms = np.zeros((self.sizes[6], 2), np.int32)
        vw = np.zeros((self.sizes[4], 3), np.int32)
        l14 = np.zeros((self.sizes[5], 2), np.int32)
        P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        self.lib().orc_get_topology(self.h, P(ai), P(ad), P(vi), P(ms), P(vw), P(l14))
        return ai

    def partem_batched(self, betas, seeds, exchange_seed, wrap, nrounds, nthreads=8):
        """Batched parallel tempering (oracle/oracle_capi.cpp orc_partem_batched):
        per-round histories (chain at each label, energies, free variables)
        and the per-pair (attempts, accepts)."""
        n = len(betas)
        L = self.lib()
        L.orc_partem_batched.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        b = np.ascontiguousarray(betas, dtype=np.float64)
        sd = np.ascontiguousarray(seeds, dtype=np.int32)
        tc = np.zeros((nrounds, n), np.int32)
        eo = np.zeros((nrounds, n))
        vl = np.zeros((nrounds, n, self.nvr))
        st = np.zeros(2 * n, np.uint64)
        rc = L.orc_partem_batched(self.h, n, b.ctypes.data, sd.ctypes.data, int(exchange_seed),
                                  int(bool(wrap)), int(nrounds), int(nthreads), tc.ctypes.data,
                                  eo.ctypes.data, vl.ctypes.data, st.ctypes.data)
        assert rc == 0, L.orc_last_error()
        return tc, eo, vl, (st[0::2], st[1::2])

    def topology(self):
        """All of orc_get_topology: (atom_i [n,11], atom_d [n,4], var_i [nv,9],
        moving sets [nms,2], vdW domains [nvw,3], 1-4 entries [n14,2]);
        1-based values as in the reference arrays."""
        na, nv = self.natoms, self.ntlvr
        ai = np.zeros((na, 11), np.int32)
        ad = np.zeros((na, 4))
        vi = np.zeros((nv, 9), np.int32)
        ms = np.zeros((max(self.sizes[6], 1), 2), np.int32)
        vw = np.zeros((max(self.sizes[4], 1), 3), np.int32)
        l14 = np.zeros((max(self.sizes[5], 1), 2), np.int32)
        P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        self.lib().orc_get_topology(self.h, P(ai), P(ad), P(vi), P(ms), P(vw), P(l14))
        return ai, ad, vi, ms[:self.sizes[6]], vw[:self.sizes[4]], l14[:self.sizes[5]]

    def pair_count(self):
        na, nv = self.natoms, self.ntlvr
        ai = np.zeros((na, 11), np.int32)
        ad = np.zeros((na, 4))
        vi = np.zeros((nv, 9), np.int32)
        ms = np.zeros((self.sizes[6], 2), np.int32)
        vw = np.zeros((self.sizes[4], 3), np.int32)
        l14 = np.zeros((self.sizes[5], 2), np.int32)
        P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        self.lib().orc_get_topology(self.h, P(ai), P(ad), P(vi), P(ms), P(vw), P(l14))
        return int((vw[:, 1] - vw[:, 0] + 1).sum()) + len(l14)


def seqfile(tmp_path, residues, name="chain"):
    """Write a sequence file with the given residue names."""
    p = tmp_path / (name + ".seq")
    p.write_text("# %s\n%s\n" % (name, " ".join(residues)))
    return str(p)


@pytest.fixture
def oracle_cls():
    return Oracle

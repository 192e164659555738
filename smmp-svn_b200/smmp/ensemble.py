"""Batched chains and replicas on the GPU (layer 2 of include/smmp_b200.h).

A :class:`Molecule` is one sequence assembled from a residue library (the work
of init_energy + init_molecule); an :class:`Ensemble` holds many chains, each a
copy of one of its molecules with its own variables, dihedral state, MT19937
stream and inverse temperature, all resident on the GPU.  Chains of different
sequences (uneven lengths) can share one ensemble and one launch.

    mol = Molecule('enkefa.seq', libdir='SMMP/')
    ens = Ensemble([mol], [0] * 64, seeds=[31433 + 1000 * k for k in range(64)],
                   betas=betas)
    ens.random_start()
    ens.set_pt(betas)                  # parallel tempering (partem_s.f)
    ens.pt_sweeps(1000)
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import check, lib

GAS_CONSTANT = 1.98773e-3   # kcal/(mol K), canon.f:57 and partem_s.f:36

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def beta_of(temperature):
    """1/(T*R) as canon.f:57 computes it."""
    return 1.0 / (temperature * GAS_CONSTANT)


class Molecule:
    """One sequence (+ optional .var file) assembled on the host."""

    def __init__(self, seqfile, varfile=None, libdir="SMMP/", ff="ecepp3", itysol=0, epsd=0,
                 grpn="nh2", grpc="cooh"):
        cfg = _lib.Config(sh2=1 if ff == "ecepp2" else 0, epsd=int(epsd), itysol=int(itysol),
                          ientyp=0, rndord=0, upchswitch=0)
        if ff not in ("ecepp2", "ecepp3"):
            raise ValueError("force field must be ecepp2 or ecepp3 on this path")
        h = lib.smmp_mol_build(libdir.encode(), ctypes.byref(cfg), seqfile.encode(),
                               (varfile or "").encode(), grpn.encode(), grpc.encode())
        if not h:
            raise _lib.SmmpError(2, lib.smmp_last_error().decode())
        self._h = ctypes.c_void_p(h)
        info = (ctypes.c_longlong * 6)()
        check(lib.smmp_mol_info(self._h, info))
        self.natoms, self.nvar, self.nvr, self.npairs, self.nheavy, self.nres = list(info)
        self.itysol = itysol
        idvr = np.zeros(max(self.nvr, 1), dtype=np.int32)
        check(lib.smmp_mol_idvr(self._h, idvr.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        self.idvr = idvr[:self.nvr]          # 0-based variable index of each free dihedral
        v0 = np.zeros(max(self.nvar, 1))
        check(lib.smmp_mol_vlvr0(self._h, v0.ctypes.data_as(_D)))
        self.vlvr0 = v0[:self.nvar]          # variables as built (library, then .var file)
        lo = np.zeros(max(self.nvar, 1), dtype=np.int32)
        hi = np.zeros(max(self.nvar, 1), dtype=np.int32)
        check(lib.smmp_mol_var_ranges(self._h, lo.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                      hi.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        self.var_lo, self.var_hi = lo[:self.nvar], hi[:self.nvar]   # atoms each variable moves

    def atoms(self):
        """Per atom (0-based): parent (-1 for the first atom), ECEPP class,
        charge, and [bond length, valence angle, dihedral, solvation radius]."""
        n = self.natoms
        par = np.zeros(n, np.int32)
        typ = np.zeros(n, np.int32)
        chg = np.zeros(n)
        geom = np.zeros((n, 4))
        ip = ctypes.POINTER(ctypes.c_int)
        check(lib.smmp_mol_atoms(self._h, par.ctypes.data_as(ip), typ.ctypes.data_as(ip),
                                 chg.ctypes.data_as(_D), geom.ctypes.data_as(_D)))
        return par, typ, chg, geom

    def variables(self):
        """Per variable: primary atom (0-based), torsion class, fixed, residue."""
        out = np.zeros((max(self.nvar, 1), 4), np.int32)
        check(lib.smmp_mol_vars(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        return out[:self.nvar]

    def pairs(self):
        """The interaction lists: rows (listing atom, partner, 1 if 1-4)."""
        out = np.zeros((max(self.npairs, 1), 3), np.int32)
        check(lib.smmp_mol_pairs(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        return out[:self.npairs]

    def outvar(self, vlvr, iml=1):
        """Text of outvar.f (outvbs, outvar.f:50-121) for the variables vlvr
        (radians, all nvar of them); iml is the molecule number printed."""
        v = np.ascontiguousarray(vlvr, dtype=np.float64)
        if len(v) < self.nvar:
            raise ValueError("vlvr needs all %d variables" % self.nvar)
        n = ctypes.c_uint64(0)
        check(lib.smmp_mol_outvar(self._h, v.ctypes.data_as(_D), int(iml), None, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        check(lib.smmp_mol_outvar(self._h, v.ctypes.data_as(_D), int(iml), buf, ctypes.byref(n)))
        return buf.value.decode()

    def outpdb(self, xyz):
        """PDB text of outpdb.f (outpdb.f:12-185) for coordinates xyz
        (natoms x 3, Angstrom)."""
        x = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1)
        if len(x) < 3 * self.natoms:
            raise ValueError("xyz needs %d atoms" % self.natoms)
        n = ctypes.c_uint64(0)
        check(lib.smmp_mol_outpdb(self._h, x.ctypes.data_as(_D), None, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        check(lib.smmp_mol_outpdb(self._h, x.ctypes.data_as(_D), buf, ctypes.byref(n)))
        return buf.value.decode()

    def __del__(self):
        if getattr(self, "_h", None):
            lib.smmp_mol_free(self._h)
            self._h = None


class Ensemble:
    """Chains of molecules on the GPU.

    chain_mol[c] selects the molecule of chain c; betas[c] its inverse
    temperature; seeds[c] the seed of its MT19937 stream (shared_stream=True:
    one stream seeds[0] consumed by all chains in turn, as partem_s.f does).
    fp32=True evaluates pair terms in FP32 with FP64 guard and accumulation.
    """

    def __init__(self, molecules, chain_mol, seeds, betas, shared_stream=False, fp32=False,
                 rndord=False):
        self.molecules = list(molecules)
        chain_mol = np.ascontiguousarray(chain_mol, dtype=np.int32)
        seeds = np.ascontiguousarray(seeds, dtype=np.int32)
        betas = np.ascontiguousarray(betas, dtype=np.float64)
        n = len(chain_mol)
        if len(betas) != n:
            raise ValueError("one beta per chain")
        if len(seeds) != (1 if shared_stream else n):
            raise ValueError("one seed per stream")
        handles = (ctypes.c_void_p * len(self.molecules))(*[m._h.value for m in self.molecules])
        flags = (2 if fp32 else 0) | (1 if rndord else 0)
        h = lib.smmp_ens_create(handles, len(self.molecules), chain_mol.ctypes.data_as(_I), n,
                                seeds.ctypes.data_as(_I), betas.ctypes.data_as(_D),
                                int(bool(shared_stream)), flags)
        if not h:
            raise _lib.SmmpError(3, lib.smmp_last_error().decode())
        self._h = ctypes.c_void_p(h)
        nc, vs, ts = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(lib.smmp_ens_sizes(self._h, ctypes.byref(nc), ctypes.byref(vs), ctypes.byref(ts)))
        self.nchains, self.vstride, self.tstride = nc.value, vs.value, ts.value
        self.chain_mol = chain_mol
        self.shared_stream = bool(shared_stream)
        self.fp32 = bool(fp32)

    def __del__(self):
        if getattr(self, "_h", None):
            lib.smmp_ens_free(self._h)
            self._h = None

    def set_stream(self, stream):
        """Run on a caller's CUDA stream (an int handle, e.g.
        torch.cuda.current_stream().cuda_stream); None restores the own stream."""
        check(lib.smmp_ens_set_stream(self._h, ctypes.c_void_p(stream) if stream else None))

    # ---------------------------------------------------------------- driving
    def random_start(self):
        check(lib.smmp_ens_random_start(self._h))

    def energy(self):
        out = np.zeros(self.nchains)
        check(lib.smmp_ens_energy(self._h, out.ctypes.data_as(_D)))
        return out

    def equilibrate(self, nequi):
        """energy() then nequi sweeps of each chain at its own beta, chains in
        order (partem_s.f:134-162)."""
        check(lib.smmp_ens_equilibrate(self._h, int(nequi)))

    def sweeps(self, n, weight=None):
        w = weight._struct() if weight is not None else None
        check(lib.smmp_ens_sweeps(self._h, int(n), ctypes.byref(w) if w is not None else None))

    def set_pt(self, betas, wrap=True, exchange_seed=4711):
        b = np.ascontiguousarray(betas, dtype=np.float64)
        if len(b) != self.nchains:
            raise ValueError("one temperature label per chain")
        check(lib.smmp_ens_set_pt(self._h, b.ctypes.data_as(_D), int(bool(wrap)),
                                  int(exchange_seed)))

    def pt_sweeps(self, n, serial=False, graph_chunk=64):
        check(lib.smmp_ens_pt_sweeps(self._h, int(n), int(bool(serial)), int(graph_chunk)))

    def set_pt_fused(self, on=True, timeout_s=30.0, barrier_extra=0):
        """Batched pt_sweeps as one cooperative launch (default) or as CUDA
        graphs of separate sweep and exchange launches; both give the same
        bits.  A grid-barrier wait longer than timeout_s ends the run with
        error code 4 on the chains that waited; barrier_extra > 0 (tests only)
        makes the barriers wait for arrivals that never come."""
        check(lib.smmp_ens_set_pt_fused(self._h, int(bool(on)), float(timeout_s),
                                        int(barrier_extra)))

    def pt_fused_last(self):
        v = ctypes.c_int(0)
        check(lib.smmp_ens_pt_fused_last(self._h, ctypes.byref(v)))
        return bool(v.value)

    def pt_map(self):
        out = np.zeros(self.nchains, dtype=np.int32)
        check(lib.smmp_ens_pt_map(self._h, out.ctypes.data_as(_I)))
        return out

    def gradient(self):
        """(nchains, vstride) dE/dv of every variable (vacuum, FP64) and the
        energies (gradient.f)."""
        g = np.zeros(self.nchains * self.vstride)
        e = np.zeros(self.nchains)
        check(lib.smmp_ens_gradient(self._h, g.ctypes.data_as(_D), e.ctypes.data_as(_D)))
        return g.reshape(self.nchains, self.vstride), e

    def pair_terms(self):
        """Pair terms each chain's sweeps have evaluated so far."""
        out = np.zeros(self.nchains, dtype=np.uint64)
        check(lib.smmp_ens_pair_terms(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))
        return out

    def pt_stats(self):
        """(attempts, accepts) of each label pair (k, k+1) since set_pt."""
        out = np.zeros(2 * self.nchains, dtype=np.uint64)
        check(lib.smmp_ens_pt_stats(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))
        return out[0::2], out[1::2]

    # ---------------------------------------------------------------- state
    def energies(self):
        out = np.zeros(self.nchains)
        check(lib.smmp_ens_get_energies(self._h, out.ctypes.data_as(_D)))
        return out

    def terms(self):
        """(nchains, 6): eyel, eyvw, eyhb, eyvr, eysl, eysm of the last full evaluation."""
        out = np.zeros(self.nchains * 6)
        check(lib.smmp_ens_get_terms(self._h, out.ctypes.data_as(_D)))
        return out.reshape(self.nchains, 6)

    def vlvr(self):
        out = np.zeros(self.nchains * self.vstride)
        check(lib.smmp_ens_get_vlvr(self._h, out.ctypes.data_as(_D)))
        return out.reshape(self.nchains, self.vstride)

    def set_vlvr(self, v):
        a = np.ascontiguousarray(v, dtype=np.float64).reshape(-1)
        if a.size != self.nchains * self.vstride:
            raise ValueError("expected (nchains, vstride) variables")
        check(lib.smmp_ens_set_vlvr(self._h, a.ctypes.data_as(_D)))

    def betas(self):
        out = np.zeros(self.nchains)
        check(lib.smmp_ens_get_betas(self._h, out.ctypes.data_as(_D)))
        return out

    def coords(self):
        out = np.zeros(self.nchains * 3 * self.tstride)
        check(lib.smmp_ens_get_coords(self._h, out.ctypes.data_as(_D)))
        return out.reshape(self.nchains, self.tstride, 3)

    def acceptance(self):
        a = np.zeros(self.nchains, dtype=np.uint64)
        p = np.zeros(self.nchains, dtype=np.uint64)
        check(lib.smmp_ens_acceptance(self._h, a.ctypes.data_as(ctypes.POINTER(ctypes.c_ulonglong)),
                                      p.ctypes.data_as(ctypes.POINTER(ctypes.c_ulonglong))))
        return a, p

    def errors(self):
        out = np.zeros(self.nchains, dtype=np.int32)
        check(lib.smmp_ens_errors(self._h, out.ctypes.data_as(_I)))
        return out

    def draw(self, slot, n):
        out = np.zeros(n)
        check(lib.smmp_ens_draw(self._h, int(slot), int(n), out.ctypes.data_as(_D)))
        return out

    def set_surrogate(self, surrogate, floor=0.2, min_stage1=64):
        """Delayed acceptance with a trained smmp.surrogate.Surrogate as the
        first stage (None: plain sweeps).  Chains whose stage-2 acceptance
        falls below `floor` after min_stage1 stage-1 passes take plain
        steps."""
        self._surrogate = surrogate          # keep its device memory alive
        check(lib.smmp_ens_set_surrogate(self._h, surrogate._h if surrogate else None,
                                         float(floor), int(min_stage1)))

    AUTOTUNE_FORMS = ("pair lists", "rows", "rows for 128+ atoms")

    def autotune(self):
        """Pick the fastest pair-work decomposition (pair lists, row passes,
        or row passes for molecules of 128 atoms or more) by timing one sweep
        of each from the same saved state; the state is restored.  Returns
        (form, (ms_lists, ms_rows, ms_by_size)), form one of AUTOTUNE_FORMS."""
        choice = ctypes.c_int()
        ms = (ctypes.c_double * 3)()
        check(lib.smmp_ens_autotune(self._h, ctypes.byref(choice), ms))
        return self.AUTOTUNE_FORMS[choice.value], (ms[0], ms[1], ms[2])

    def set_window(self, k):
        """Proposals per speculative window of the sweep (1: one at a time);
        returns the size applied (large molecules get smaller windows)."""
        got = ctypes.c_int()
        check(lib.smmp_ens_set_window(self._h, int(k), ctypes.byref(got)))
        return got.value

    def window(self):
        """(window in use, autotuner's one-sweep times with windows 2, 4, 8)."""
        k = ctypes.c_int()
        ms = (ctypes.c_double * 3)()
        check(lib.smmp_ens_window(self._h, ctypes.byref(k), ms))
        return k.value, (ms[0], ms[1], ms[2])

    def set_pair_work(self, form):
        """Pair-work form by hand: one of AUTOTUNE_FORMS (or its index)."""
        k = self.AUTOTUNE_FORMS.index(form) if isinstance(form, str) else int(form)
        check(lib.smmp_ens_set_pair_work(self._h, k))

    def da_stats(self):
        """(stage-1 passes, stage-2 accepts) per chain."""
        a = np.zeros(self.nchains, dtype=np.uint64)
        b = np.zeros(self.nchains, dtype=np.uint64)
        check(lib.smmp_ens_da_stats(self._h, a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                    b.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))
        return a, b

    def checkpoint(self):
        n = ctypes.c_uint64(0)
        check(lib.smmp_ens_checkpoint(self._h, None, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        check(lib.smmp_ens_checkpoint(self._h, buf, ctypes.byref(n)))
        return buf.raw[:n.value]

    def restore(self, blob):
        buf = ctypes.create_string_buffer(blob, len(blob))
        check(lib.smmp_ens_restore(self._h, buf, len(blob)))

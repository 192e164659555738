"""Python 3 stand-in for SMMP's f2py module ``smmp`` on the energy-and-sweep path.

The call shapes are those of trunk/smmp.pyf, so code written against the
reference (universe.py, protein.py, algorithms.py) runs unchanged on the path:

    import smmp
    smmp.epar_l.sh2 = 0; smmp.isolty.itysol = 0
    smmp.init_energy('SMMP/')
    smmp.init_molecule(1, 'nh2', 'cooh', 'enkefa.seq', 'enkefa.var')
    e = smmp.energy()
    eol, acz = smmp.metropolis(e, 0, smmp.can_weight)

Every energy, rebuild and sweep runs in the sm_100a kernels of
libsmmp_b200.so.  COMMON blocks are exposed as attribute views
(``smmp.var_r.vlvr``, ``smmp.bet.beta`` ...); writing into ``var_r.vlvr`` is
seen by the next call, as writing into the Fortran COMMON is.  Batched
ensembles of chains are in :mod:`smmp.ensemble`.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import SmmpError, check, lib

__all__ = ["init_energy", "init_molecule", "energy", "setvar", "metropolis", "outvar", "outpdb",
           "sgrnd",
           "grnd", "canon", "anneal", "can_weight", "MucaWeight", "SmmpError",
           "epar_l", "isolty", "updchois", "bet", "mol_par", "var_r", "var_i", "eny_r",
           "updstats", "gpu_available", "reset", "coordinates", "MucaState",
           "mulcan_par", "enysol", "gradient", "minim"]


def gpu_available():
    return bool(lib.smmp_gpu_available())


# ------------------------------------------------------------------ COMMON views
class _ConfigBlock:
    """Attribute view of the switches of /epar_l/, /isolty/ and /updchois/."""

    _map = {}

    def __getattr__(self, name):
        if name in self._map:
            c = _lib.Config()
            check(lib.smmp_get_config(ctypes.byref(c)))
            return getattr(c, self._map[name])
        if name in self._fixed:
            return self._fixed[name]
        raise AttributeError(name)

    def __setattr__(self, name, value):
        if name in self._map:
            c = _lib.Config()
            check(lib.smmp_get_config(ctypes.byref(c)))
            setattr(c, self._map[name], int(value))
            check(lib.smmp_set_config(ctypes.byref(c)))
        elif name in self._fixed:
            if value != self._fixed[name]:
                raise SmmpError(1, "%s=%r is outside this path" % (name, value))
        else:
            raise AttributeError(name)


class _EparL(_ConfigBlock):          # INCL.H:327 common /epar_l/ flex, tesgrd, sh2, epsd, ientyp
    _map = {"sh2": "sh2", "epsd": "epsd", "ientyp": "ientyp"}
    _fixed = {"flex": 0, "tesgrd": 0}


class _Isolty(_ConfigBlock):         # INCL.H:69 common /isolty/ itysol, isolscl
    _map = {"itysol": "itysol"}
    _fixed = {"isolscl": 0}


class _Updchois(_ConfigBlock):       # INCL.H:114 common /updchois/ rndord, upchswitch, bgsprob
    _map = {"rndord": "rndord", "upchswitch": "upchswitch"}
    _fixed = {"bgsprob": 0}


class _Bet:                          # INCL.H:57 common /bet/ beta
    @property
    def beta(self):
        return lib.smmp_get_beta()

    @beta.setter
    def beta(self, v):
        check(lib.smmp_set_beta(float(v)))


def _sizes():
    na, nv, nf = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    check(lib.smmp_get_sizes(ctypes.byref(na), ctypes.byref(nv), ctypes.byref(nf)))
    return na.value, nv.value, nf.value


class _MolPar:                       # INCL.H:87 common /mol_par/ nvr
    @property
    def nvr(self):
        return _sizes()[2]


class _WriteBack(np.ndarray):
    """Array whose item assignment is written back to the library."""

    def __setitem__(self, key, value):
        super().__setitem__(key, value)
        push = getattr(self, "_push", None)
        if push is not None:
            push(np.asarray(self))

    def __array_finalize__(self, obj):
        self._push = getattr(obj, "_push", None)


class _VarR:                         # INCL.H:271 common /var_r/ olvlvr, vlvr, axvr
    @property
    def vlvr(self):
        nv = _sizes()[1]
        a = np.zeros(nv)
        check(lib.smmp_get_vlvr(a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        v = a.view(_WriteBack)
        v._push = lambda arr: check(lib.smmp_set_vlvr(
            np.ascontiguousarray(arr, dtype=np.float64).ctypes.data_as(
                ctypes.POINTER(ctypes.c_double))))
        return v

    @vlvr.setter
    def vlvr(self, values):
        a = np.ascontiguousarray(values, dtype=np.float64)
        check(lib.smmp_set_vlvr(a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))

    @property
    def axvr(self):
        a = np.zeros(_sizes()[1])
        check(lib.smmp_get_axvr(a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return a


class _VarI:                         # INCL.H:272 common /var_i/ ... idvr
    @property
    def idvr(self):
        a = np.zeros(_sizes()[2], dtype=np.int32)
        check(lib.smmp_get_idvr(a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        return a


class _EnyR:                         # INCL.H:343 common /eny_r/ eyel, eyvw, eyhb, eyvr, eysm, eysl
    def _t(self):
        t = (ctypes.c_double * 6)()
        check(lib.smmp_energy_terms(t))
        return list(t)

    eyel = property(lambda s: s._t()[0])
    eyvw = property(lambda s: s._t()[1])
    eyhb = property(lambda s: s._t()[2])
    eyvr = property(lambda s: s._t()[3])
    eysl = property(lambda s: s._t()[4])
    eysm = property(lambda s: s._t()[5])


class _UpdStats:                     # metropolis.f common /updstats/ ncalls, nacalls
    def _get(self):
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        check(lib.smmp_get_acceptance(ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    ncalls = property(lambda s: s._get()[0])
    nacalls = property(lambda s: s._get()[1])


epar_l = _EparL()
isolty = _Isolty()
updchois = _Updchois()
bet = _Bet()
mol_par = _MolPar()
var_r = _VarR()
var_i = _VarI()
eny_r = _EnyR()
updstats = _UpdStats()


# ------------------------------------------------------------------ weights
class _CanWeight:
    """can_weight (canon.f:135-149): W(E) = beta*E, evaluated on the GPU."""

    def __call__(self, x):
        return bet.beta * x

    def _struct(self):
        return _lib.Weight(kind=0)


can_weight = _CanWeight()


class MucaWeight:
    """Multicanonical weight (mulcan_par_mod.f90:380-410) on the GPU.

    kind=1: (beta + b[k])*E + alpha[k]; kind=2: b[k]*E + alpha[k], with
    k = int(clamp(E/ebin + sign(0.5, E), kmin, kmax)); b, alpha indexed k-kmin.
    """

    def __init__(self, b, alpha, kmin, kmax, ebin, kind=1):
        self.b = np.ascontiguousarray(b, dtype=np.float64)
        self.alpha = np.ascontiguousarray(alpha, dtype=np.float64)
        if len(self.b) != kmax - kmin + 1 or len(self.alpha) != kmax - kmin + 1:
            raise ValueError("b and alpha need kmax-kmin+1 entries")
        self.kmin, self.kmax, self.ebin, self.kind = int(kmin), int(kmax), float(ebin), int(kind)

    def __call__(self, x):
        k = int(min(self.kmax, max(self.kmin, x / self.ebin + np.copysign(0.5, x))))
        bb, aa = self.b[k - self.kmin], self.alpha[k - self.kmin]
        return ((bet.beta + bb) * x + aa) if self.kind == 1 else (bb * x + aa)

    def _struct(self):
        P = ctypes.POINTER(ctypes.c_double)
        return _lib.Weight(kind=self.kind, kmin=self.kmin, kmax=self.kmax, ebin=self.ebin,
                           b=self.b.ctypes.data_as(P), alpha=self.alpha.ctypes.data_as(P))


def _weight_struct(w):
    """Weight argument of metropolis: GPU weights directly, any other callable
    through a host callback (the f2py callback of smmp.pyf:3-10)."""
    if w is None or isinstance(w, (_CanWeight, MucaWeight)):
        return (w or can_weight)._struct(), None
    if not callable(w):
        raise TypeError("weight must be callable")
    cb = _lib.WEIGHT_FN(lambda x, _u: float(w(x)))
    return _lib.Weight(kind=3, callback=cb), cb


# ------------------------------------------------------------------ routines
def _b(s):
    return (s if s is not None else " ").encode()


def reset():
    """Drop the global system (a fresh process of the reference)."""
    check(lib.smmp_reset())


def init_energy(libdir):
    """init_energy(libdir) -- smmp.pyf:4404, init_energy.f:14."""
    check(lib.smmp_init_energy(_b(libdir)))


def init_molecule(iabin, grpn, grpc, seqfile=" ", varfile=" "):
    """init_molecule(iabin, grpn, grpc, seqfile, varfile) -- smmp.pyf:5011."""
    check(lib.smmp_init_molecule(int(iabin), _b(grpn), _b(grpc), _b(seqfile), _b(varfile)))


def energy():
    """energy() -- smmp.pyf:380, energy.f:12."""
    e = ctypes.c_double()
    check(lib.smmp_energy(ctypes.byref(e)))
    return e.value


def enysol(nmol=0):
    """enysol(nmol=0) -- smmp.pyf:664, enysol.f:13: the numerical solvation
    energy of the current conformation (rebuilt from the current variables)."""
    e = ctypes.c_double()
    check(lib.smmp_enysol(int(nmol), ctypes.byref(e)))
    return e.value


def gradient():
    """gradient() -- gradient.f:13 (vacuum): (energy, dE/dv of every
    variable); the derivatives are also /eny_r/ gdeyvr of the reference."""
    n = _sizes()[1]
    g = np.zeros(max(n, 1))
    e = ctypes.c_double()
    check(lib.smmp_gradient(g.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(e)))
    return e.value, g[:n]


def minim(imin, maxit, eps):
    """minim(imin, maxit, eps) -- smmp.pyf:1234, minim.f:13: minimise over the
    free variables (1 quasi-Newton, 2 conjugate gradients) with the GPU
    gradient; the variables are left at the minimum.  Returns the number of
    energy+gradient evaluations."""
    nop = ctypes.c_int()
    check(lib.smmp_minim(int(imin), int(maxit), float(eps), ctypes.byref(nop)))
    return nop.value


def setvar(nml, vlvrx):
    """setvar(nml, vlvrx) -- smmp.pyf:949, setvar.f:13."""
    a = np.ascontiguousarray(vlvrx, dtype=np.float64)
    check(lib.smmp_setvar(int(nml), a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))


def metropolis(eol, acz, dummy=None):
    """metropolis(eol, acz, dummy) -> (eol, acz) -- smmp.pyf:22-25, metropolis.f:13."""
    e, a = ctypes.c_double(eol), ctypes.c_double(acz)
    ws, keep = _weight_struct(dummy)
    check(lib.smmp_metropolis(ctypes.byref(e), ctypes.byref(a), ctypes.byref(ws)))
    del keep
    return e.value, a.value


def outvar(nml, fileName=""):
    """outvar(nml, fileName) -- outvar.f:12: the current variables in the .var
    command language, to the file or (fileName blank) to standard output."""
    check(lib.smmp_outvar(int(nml), (fileName or "").encode()))


def outpdb(nml, fileName=""):
    """outpdb(nml, fileName) -- outpdb.f:12: the current conformation in PDB
    format, to the file or (fileName blank) to standard output."""
    check(lib.smmp_outpdb(int(nml), (fileName or "").encode()))


def sgrnd(seed):
    """sgrnd(seed) -- smmp.pyf:5620, twister.f:64."""
    check(lib.smmp_sgrnd(int(seed)))


def grnd():
    """grnd() -- twister.f:104."""
    v = lib.smmp_grnd()
    if v != v:
        check(3)
    return v


def canon(nequi, nswp, nmes, temp, lrand=1):
    """canon(nequi, nswp, nmes, temp, lrand) -- smmp.pyf:3522, canon.f:12.

    Returns (energies every nmes sweeps, energy after equilibration,
    acceptance rate, last energy)."""
    n = nswp // nmes + 1
    trace = np.zeros(n)
    out = (ctypes.c_double * 3)()
    check(lib.smmp_canon(int(nequi), int(nswp), int(nmes), float(temp), int(lrand),
                         trace.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), out))
    return trace, out[0], out[1], out[2]


def anneal(nequi, nswp, nmes, tmax, tmin, lrand=1):
    """anneal(nequi, nswp, nmes, tmax, tmin, lrand) -- smmp.pyf:2663, anneal.f:13.

    Returns (start energy, energy after equilibration, acceptance, last
    energy, lowest energy, sweep of the lowest energy)."""
    out = (ctypes.c_double * 6)()
    check(lib.smmp_anneal(int(nequi), int(nswp), int(nmes), float(tmax), float(tmin),
                          int(lrand), out))
    return tuple(out[:5]) + (int(out[5]),)


class MucaState:
    """Weight parameters of the multicanonical recursion over the energy bins
    kmin..kmax of width ebin (arrays indexed k - kmin), as mulcan_par keeps
    them: accumulated histogram xhist, recursion weights g1, b, alpha and the
    entropy estimate ent."""

    def __init__(self, kmin, kmax, ebin):
        if kmax - kmin < 2 or ebin <= 0:
            raise ValueError("need at least three bins and ebin > 0")
        self.kmin, self.kmax, self.ebin = int(kmin), int(kmax), float(ebin)
        n = self.kmax - self.kmin + 1
        self.xhist, self.g1, self.b, self.alpha, self.ent = (np.zeros(n) for _ in range(5))

    def update(self, ihist, beta):
        """mulcan_par_mod.f90:93-145: the histogram of the last sweeps
        (int array, zeroed on return) updates the weights."""
        h = np.ascontiguousarray(ihist, dtype=np.int32)
        D = ctypes.POINTER(ctypes.c_double)
        check(lib.smmp_muca_update(self.kmin, self.kmax, self.ebin, float(beta),
                                   h.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                   *(a.ctypes.data_as(D) for a in
                                     (self.xhist, self.g1, self.b, self.alpha, self.ent))))
        ihist[:] = h

    def finish(self, beta):
        """mulcan_par_mod.f90:163-168: beta folded into b (weights of kind 2)."""
        D = ctypes.POINTER(ctypes.c_double)
        check(lib.smmp_muca_finish(self.kmin, self.kmax, self.ebin, float(beta),
                                   self.b.ctypes.data_as(D), self.alpha.ctypes.data_as(D)))

    def weight(self, kind=1):
        return MucaWeight(self.b, self.alpha, self.kmin, self.kmax, self.ebin, kind=kind)


def _addang(a1, a2):
    """addang (difang.f:38-60): a1 + a2 wrapped into (-pi, pi]."""
    pi2 = 2.0 * np.pi
    d = float(np.fmod(a1 + a2, pi2))
    return d if abs(d) <= np.pi else d - float(np.copysign(pi2, d))


def mulcan_par(nsweep, nup, temp, kmin, kmax, binWidth, l_iter=False):
    """mulcan_par(nsweep, nup, temp, kmin, kmax, binWidth, l_iter) --
    mulcan_par_mod.f90:23: multicanonical weight iteration.  A random start,
    then nsweep sweeps with muca_weight, the weights updated from the
    histogram every nup sweeps (mpar_full.d written at each update, read
    first when l_iter); the final weights (beta folded in) go to muca.d and
    are returned as a MucaState."""
    beta = 1.0 / (temp * 1.98773e-3)
    bet.beta = beta
    st = MucaState(kmin, kmax, binWidth)
    if l_iter:
        rows = np.loadtxt("mpar_full.d", ndmin=2)
        for r in rows:
            k = int(r[0]) - st.kmin
            st.xhist[k], st.g1[k], st.b[k], st.alpha[k], st.ent[k] = r[1:6]
    ihist = np.zeros(st.kmax - st.kmin + 1, dtype=np.int32)
    v = var_r.vlvr
    ax = var_r.axvr
    for iv in np.asarray(var_i.idvr) - 1:   # random start (mulcan_par_mod.f90:79-84)
        dv = ax[iv] * (grnd() - 0.5)
        v[iv] = _addang(np.pi, dv)
    var_r.vlvr = v
    eol = energy()
    outpdb(1, "start.pdb")
    acz = 0.0
    w = st.weight(1)
    for nsw in range(1, nsweep + 1):
        eol, acz = metropolis(eol, acz, w)
        x = eol / st.ebin + np.copysign(0.5, eol)
        muold = int(min(float(st.kmax), max(float(st.kmin), x)))
        ihist[muold - st.kmin] += 1
        if nsw % nup == 0:
            st.update(ihist, beta)
            with open("mpar_full.d", "w") as f:
                for k in range(st.kmax, st.kmin - 1, -1):
                    i = k - st.kmin
                    f.write("%5d%15.4f%15.4f%15.4f%15.4f%15.4f\n" % (
                        k, st.xhist[i], st.g1[i], st.b[i], st.alpha[i], st.ent[i]))
            w = st.weight(1)
    st.acceptance = acz / float((nsweep + 1) * mol_par.nvr)   # nsw = nsweep+1 after the DO loop
    st.last_energy = eol
    st.finish(beta)
    with open("muca.d", "w") as f:
        for k in range(st.kmin, st.kmax + 1):
            f.write("%12d %24.16E %24.16E\n" % (k, st.b[k - st.kmin], st.alpha[k - st.kmin]))
    return st


def coordinates():
    """Cartesian coordinates (natoms, 3) of the current conformation."""
    na = _sizes()[0]
    a = np.zeros(3 * na)
    check(lib.smmp_get_coords(a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    return a.reshape(na, 3)

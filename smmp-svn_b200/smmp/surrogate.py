"""Learned energy surrogate (no counterpart in the reference).

An MLP on the sin/cos of a molecule's free dihedrals (3 hidden layers of 256,
SiLU), BF16 weights with FP32 accumulation, trained on the GPU by the
library's tensor-core forward and backward kernels with Adam.  The sweep
kernels use a trained surrogate as the first stage of a two-stage
(delayed-acceptance) Metropolis step; see Ensemble.set_surrogate.
"""
import ctypes

import numpy as np

from ._lib import check, lib

_D = ctypes.POINTER(ctypes.c_double)
_F = ctypes.POINTER(ctypes.c_float)


def _dptr(a):
    return a.ctypes.data_as(_D)


class Surrogate:
    def __init__(self, nang, seed=1234):
        self.nang = int(nang)
        self._h = lib.smmp_sur_create(self.nang, int(seed))
        if not self._h:
            raise RuntimeError(lib.smmp_last_error().decode())
        nin, pad, n = ctypes.c_int(), ctypes.c_int(), ctypes.c_int64()
        check(lib.smmp_sur_sizes(self._h, ctypes.byref(nin), ctypes.byref(pad), ctypes.byref(n)))
        self.nin, self.nin_pad, self.nparams = nin.value, pad.value, n.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib.smmp_sur_free(h)
            self._h = None

    def _ang(self, ang):
        a = np.ascontiguousarray(ang, dtype=np.float64)
        if a.ndim != 2 or a.shape[1] != self.nang:
            raise ValueError("angles must be (n, %d)" % self.nang)
        return a

    def set_data(self, ang, energy, clip=1e30):
        a = self._ang(ang)
        e = np.ascontiguousarray(energy, dtype=np.float64)
        check(lib.smmp_sur_set_data(self._h, _dptr(a), _dptr(e), a.shape[0], float(clip)))

    def train(self, epochs, batch=4096, lr=1e-3, seed=7):
        loss = ctypes.c_double()
        check(lib.smmp_sur_train(self._h, int(epochs), int(batch), float(lr), int(seed),
                                 ctypes.byref(loss)))
        return loss.value

    def predict(self, ang):
        a = self._ang(ang)
        out = np.zeros(a.shape[0])
        check(lib.smmp_sur_predict(self._h, _dptr(a), a.shape[0], _dptr(out)))
        return out

    def gradients(self, ang, energy):
        a = self._ang(ang)
        e = np.ascontiguousarray(energy, dtype=np.float64)
        g = np.zeros(self.nparams, dtype=np.float32)
        loss = ctypes.c_double()
        check(lib.smmp_sur_gradients(self._h, _dptr(a), _dptr(e), a.shape[0],
                                     g.ctypes.data_as(_F), ctypes.byref(loss)))
        return loss.value, g

    def params(self):
        p = np.zeros(self.nparams, dtype=np.float32)
        norm = np.zeros(2, dtype=np.float32)
        check(lib.smmp_sur_get_params(self._h, p.ctypes.data_as(_F), norm.ctypes.data_as(_F)))
        return p, norm

    def set_params(self, p, norm=None):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.nparams:
            raise ValueError("expected %d parameters" % self.nparams)
        n = None if norm is None else np.ascontiguousarray(norm, dtype=np.float32)
        check(lib.smmp_sur_set_params(self._h, p.ctypes.data_as(_F),
                                      None if n is None else n.ctypes.data_as(_F)))

    def layout(self):
        """Slices of the flat parameter vector: W1, b1, W2, b2, W3, b3, w4, b4."""
        H = 256
        sizes = [("W1", (self.nin_pad, H)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)),
                 ("W3", (H, H)), ("b3", (H,)), ("w4", (H,)), ("b4", (1,))]
        out, off = {}, 0
        for name, shape in sizes:
            n = int(np.prod(shape))
            out[name] = (slice(off, off + n), shape)
            off += n
        return out


def collect_samples(ens, molecule, nsweeps, pt=True):
    """Run nsweeps sweeps (parallel tempering when pt) of an ensemble of one
    molecule and return its states after every sweep: (angles [n, nvr] of the
    free dihedrals, energies [n])."""
    ang, en = [], []
    for _ in range(int(nsweeps)):
        if pt:
            ens.pt_sweeps(1, graph_chunk=1)
        else:
            ens.sweeps(1)
        ang.append(ens.vlvr()[:, molecule.idvr].copy())
        en.append(ens.energies().copy())
    return np.concatenate(ang), np.concatenate(en)

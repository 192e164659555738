"""ctypes binding of libsmmp_b200.so (declarations follow include/smmp_b200.h).

The library is loaded from this directory; importing raises ImportError when it
is missing, so no code path silently falls back to anything else.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# SMMP_B200_LIB selects another build of the library (e.g. a debug build).
LIB_PATH = os.environ.get("SMMP_B200_LIB") or os.path.join(_HERE, "libsmmp_b200.so")

c_int = ctypes.c_int
c_double = ctypes.c_double
c_char_p = ctypes.c_char_p
c_void_p = ctypes.c_void_p
P = ctypes.POINTER


class Config(ctypes.Structure):
    _fields_ = [("sh2", c_int), ("epsd", c_int), ("itysol", c_int), ("ientyp", c_int),
                ("rndord", c_int), ("upchswitch", c_int)]


WEIGHT_FN = ctypes.CFUNCTYPE(c_double, c_double, c_void_p)


class Weight(ctypes.Structure):
    _fields_ = [("kind", c_int), ("kmin", c_int), ("kmax", c_int), ("ebin", c_double),
                ("b", P(c_double)), ("alpha", P(c_double)), ("callback", WEIGHT_FN),
                ("user", c_void_p)]


_SIGS = {
    "smmp_last_error": (c_char_p, []),
    "smmp_gpu_available": (c_int, []),
    "smmp_reset": (c_int, []),
    "smmp_set_config": (c_int, [P(Config)]),
    "smmp_get_config": (c_int, [P(Config)]),
    "smmp_init_energy": (c_int, [c_char_p]),
    "smmp_init_molecule": (c_int, [c_int, c_char_p, c_char_p, c_char_p, c_char_p]),
    "smmp_energy": (c_int, [P(c_double)]),
    "smmp_energy_terms": (c_int, [P(c_double)]),
    "smmp_enysol": (c_int, [c_int, P(c_double)]),
    "smmp_gradient": (c_int, [P(c_double), P(c_double)]),
    "smmp_minim": (c_int, [c_int, c_int, c_double, P(c_int)]),
    "smmp_ens_gradient": (c_int, [c_void_p, P(c_double), P(c_double)]),
    "smmp_setvar": (c_int, [c_int, P(c_double)]),
    "smmp_metropolis": (c_int, [P(c_double), P(c_double), P(Weight)]),
    "smmp_sgrnd": (c_int, [ctypes.c_int32]),
    "smmp_grnd": (c_double, []),
    "smmp_canon": (c_int, [c_int, c_int, c_int, c_double, c_int, P(c_double), P(c_double)]),
    "smmp_anneal": (c_int, [c_int, c_int, c_int, c_double, c_double, c_int, P(c_double)]),
    "smmp_set_beta": (c_int, [c_double]),
    "smmp_get_beta": (c_double, []),
    "smmp_get_sizes": (c_int, [P(c_int), P(c_int), P(c_int)]),
    "smmp_get_vlvr": (c_int, [P(c_double)]),
    "smmp_set_vlvr": (c_int, [P(c_double)]),
    "smmp_get_idvr": (c_int, [P(c_int)]),
    "smmp_get_axvr": (c_int, [P(c_double)]),
    "smmp_get_coords": (c_int, [P(c_double)]),
    "smmp_get_acceptance": (c_int, [P(ctypes.c_longlong), P(ctypes.c_longlong)]),
    "smmp_mol_build": (c_void_p, [c_char_p, P(Config), c_char_p, c_char_p, c_char_p, c_char_p]),
    "smmp_mol_free": (None, [c_void_p]),
    "smmp_mol_info": (c_int, [c_void_p, P(ctypes.c_longlong)]),
    "smmp_mol_idvr": (c_int, [c_void_p, P(c_int)]),
    "smmp_mol_vlvr0": (c_int, [c_void_p, P(c_double)]),
    "smmp_mol_var_ranges": (c_int, [c_void_p, P(c_int), P(c_int)]),
    "smmp_mol_atoms": (c_int, [c_void_p, P(c_int), P(c_int), P(c_double), P(c_double)]),
    "smmp_mol_pairs": (c_int, [c_void_p, P(c_int)]),
    "smmp_mol_vars": (c_int, [c_void_p, P(c_int)]),
    "smmp_mol_outvar": (c_int, [c_void_p, P(c_double), c_int, c_void_p, P(ctypes.c_uint64)]),
    "smmp_outvar": (c_int, [c_int, c_char_p]),
    "smmp_muca_update": (c_int, [c_int, c_int, c_double, c_double, P(c_int), P(c_double),
                                 P(c_double), P(c_double), P(c_double), P(c_double)]),
    "smmp_muca_finish": (c_int, [c_int, c_int, c_double, c_double, P(c_double), P(c_double)]),
    "smmp_outpdb": (c_int, [c_int, c_char_p]),
    "smmp_mol_outpdb": (c_int, [c_void_p, P(c_double), c_void_p, P(ctypes.c_uint64)]),
    "smmp_ens_create": (c_void_p, [P(c_void_p), c_int, P(c_int), c_int, P(c_int), P(c_double),
                                   c_int, c_int]),
    "smmp_ens_free": (None, [c_void_p]),
    "smmp_ens_set_stream": (c_int, [c_void_p, c_void_p]),
    "smmp_ens_random_start": (c_int, [c_void_p]),
    "smmp_ens_energy": (c_int, [c_void_p, P(c_double)]),
    "smmp_ens_equilibrate": (c_int, [c_void_p, c_int]),
    "smmp_ens_sweeps": (c_int, [c_void_p, c_int, P(Weight)]),
    "smmp_ens_set_pt": (c_int, [c_void_p, P(c_double), c_int, c_int]),
    "smmp_ens_pt_sweeps": (c_int, [c_void_p, c_int, c_int, c_int]),
    "smmp_ens_set_pt_fused": (c_int, [c_void_p, c_int, c_double, c_int]),
    "smmp_ens_pt_fused_last": (c_int, [c_void_p, c_void_p]),
    "smmp_ens_pt_map": (c_int, [c_void_p, P(c_int)]),
    "smmp_ens_sizes": (c_int, [c_void_p, P(c_int), P(c_int), P(c_int)]),
    "smmp_ens_get_energies": (c_int, [c_void_p, P(c_double)]),
    "smmp_ens_get_terms": (c_int, [c_void_p, P(c_double)]),
    "smmp_ens_get_vlvr": (c_int, [c_void_p, P(c_double)]),
    "smmp_ens_set_vlvr": (c_int, [c_void_p, P(c_double)]),
    "smmp_ens_get_betas": (c_int, [c_void_p, P(c_double)]),
    "smmp_ens_get_coords": (c_int, [c_void_p, P(c_double)]),
    "smmp_ens_acceptance": (c_int, [c_void_p, P(ctypes.c_ulonglong), P(ctypes.c_ulonglong)]),
    "smmp_ens_errors": (c_int, [c_void_p, P(c_int)]),
    "smmp_ens_draw": (c_int, [c_void_p, c_int, c_int, P(c_double)]),
    "smmp_ens_checkpoint": (c_int, [c_void_p, c_void_p, P(ctypes.c_uint64)]),
    "smmp_ens_restore": (c_int, [c_void_p, c_void_p, ctypes.c_uint64]),
    "smmp_sur_create": (c_void_p, [c_int, ctypes.c_uint64]),
    "smmp_sur_free": (None, [c_void_p]),
    "smmp_sur_sizes": (c_int, [c_void_p, P(c_int), P(c_int), P(ctypes.c_int64)]),
    "smmp_sur_set_data": (c_int, [c_void_p, P(c_double), P(c_double), c_int, c_double]),
    "smmp_sur_train": (c_int, [c_void_p, c_int, c_int, c_double, ctypes.c_uint64, P(c_double)]),
    "smmp_sur_predict": (c_int, [c_void_p, P(c_double), c_int, P(c_double)]),
    "smmp_sur_gradients": (c_int, [c_void_p, P(c_double), P(c_double), c_int,
                                   P(ctypes.c_float), P(c_double)]),
    "smmp_sur_predict_noalloc": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p]),
    "smmp_ens_set_surrogate": (c_int, [c_void_p, c_void_p, c_double, c_int]),
    "smmp_ens_autotune": (c_int, [c_void_p, P(c_int), P(c_double)]),
    "smmp_ens_set_window": (c_int, [c_void_p, c_int, P(c_int)]),
    "smmp_ens_window": (c_int, [c_void_p, P(c_int), P(c_double)]),
    "smmp_ens_set_pair_work": (c_int, [c_void_p, c_int]),
    "smmp_ens_pt_stats": (c_int, [c_void_p, P(ctypes.c_uint64)]),
    "smmp_ens_pair_terms": (c_int, [c_void_p, P(ctypes.c_uint64)]),
    "smmp_ens_da_stats": (c_int, [c_void_p, P(ctypes.c_uint64), P(ctypes.c_uint64)]),
    "smmp_sur_get_params": (c_int, [c_void_p, P(ctypes.c_float), P(ctypes.c_float)]),
    "smmp_sur_set_params": (c_int, [c_void_p, P(ctypes.c_float), P(ctypes.c_float)]),
}

EXPORTED = sorted(_SIGS)


def load():
    if not os.path.exists(LIB_PATH):
        raise ImportError("libsmmp_b200.so is not built (run smmp-svn_b200/build.py): "
                          + LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = load()


class SmmpError(RuntimeError):
    """A library call returned a nonzero status."""

    def __init__(self, status, message):
        super().__init__("%s (status %d)" % (message, status))
        self.status = status


def check(status):
    if status != 0:
        raise SmmpError(status, lib.smmp_last_error().decode(errors="replace"))
    return status

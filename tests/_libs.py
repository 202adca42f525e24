"""ctypes bindings for the test-only libraries: the oracle (oracle/liboracle.so)
and the CPU build of the reference's own sources (oracle/_ref/libgevref.so)."""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libgevref.so")

_d = ctypes.c_double
_i = ctypes.c_int
_l = ctypes.c_int64
_p = ctypes.c_void_p


def ptr(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_p)


# argument signatures shared by orc_* and ref_* twins
_SIGS = {
    "project_T00": ([_i, _l, _p, _p, _d, _p, _d, _d, _p], None),
    "project_Tij": ([_i, _l, _p, _p, _d, _p, _d, _d, _p], None),
    "project_T0i": ([_i, _l, _p, _p, _d, _p, _d, _p], None),
    "project_cic": ([_i, _l, _p, _d, _p], None),
    "prepare_T00": ([_i, _p, _p, _p, _d, _d, _d, _d, _p], _d),
    "prepare_Tij": ([_i, _p, _p, _d, _p], None),
    "solve_poisson": ([_i, _p, _p, _d, _d], None),
    "project_scalar": ([_i, _p, _p, _i], None),
    "project_vector": ([_i, _p, _p, _d, _d], None),
    "evolve_vector": ([_i, _p, _p, _d], None),
    "project_tensor": ([_i, _p, _p], None),
    "evolve_tensor": ([_i, _p, _p, _p, _d, _d, _d], None),
    "update_q": ([_i, _l, _p, _p, _p, _p, _p, _i, _d, _d, _d], _d),
    "update_pos": ([_i, _l, _p, _p, _p, _p, _p, _i, _d, _d, _d], None),
    "power_spectrum": ([_i, _p, _i, _p, _p, _p, _p, _p], None),
    "update_q_newton": ([_i, _l, _p, _p, _p, _d, _d], _d),
}


class _Lib:
    def __init__(self, path, prefix, extra):
        self.lib = ctypes.CDLL(path)
        self.prefix = prefix
        for name, (args, res) in list(_SIGS.items()) + list(extra.items()):
            fn = getattr(self.lib, prefix + name, None)
            if fn is None:
                continue
            fn.argtypes = args
            fn.restype = res
            setattr(self, name, fn)


_ORC_EXTRA = {
    "r2c": ([_i, _p, _p], None),
    "c2r": ([_i, _p, _p], None),
    "hconf": ([_d, _d, _p], _d),
    "particle_horizon": ([_d, _d, _p], _d),
    "lightcone_select": ([_i, _l, _p, _p, _p, _p, _p, _d, _d, _d, _d, _d, _l, _p, _p, _p, _d], _l),
    "find_intersecting": ([_p, _p, _d, _d, _d, _p, _p], _i),
    "update_pos_newton": ([_l, _p, _p, _d, _d], None),
    "initialize_q": ([_i, _l, _p, _p, _p, _d], None),
}
_REF_EXTRA = {
    "update_pos_newton": ([_i, _l, _p, _p, _d, _d], None),
    "hconf": ([_d, _d, _d, _d, _d], _d),
    "rk4bg": ([_d, _d, _d, _d, _d, _d], _d),
    "particle_horizon": ([_d, _d, _d, _d, _d], _d),
    "find_intersecting": ([_p, _p, _d, _d, _d, _p, _p], _i),
    "max_intersects": ([], _i),
    "sitmo_words": ([ctypes.c_uint32, ctypes.c_uint64, _l, _p], None),
    "express_write": ([ctypes.c_char_p, _i, _l, _p, _p, _p, _p], _i),
    "express_read": ([ctypes.c_char_p, _i, _l, _p, _p, _p, _p, _p], _i),
    "spline_eval": ([_p, _p, _i, _p, _i, _p], None),
    "ics_basic": ([_i, _d, _d, _d, _d, _d, _d, _p, _p, _i, ctypes.c_uint32, _i, _i, _i, _i, _p, _l,
                   _p, _p, _p, _p, _p, _p, _p], _i),
    # the reference's own lightcone kernels, run on the GPU
    "lightcone_shell": ([_i, _l, _p, _p, _p, _p, _p, _p, _d, _d, _d, _d, _d, _d, _d, _i, _i, _p, _l, _l,
                         _p, _p, _p, _p, _p, _p, _p], _i),
}

_oracle = None
_ref = None


def oracle():
    global _oracle
    if _oracle is None:
        _oracle = _Lib(ORACLE_SO, "orc_", _ORC_EXTRA)
        # orc_power_spectrum carries an extra kmax argument
        _oracle.lib.orc_power_spectrum.argtypes = [_i, _p, _i, _p, _p, _p, _p, _p, _d]
    return _oracle


def ref():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            return None
        _ref = _Lib(REF_SO, "ref_", _REF_EXTRA)
    return _ref


class OrcCosmo(ctypes.Structure):
    _fields_ = [("Omega_m", _d), ("Omega_Lambda", _d), ("Omega_rad", _d)]


def kshape(N):
    return (N, N, N // 2 + 1)

"""Gadget-2 files through the C ABI (gev_gadget2_write, gev_snapshot_gadget2)
and a reader for them.

The header layout is gevolution's gadget2_header (metadata.hpp:159-178);
files hold the header, POS, VEL and ID blocks, each enclosed by uint32 record
lengths.  `header()` fills the fields the way the reference's lightcone and
snapshot outputs do (output.hpp:2097-2123, :417-440).
"""
import ctypes

import numpy as np

from . import GevError, _sig

_u32, _i32, _d, _p, _l = ctypes.c_uint32, ctypes.c_int32, ctypes.c_double, ctypes.c_void_p, ctypes.c_int64

GADGET_LENGTH_CONVERSION = 0.001      # kpc/h per Mpc/h (metadata.hpp)
GADGET_MASS_CONVERSION = 1.0e10       # M_sun/h
GADGET_VELOCITY_CONVERSION = 3.335640952e-6
C_RHO_CRIT = 2.77459457e11            # M_sun h^2 / Mpc^3


class Gadget2Header(ctypes.Structure):
    _fields_ = [("npart", _u32 * 6), ("mass", _d * 6), ("time", _d), ("redshift", _d), ("flag_sfr", _i32),
                ("flag_feedback", _i32), ("npartTotal", _u32 * 6), ("flag_cooling", _i32), ("num_files", _i32),
                ("BoxSize", _d), ("Omega0", _d), ("OmegaLambda", _d), ("HubbleParam", _d), ("flag_age", _i32),
                ("flag_metals", _i32), ("npartTotalHW", _u32 * 6), ("fill", ctypes.c_char * 64)]


assert ctypes.sizeof(Gadget2Header) == 256

_write = _sig("gev_gadget2_write", [ctypes.c_char_p, ctypes.POINTER(Gadget2Header), _p, _p, _p, _l])
_snapshot = _sig("gev_snapshot_gadget2", [_p, ctypes.c_char_p, ctypes.POINTER(Gadget2Header), _i32])
_read = _sig("gev_gadget2_read", [ctypes.c_char_p, ctypes.POINTER(Gadget2Header), _p, _p, _p, _l, ctypes.POINTER(_l)])
_load = _sig("gev_particles_load_gadget2", [_p, ctypes.c_char_p, _d, ctypes.POINTER(Gadget2Header)])
_xwrite = _sig("gev_express_write", [_p, ctypes.c_char_p, ctypes.POINTER(Gadget2Header), _i32])
_xread = _sig("gev_express_read", [_p, ctypes.c_char_p, _d, ctypes.POINTER(Gadget2Header)])


def header(a, boxsize_mpc_h, omega_m, omega_lambda, h, numpcl, omega_cdm=None, tracer_factor=1):
    """A header as output.hpp fills it for CDM particles (no baryons)."""
    hd = Gadget2Header()
    hd.num_files = 1
    hd.Omega0, hd.OmegaLambda, hd.HubbleParam = omega_m, omega_lambda, h
    hd.BoxSize = boxsize_mpc_h / GADGET_LENGTH_CONVERSION
    hd.time, hd.redshift = a, 1.0 / a - 1.0
    om = omega_m if omega_cdm is None else omega_cdm
    hd.mass[1] = tracer_factor * C_RHO_CRIT * om * boxsize_mpc_h ** 3 / numpcl / GADGET_MASS_CONVERSION
    return hd


def write(path, hdr, pos, vel, ids):
    pos = np.ascontiguousarray(pos, dtype=np.float32)
    vel = np.ascontiguousarray(vel, dtype=np.float32)
    ids = np.ascontiguousarray(ids, dtype=np.int64)
    n = len(ids)
    rc = _write(str(path).encode(), ctypes.byref(hdr), pos.ctypes.data_as(_p), vel.ctypes.data_as(_p),
                ids.ctypes.data_as(_p), n)
    if rc != 0:
        raise GevError(rc, "gev_gadget2_write failed for %s" % path)


def snapshot(ctx, path, hdr, tracer_factor=1):
    rc = _snapshot(ctx._h, str(path).encode(), ctypes.byref(hdr), int(tracer_factor))
    if rc != 0:
        raise GevError(rc, "gev_snapshot_gadget2 failed for %s" % path)


def read_c(path):
    """gev_gadget2_read: (header, pos [n,3] float32, vel [n,3] float32, ids int64)."""
    hdr = Gadget2Header()
    n = _l()
    rc = _read(str(path).encode(), ctypes.byref(hdr), None, None, None, 0, ctypes.byref(n))
    if rc != 0:
        raise GevError(rc, "gev_gadget2_read failed for %s" % path)
    pos = np.empty((n.value, 3), dtype=np.float32)
    vel = np.empty((n.value, 3), dtype=np.float32)
    ids = np.empty(n.value, dtype=np.int64)
    rc = _read(str(path).encode(), ctypes.byref(hdr), pos.ctypes.data_as(_p), vel.ctypes.data_as(_p),
               ids.ctypes.data_as(_p), n.value, ctypes.byref(n))
    if rc != 0:
        raise GevError(rc, "gev_gadget2_read failed for %s" % path)
    return hdr, pos, vel, ids


def load(ctx, path, mass):
    """gev_particles_load_gadget2: the file's particles into the context; returns the header."""
    hdr = Gadget2Header()
    rc = _load(ctx._h, str(path).encode(), float(mass), ctypes.byref(hdr))
    if rc != 0:
        raise GevError(rc, "gev_particles_load_gadget2 failed for %s" % path)
    return hdr


def express_write(ctx, filename, hdr, real_bytes=8):
    """gev_express_write: the context's particles as the reference's express
    file "<filename without numeric suffix>.0" (Real of real_bytes)."""
    rc = _xwrite(ctx._h, str(filename).encode(), ctypes.byref(hdr), int(real_bytes))
    if rc != 0:
        raise GevError(rc, "gev_express_write failed for %s" % filename)


def express_read(ctx, filename, mass):
    """gev_express_read: an express file's particles into the context; returns its Gadget-2 header."""
    hdr = Gadget2Header()
    rc = _xread(ctx._h, str(filename).encode(), float(mass), ctypes.byref(hdr))
    if rc != 0:
        raise GevError(rc, "gev_express_read failed for %s" % filename)
    return hdr


def read(path):
    """(header, pos [n,3] float32, vel [n,3] float32, ids int64) of a Gadget-2 file, parsed in Python
    (an independent reading of the byte layout)."""
    raw = open(path, "rb").read()
    off = 0
    blocks = []
    while off < len(raw):
        (n0,) = np.frombuffer(raw, dtype=np.uint32, count=1, offset=off)
        body = raw[off + 4:off + 4 + int(n0)]
        (n1,) = np.frombuffer(raw, dtype=np.uint32, count=1, offset=off + 4 + int(n0))
        if n0 != n1:
            raise ValueError("record length mismatch at offset %d" % off)
        blocks.append(body)
        off += 8 + int(n0)
    if len(blocks) != 4 or len(blocks[0]) != 256:
        raise ValueError("not a four-block Gadget-2 file")
    hdr = Gadget2Header.from_buffer_copy(blocks[0])
    pos = np.frombuffer(blocks[1], dtype=np.float32).reshape(-1, 3)
    vel = np.frombuffer(blocks[2], dtype=np.float32).reshape(-1, 3)
    ids = np.frombuffer(blocks[3], dtype=np.int64)
    return hdr, pos, vel, ids

"""C ABI checks that need no GPU: the library loads, exports every entry point
include/gev.h declares, rejects invalid configurations and null contexts before
touching the device, and its host-side background integrator (background.hpp)
agrees with the oracle.  Also checks the roofline byte model used by bench.py."""
import ctypes
import os
import re

import numpy as np
import pytest

from _libs import OrcCosmo, oracle

gev = pytest.importorskip("gevb200")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gev.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"//[^\n]*", "", src)
    return sorted(set(re.findall(r"\b(gev_[a-z0-9_]+)\s*\(", src)))


def test_exports_every_declared_symbol():
    names = declared_functions()
    assert len(names) >= 25, names
    lib = ctypes.CDLL(gev.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_string():
    assert gev.version()


@pytest.mark.parametrize("field", ["N", "precision", "vector_method", "N_big"])
def test_invalid_config_rejected(field):
    cfg = gev.Config(N=32, precision=gev.MIXED, capacity=100, boxsize=100.0,
                     vector_method=gev.VECTOR_ELLIPTIC, tensor=0, device=0, reserved=0)
    if field == "N":
        cfg.N = 20
    elif field == "precision":
        cfg.precision = 7
    elif field == "vector_method":
        cfg.vector_method = 5
    else:
        cfg.N = 1024
    h = ctypes.c_void_p()
    rc = gev._create(ctypes.byref(cfg), ctypes.byref(h))
    assert rc == gev.GEV_ERR_ARG
    assert not h.value
    assert b"invalid configuration" in gev._last_error(None)


def test_null_context():
    assert gev._pcount(None, ctypes.byref(ctypes.c_int64())) == gev.GEV_ERR_ARG
    assert gev._project(None, gev.PROJ_T00, 1.0, 1.0, 0, 0) == gev.GEV_ERR_ARG
    assert gev._lib.gev_kernel_launches(None) == -1


COSMO = dict(Omega_m=0.31, Omega_Lambda=0.69 - 8.5e-5, Omega_rad=8.5e-5)
FOURPIG = 1.5 / 3000.0 ** 2 * 300.0 ** 2   # 4 pi G in units of the box (boxsize 300 Mpc/h)


def _cosmos():
    c = gev.Cosmo(Omega_m=COSMO["Omega_m"], Omega_Lambda=COSMO["Omega_Lambda"], Omega_rad=COSMO["Omega_rad"],
                  fourpiG=FOURPIG, Cf=1.0, steplimit=1.0, z_relax=100.0, boxsize=300.0)
    o = OrcCosmo(**COSMO)
    return c, o


@pytest.mark.parametrize("a", [0.01, 0.1, 0.5, 1.0])
def test_background_matches_oracle(a):
    c, o = _cosmos()
    orc = oracle()
    h_gpu = gev._lib.gev_hconf
    h_gpu.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.POINTER(gev.Cosmo)]
    h_gpu.restype = ctypes.c_double
    h_orc = orc.lib.orc_hconf
    h_orc.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.POINTER(OrcCosmo)]
    h_orc.restype = ctypes.c_double
    assert abs(h_gpu(a, FOURPIG, ctypes.byref(c)) / h_orc(a, FOURPIG, ctypes.byref(o)) - 1) < 1e-14

    ph_gpu = gev._lib.gev_particle_horizon
    ph_gpu.argtypes = h_gpu.argtypes
    ph_gpu.restype = ctypes.c_double
    ph_orc = orc.lib.orc_particle_horizon
    ph_orc.argtypes = h_orc.argtypes
    ph_orc.restype = ctypes.c_double
    assert abs(ph_gpu(a, FOURPIG, ctypes.byref(c)) / ph_orc(a, FOURPIG, ctypes.byref(o)) - 1) < 1e-12

    rk_gpu = gev._lib.gev_rungekutta4bg
    rk_gpu.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.c_double, ctypes.POINTER(gev.Cosmo), ctypes.c_double]
    rk_gpu.restype = None
    rk_orc = orc.lib.orc_rk4bg
    rk_orc.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.c_double, ctypes.POINTER(OrcCosmo), ctypes.c_double]
    rk_orc.restype = None
    a1, a2 = ctypes.c_double(a), ctypes.c_double(a)
    dtau = 0.01 / h_orc(a, FOURPIG, ctypes.byref(o))
    rk_gpu(ctypes.byref(a1), FOURPIG, ctypes.byref(c), dtau)
    rk_orc(ctypes.byref(a2), FOURPIG, ctypes.byref(o), dtau)
    assert a1.value > a
    assert abs(a1.value / a2.value - 1) < 1e-14


def test_roofline_model_consistency():
    from gevb200 import roofline
    for N in (64, 512):
        for prec in ("mixed", "fp64"):
            total = roofline.step_bytes(N, prec)
            P = roofline.PARTICLE_BYTES[prec]
            F = roofline.FIELD_BYTES[prec]
            assert total == sum(roofline.stage_bytes(s, N, prec) for s in roofline.STAGES[prec])
            if prec == "fp64":
                # 2 deposits + kick/drift read particles 4 times in total (kick/drift reads and writes)
                assert total == N ** 3 * (4 * P + 55 * F)
            else:
                # one deposit: particles 3 times; the T0i sums add phi to the B solve's reads
                assert total == N ** 3 * (3 * P + 55 * F)

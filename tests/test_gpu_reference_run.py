"""Whole runs against the reference's own code, from the same configuration.

The reference side runs on the host cores from oracle/_ref (the reference's
own sources with the single-rank LATfield2 stand-in): its initial-condition
generator (ref_ics_basic: generateIC_basic's tabulated-spectrum branch with
the sc1 template tiled N/4 times, k-sphere, corrected displacement, as the
configurations set it) and then ref_step, one cycle of main.cu:608-1317 at a
time.  The library side generates the same initial conditions with
gev_ics_basic (FP64 context) and runs gev_step on the GPU -- in FP64, and in
mixed precision from the FP64 context's initial state.  Both run the same
number of cycles.

Compared at the end, as the north star states them:
  * the matter power spectrum, the reference's extractPowerSpectrum
    (tools.hpp:65-314) of its CIC density against gev_power_spectrum, over the
    occupied bins below half the Nyquist wavenumber: max relative error;
  * the RMS particle displacement from the initial lattice positions:
    relative error of the RMS, and the RMS of the per-particle displacement
    difference relative to the RMS displacement.
Tolerance 1e-4 relative for the power spectrum and the RMS displacement, FP64
and mixed precision.  FP64 also matches particle by particle (1e-6).

Setting GEV_VALIDATION_REPORT to a file path writes the measured errors there
as JSON lines."""
import ctypes
import json
import math
import os

import numpy as np
import pytest

from _libs import oracle, ptr, ref

gev = pytest.importorskip("gevb200")
from gevb200.ics import linear_pk, sc1_template  # noqa: E402

pytestmark = pytest.mark.gpu

C_LIGHT = 2997.92458
OM, OL, H_LITTLE = 0.32, 0.68, 0.67


class _Sim(ctypes.Structure):   # orc_sim (oracle.h)
    _fields_ = [("N", ctypes.c_int), ("boxsize", ctypes.c_double), ("fourpiG", ctypes.c_double),
                ("mass", ctypes.c_double), ("Om", ctypes.c_double), ("OL", ctypes.c_double),
                ("Orad", ctypes.c_double), ("z_relax", ctypes.c_double), ("Cf", ctypes.c_double),
                ("steplimit", ctypes.c_double), ("with_B", ctypes.c_int)]


class _State(ctypes.Structure):   # orc_state
    _fields_ = [("a", ctypes.c_double), ("tau", ctypes.c_double), ("dtau", ctypes.c_double),
                ("dtau_old", ctypes.c_double), ("cycle", ctypes.c_int), ("T00hom", ctypes.c_double),
                ("phi_hom", ctypes.c_double), ("maxvel", ctypes.c_double)]


def _reference():
    r = ref()
    if r is None:
        pytest.skip("reference CPU build (oracle/_ref) not present")
    r.lib.ref_step.argtypes = [ctypes.POINTER(_Sim), ctypes.POINTER(_State), ctypes.c_int64] + [ctypes.c_void_p] * 5
    r.lib.ref_step.restype = None
    return r


def _report(rec):
    path = os.environ.get("GEV_VALIDATION_REPORT")
    print(json.dumps(rec))
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(rec) + "\n")


def _table(a0):
    kt = np.logspace(-5, 3, 4096)
    return kt, linear_pk(kt, a0, H_LITTLE, OM)


def _ref_ics(N, box, a0, seed):
    """The reference generator's particles (ID order), phi, chi and B_i."""
    r = _reference()
    fourpiG = 1.5 * box * box / C_LIGHT ** 2
    kt, pt = _table(a0)
    tmpl = sc1_template()
    n = N ** 3
    pos, q, ids = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(n, dtype=np.int64)
    phi, chi, Bi, mv = np.zeros(n), np.zeros(n), np.zeros(3 * n), np.zeros(1)
    rc = r.ics_basic(N, box, a0, fourpiG, OM, OL, 0.0, ptr(kt), ptr(pt), len(kt), seed, 1, 1, 1, N // 4, ptr(tmpl),
                     len(tmpl), ptr(pos), ptr(q), ptr(ids), ptr(phi), ptr(chi), ptr(Bi), ptr(mv))
    assert rc == 0 and np.array_equal(ids, np.arange(n))
    return pos, q, ids, phi, chi, Bi


def _lib_ics(c, N, box, a0, seed):
    """gev_ics_basic with the same arguments into context c."""
    fourpiG = 1.5 * box * box / C_LIGHT ** 2
    kt, pt = _table(a0)
    c.ics_basic(box, a0, fourpiG, OM, OL, kt, pt, sc1_template(), N // 4, seed=seed, ksphere=True,
                correct_displacement=True, gr=True)


def _ref_spectrum(N, pos, mass, nb):
    r, o = ref(), oracle()
    rho = np.zeros(N ** 3)
    r.project_cic(N, len(pos), ptr(pos), mass, ptr(rho))
    FT = np.zeros((N, N, N // 2 + 1), dtype=np.complex128)
    o.r2c(N, ptr(rho), ptr(FT))
    out = [np.zeros(nb) for _ in range(4)]
    occ = np.zeros(nb, dtype=np.int32)
    r.power_spectrum(N, ptr(FT), nb, ptr(out[0]), ptr(out[1]), ptr(out[2]), ptr(out[3]), ptr(occ))
    return out[0], out[1], occ


def _displacement(p, p0):
    d = p - p0
    return d - np.round(d)


def _run(N, box, z_in, seed, cycles=None, nbins=1024):
    """Both codes from the same configuration; cycles=None runs to z = 0."""
    r = _reference()
    a0 = 1.0 / (1.0 + z_in)
    fourpiG = 1.5 * box * box / C_LIGHT ** 2
    mass = OM / N ** 3
    pos0, q0, ids, phi0, chi0, Bi0 = _ref_ics(N, box, a0, seed)
    cosmo = gev.Cosmo(OM, OL, 0.0, fourpiG, 48.0, 0.04, z_in, box)
    H = gev.hconf(a0, fourpiG, ctypes.byref(cosmo))
    tau0 = gev.particle_horizon(a0, fourpiG, ctypes.byref(cosmo))
    dtau0 = min(48.0 / N, 0.04 / H)

    # the reference's cycle on the host cores
    sim = _Sim(N, box, fourpiG, mass, OM, OL, 0.0, z_in, 48.0, 0.04, 1)
    st = _State(a0, tau0, dtau0, 0.0, 0, 0, 0, 0)
    p_ref, q_ref = pos0.copy(), q0.copy()
    phi, chi, Bi = phi0.copy(), chi0.copy(), Bi0.copy()
    n = 0
    while (cycles is None and 1.0 / st.a - 1.0 > 0.0) or (cycles is not None and n < cycles):
        r.lib.ref_step(ctypes.byref(sim), ctypes.byref(st), len(p_ref), ptr(p_ref), ptr(q_ref), ptr(phi), ptr(chi), ptr(Bi))
        n += 1
    kb, pk_ref, occ = _ref_spectrum(N, p_ref, mass, nb=nbins)
    d_ref = _displacement(p_ref, pos0)
    rms_ref = math.sqrt((d_ref ** 2).sum(axis=1).mean())
    sel = (occ > 0) & (kb < 0.5 * math.pi * N)

    out = {}
    # the library's initial conditions, FP64, and their distance from the reference's
    with gev.Context(N, precision=gev.FP64, capacity=N ** 3, boxsize=box) as g:
        _lib_ics(g, N, box, a0, seed)
        lp, lq, li = g.get_particles()
        lphi, lchi = g.get_field(gev.FIELD_PHI).ravel(), g.get_field(gev.FIELD_CHI).ravel()
    o = np.argsort(li)
    lp, lq, li = np.ascontiguousarray(lp[o]), np.ascontiguousarray(lq[o]), li[o]
    assert np.array_equal(li, ids)
    d0 = _displacement(pos0, (np.floor(pos0 * N) + 0.5) / N)
    ics_err = float(np.abs(_displacement(lp, pos0)).max() / np.abs(d0).max())
    for prec, name in ((gev.FP64, "fp64"), (gev.MIXED, "mixed")):
        gst = gev.State(a0, tau0, dtau0, 0.0, 0, 0.0, 0.0, 0.0)
        with gev.Context(N, precision=prec, capacity=N ** 3, boxsize=box) as c:
            if prec == gev.FP64:
                _lib_ics(c, N, box, a0, seed)
            else:
                c.set_particles(lp, lq, li, mass)
                c.set_field(gev.FIELD_PHI, lphi)
                c.set_field(gev.FIELD_CHI, lchi)
            for _ in range(n):
                c.step(cosmo, gst)
            phi_g = c.get_field(gev.FIELD_PHI).ravel()
            kb_g, pk_g, _, _, occ_g = c.power_spectrum(nbins)
            p_g, _, i_g = c.get_particles()
        o = np.argsort(i_g)
        d_g = _displacement(p_g[o], pos0)
        rms_g = math.sqrt((d_g ** 2).sum(axis=1).mean())
        diff = _displacement(p_g[o], p_ref)
        out[name] = {
            "a_rel": abs(gst.a / st.a - 1.0),
            "pk_max_rel_err": float(np.abs(pk_g[sel] / pk_ref[sel] - 1.0).max()),
            "rms_disp_rel_err": abs(rms_g / rms_ref - 1.0),
            "per_particle_disp_rel": math.sqrt((diff ** 2).sum(axis=1).mean()) / rms_ref,
            "phi_rel_err": float(np.abs(phi_g - phi).max() / np.abs(phi).max()),
            "bins_differing": int((occ_g != occ).sum()),
        }
    rec = {"N": N, "boxsize": box, "z_in": z_in, "cycles": n, "z_end": 1.0 / st.a - 1.0, "seed": seed,
           "rms_displacement_box": rms_ref, "pk_bins_compared": int(sel.sum()),
           "ics_max_disp_rel_err": ics_err, **out}
    _report(rec)
    return rec


def test_c1_run_to_z0_matches_reference():
    """Config C1: box 320 Mpc/h, 64^3 grid and particles, z = 100 -> 0 with
    Courant factor 48 and time step limit 0.04."""
    rec = _run(64, 320.0, 100.0, seed=11)
    assert rec["z_end"] <= 0.0 and rec["cycles"] > 50
    for name in ("fp64", "mixed"):
        r = rec[name]
        assert r["bins_differing"] == 0, (name, r)
        assert r["a_rel"] < 1e-13, name
        assert r["pk_max_rel_err"] < 1e-4, (name, r)
        assert r["rms_disp_rel_err"] < 1e-4, (name, r)
    assert rec["fp64"]["per_particle_disp_rel"] < 1e-6, rec["fp64"]
    assert rec["ics_max_disp_rel_err"] < 1e-7, rec


def test_c2_window_matches_reference():
    """Config C2's grid and box (1280 Mpc/h, 256^3) for a window of four
    cycles from z = 100: the production-size cycle against the reference's."""
    rec = _run(256, 1280.0, 100.0, seed=12, cycles=4)
    for name in ("fp64", "mixed"):
        r = rec[name]
        assert r["bins_differing"] == 0, (name, r)
        assert r["a_rel"] < 1e-13, name
        assert r["pk_max_rel_err"] < 1e-4, (name, r)
        assert r["rms_disp_rel_err"] < 1e-4, (name, r)
    assert rec["fp64"]["per_particle_disp_rel"] < 1e-6, rec["fp64"]
    assert rec["ics_max_disp_rel_err"] < 1e-7, rec


def test_128_run_to_z0_matches_reference():
    """Grid and particles 128^3 in a 640 Mpc/h box (5 Mpc/h cells, as the
    configurations), z = 100 -> 0: the full run against the reference's own
    initial conditions and cycle."""
    rec = _run(128, 640.0, 100.0, seed=13)
    assert rec["z_end"] <= 0.0
    for name in ("fp64", "mixed"):
        r = rec[name]
        assert r["bins_differing"] == 0, (name, r)
        assert r["a_rel"] < 1e-13, name
        assert r["pk_max_rel_err"] < 1e-4, (name, r)
        assert r["rms_disp_rel_err"] < 1e-4, (name, r)
    assert rec["fp64"]["per_particle_disp_rel"] < 1e-6, rec["fp64"]
    assert rec["ics_max_disp_rel_err"] < 1e-7, rec

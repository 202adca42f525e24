"""The particle lightcone shell against the reference's own CUDA kernels.

oracle/_ref/libgevref.so compiles Particles_gevolution.hpp's output kernels
(count_tracer_particles, buffer_tracer_IDs, count_lightcone_duplicate_ids,
buffer_tracer_particles with bufferTracerParticle's EXACT_OUTPUT_REDSHIFTS
interpolation, mark/gather_lightcone_kept_particles, the ID prelog bins) from
the reference tree, and ref_lightcone_shell runs them on the GPU in
saveGadget2's order (Particles_gevolution.hpp:1567-2165) on one rank.  These
tests pin the oracle's restatement (orc_lightcone_select) and the library's
gev_lightcone (selection, check-zone de-duplication against the previous
cycle's ID log, interpolated positions and velocities) to that code."""
import numpy as np
import pytest

from _fixtures import particles, rel_err, trough_phi
from _libs import oracle, ptr, ref

gev = pytest.importorskip("gevb200")

pytestmark = pytest.mark.gpu

MASS = 0.32 / 32768
ZONE = 0.05   # LIGHTCONE_IDCHECK_ZONE (metadata.hpp:39)


def _ref_lib():
    r = ref()
    if r is None or not hasattr(r, "lightcone_shell"):
        pytest.skip("the reference build (oracle/_ref) is not present")
    return r


def ref_shell(N, pos, q, ids, phi, vertex, direction, opening, dist, dtau, dtau_old, a, dadtau, box, tracer=1,
              scatter=1, backlog=()):
    """The reference kernels' shell: (pos, vel, ids, n_header, prelog)."""
    r = _ref_lib()
    cap = len(pos)
    op = np.zeros((cap, 3), dtype=np.float32)
    ov = np.zeros((cap, 3), dtype=np.float32)
    oi = np.zeros(cap, dtype=np.int64)
    pl = np.zeros(cap, dtype=np.int64)
    bl = np.asarray(sorted(backlog), dtype=np.int64)
    n = np.zeros(1, dtype=np.int64); nh = np.zeros(1, dtype=np.int64); npl = np.zeros(1, dtype=np.int64)
    rc = r.lightcone_shell(N, len(pos), ptr(pos), ptr(q), ptr(ids), ptr(phi), ptr(np.asarray(vertex, dtype=float)),
                           ptr(np.asarray(direction, dtype=float)), opening, dist, dtau, dtau_old, a, dadtau, box, tracer,
                           scatter, ptr(bl) if len(bl) else None, len(bl), cap, ptr(op), ptr(ov), ptr(oi), ptr(n),
                           ptr(nh), ptr(pl), ptr(npl))
    assert rc == 0, rc
    k = int(n[0])
    return op[:k], ov[:k], oi[:k], int(nh[0]), pl[:int(npl[0])]


def by_id(p, v, i):
    o = np.argsort(i)
    return p[o], v[o], i[o]


SHELLS = [
    # vertex, direction, opening, d - tau: one image (box centre), eight images (box corner), a cone
    ((0.5, 0.5, 0.5), (1.0, 0.0, 0.0), -1.0, 0.3),
    ((0.0, 0.0, 0.0), (1.0, 0.0, 0.0), -1.0, 0.35),
    ((0.1, 0.2, 0.3), (0.6, 0.0, 0.8), 0.7, 0.4),
]


@pytest.mark.parametrize("shell", range(len(SHELLS)))
@pytest.mark.parametrize("use_phi", [True, False])
def test_oracle_selection_matches_reference_kernels(shell, use_phi):
    """orc_lightcone_select (selection, images, interpolated position and
    velocity) against buffer_tracer_particles on an empty ID log."""
    import ctypes
    N = 32
    pos, q, ids = particles(N, seed=21, lattice=True, disp=0.45, qscale=1e-3)
    phi = trough_phi(N, 1e-5) if use_phi else None
    vertex, direction, opening, dist = SHELLS[shell]
    a, dadtau, box, dtau, dtau_old = 0.5, 0.4, 320.0, 0.02, 0.018
    rp, rv, ri, nh, _ = ref_shell(N, pos, q, ids, phi, vertex, direction, opening, dist, dtau, dtau_old, a, dadtau, box)
    assert len(ri) > 100 and nh == len(ri)

    class OLc(ctypes.Structure):
        _fields_ = [("vertex", ctypes.c_double * 3), ("direction", ctypes.c_double * 3), ("opening", ctypes.c_double),
                    ("dist_lo", ctypes.c_double), ("dist_hi", ctypes.c_double)]

    o = oracle()
    cap = len(pos)
    op = np.zeros((cap, 3), dtype=np.float32); ov = np.zeros((cap, 3), dtype=np.float32)
    oi = np.zeros(cap, dtype=np.int64)
    ol = OLc(vertex, direction, opening, 0.0, dist)
    n = o.lightcone_select(N, len(pos), ptr(pos), ptr(q), ptr(ids), ptr(phi), ctypes.byref(ol), 1.0, dtau, dtau_old,
                           a, dadtau, cap, ptr(op), ptr(ov), ptr(oi), box)
    assert n == len(ri)
    rp, rv, ri = by_id(rp, rv, ri)
    op, ov, oi = by_id(op[:n], ov[:n], oi[:n])
    assert np.array_equal(ri, oi)
    assert rel_err(op, rp) < 1e-6
    assert rel_err(ov, rv) < 1e-6


@pytest.mark.parametrize("prec", [gev.FP64, gev.MIXED])
@pytest.mark.parametrize("shell", range(len(SHELLS)))
@pytest.mark.parametrize("tracer", [1, 3])
def test_library_shell_matches_reference_kernels(prec, shell, tracer):
    """Two consecutive cycles of one shell: gev_lightcone against the
    reference kernels, the second cycle de-duplicated against the IDs the
    first one logged (the reference's backlog is that prelog, sorted and made
    unique as LightconeIDBacklog::finalize does)."""
    N = 32
    pos, q, ids = particles(N, seed=22, lattice=True, disp=0.45, qscale=1e-3)
    phi = trough_phi(N, 1e-5)
    vertex, direction, opening, dist0 = SHELLS[shell]
    a, dadtau, box, dtau = 0.5, 0.4, 320.0, 0.02
    d_h = 1.0 + dist0
    lc = gev.LightconeArgs(vertex, direction, opening, (dist0 + 0.2, dist0 - 0.2), d_h, tracer, 0)
    backlog = ()
    deduplicated = 0
    with gev.Context(N, precision=prec, capacity=len(pos), boxsize=box) as c:
        c.set_particles(pos, q, ids, MASS)
        c.set_field(gev.FIELD_PHI, phi)
        for cyc, tau in enumerate((1.0, 1.0 + dtau)):
            gp, gv, gi = c.lightcone(lc, tau, dtau, dtau, a, dadtau, len(pos))
            rp, rv, ri, nh, prelog = ref_shell(N, pos, q, ids, phi, vertex, direction, opening, d_h - tau, dtau, dtau,
                                               a, dadtau, box, tracer=tracer, backlog=backlog)
            assert len(ri) > 20 and nh == len(ri)
            if cyc == 1:
                # how many of this cycle's check zone the last cycle logged
                r_all = ref_shell(N, pos, q, ids, phi, vertex, direction, opening, d_h - tau, dtau, dtau, a, dadtau,
                                  box, tracer=tracer)[2]
                deduplicated = len(r_all) - len(ri)
            backlog = prelog
            gp, gv, gi = by_id(gp, gv, gi)
            rp, rv, ri = by_id(rp, rv, ri)
            assert np.array_equal(gi, ri)
            tol = 1e-6 if prec == gev.FP64 else 1e-4
            assert rel_err(gp, rp) < tol
            assert rel_err(gv, rv) < tol
    if shell < 2 and tracer == 1:   # full-sky shells: the overlap is populated
        assert deduplicated > 0


def test_prelog_bins_hold_the_same_ids():
    """saveGadget2<1> (nine ID-log bins by the rank's domain edges) and
    saveGadget2<0> (one bin) log the same IDs on one rank."""
    N = 32
    pos, q, ids = particles(N, seed=23, lattice=True, disp=0.45, qscale=1e-3)
    vertex, direction, opening, dist = SHELLS[1]
    args = (N, pos, q, ids, None, vertex, direction, opening, dist, 0.02, 0.02, 0.5, 0.4, 320.0)
    p1 = ref_shell(*args, scatter=1)[4]
    p0 = ref_shell(*args, scatter=0)[4]
    assert len(p0) > 0 and sorted(p0) == sorted(p1)

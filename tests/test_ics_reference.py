"""gev_ics_basic against the reference's own initial-condition generator.

oracle/_ref/libgevref.so compiles ic_basic.hpp from the reference tree, and
ref_ics_basic calls its generateIC_basic as main.cu does for a tabulated
power spectrum (the spectrum and the particle template are written to files
that loadPowerSpectrum and loadHomogeneousTemplate read).  The CPU tests pin
the two pieces this build restates from published algorithms: the random
stream (sitmo::prng_engine = Threefry-4x64-20, against the reference's
prng_engine.hpp) and the natural cubic spline that stands in for GSL's
cspline (against scipy).  The GPU tests compare whole initial conditions:
particle positions and momenta by ID, phi, chi and B_i."""
import numpy as np
import pytest

from _fixtures import rel_err
from _libs import ptr, ref

gev = pytest.importorskip("gevb200")


def _ref():
    r = ref()
    if r is None or not hasattr(r, "ics_basic"):
        pytest.skip("the reference build (oracle/_ref) is not present")
    return r


def test_sitmo_stream_matches_reference_engine():
    """gev_sitmo_words against sitmo::prng_engine (seed, discard, draws) at
    the stream offsets generateDisplacementField uses."""
    r = _ref()
    H = 65536
    for seed in (0, 1, 42, 2 ** 31 + 7, 2 ** 32 - 1):
        for start in (0, 3, 8, 9, 17 * H, ((H + 5) * H + 200) * H, ((3 * H + 511) * H + 300) * H + 77):
            want = np.zeros(300, dtype=np.uint32)
            r.sitmo_words(seed, start, len(want), ptr(want))
            got = gev.sitmo_words(seed, start, len(want))
            assert np.array_equal(got, want), (seed, start)


def test_spline_standin_matches_scipy():
    """The GSL cspline stand-in is the natural cubic spline."""
    from scipy.interpolate import CubicSpline
    r = _ref()
    rng = np.random.default_rng(3)
    x = np.sort(rng.uniform(0.0, 10.0, 40))
    y = np.sin(x) + 0.1 * rng.standard_normal(40)
    v = np.concatenate([np.linspace(x[0], x[-1], 997), x])
    out = np.zeros_like(v)
    r.spline_eval(ptr(x), ptr(y), len(x), ptr(v), len(v), ptr(out))
    want = CubicSpline(x, y, bc_type="natural")(v)
    assert np.max(np.abs(out - want)) < 1e-12 * np.max(np.abs(want))


def test_sc1_template_holds_the_reference_positions():
    """gevb200.ics.sc1_template() has the positions of the reference's
    sc1_crystal.dat (read where the reference tree is present)."""
    import os
    import struct
    from gevb200.ics import sc1_template
    t = sc1_template()
    assert t.shape == (64, 3) and t.dtype == np.float32
    path = os.path.join(os.environ.get("GEV_REFERENCE_DIR", "/root/reference"), "sc1_crystal.dat")
    if not os.path.exists(path):
        pytest.skip("the reference tree is not present")
    b = open(path, "rb").read()
    n = struct.unpack("<I", b[:4])[0]
    npart = struct.unpack("<6I", b[4:28])[1]
    box = struct.unpack("<d", b[4 + 128:4 + 136])[0]          # gadget2_header.BoxSize
    start = 4 + n + 4 + 4
    pos = np.frombuffer(b[start:start + 12 * npart], dtype="<f4").reshape(-1, 3) / np.float32(box)
    assert npart == 64
    assert sorted(map(tuple, pos.tolist())) == sorted(map(tuple, t.tolist()))


def template_4x4x4(seed=5):
    """A 64-particle simple-cubic template, (i + 1/2) / 4 per axis (the
    positions of the reference's sc1 template), in a seeded order."""
    g = (np.arange(4) + 0.5) / 4.0
    t = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1).reshape(-1, 3)
    return t[np.random.default_rng(seed).permutation(64)].astype(np.float32)


def pk_table():
    from gevb200.ics import linear_pk
    k = np.logspace(-4, 1.5, 600)
    return k, linear_pk(k, 1.0 / 101.0, 0.67, 0.32)


CASES = [
    # correct displacement, k-sphere, GR
    (True, True, True),
    (False, False, True),
    (True, False, False),
]


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [gev.FP64, gev.MIXED])
@pytest.mark.parametrize("case", range(len(CASES)))
def test_ics_basic_matches_reference_generator(prec, case):
    correct, ksphere, gr = CASES[case]
    r = _ref()
    N, T = 32, 8
    box = 5.0 * N
    a = 1.0 / 101.0
    fourpiG = 1.5 * box * box / 2997.92458 ** 2
    Om, OL = 0.32, 0.68
    seed = 20260101 + case
    tmpl = template_4x4x4()
    k, pk = pk_table()
    np_ = len(tmpl) * T ** 3
    pos = np.zeros((np_, 3)); q = np.zeros((np_, 3)); ids = np.zeros(np_, dtype=np.int64)
    phi = np.zeros(N ** 3); chi = np.zeros(N ** 3); Bi = np.zeros(3 * N ** 3); mv = np.zeros(1)
    rc = r.ics_basic(N, box, a, fourpiG, Om, OL, 0.0, ptr(k), ptr(pk), len(k), seed, int(ksphere), int(correct),
                     int(gr), T, ptr(tmpl), len(tmpl), ptr(pos), ptr(q), ptr(ids), ptr(phi), ptr(chi), ptr(Bi), ptr(mv))
    assert rc == 0
    assert np.array_equal(ids, np.arange(np_))
    with gev.Context(N, precision=prec, capacity=np_, boxsize=box) as c:
        c.ics_basic(box, a, fourpiG, Om, OL, k, pk, tmpl, T, seed=seed, ksphere=ksphere, correct_displacement=correct,
                    gr=gr)
        gp, gq, gi = c.get_particles()
        o = np.argsort(gi)
        gp, gq, gi = gp[o], gq[o], gi[o]
        assert np.array_equal(gi, ids)
        # displacements from the template lattice (periodic difference)
        t = np.arange(np_)
        j, tt = t % len(tmpl), t // len(tmpl)
        tile = np.stack([tt % T, (tt // T) % T, tt // T ** 2], axis=1)
        x0 = (tile + tmpl[j].astype(np.float64)) / T
        dref = (pos - x0 + 0.5) % 1.0 - 0.5
        dgpu = (gp - x0 + 0.5) % 1.0 - 0.5
        # FP64: the amplitudes r1 are FP32 in both (boxMullerRadialAmplitude);
        # the reference takes glibc's logf on the host, the GPU an FP64 log
        # rounded once, so a few modes may differ by one FP32 ulp (6e-8 of
        # that mode) -- a wrong stream or kernel shows at the 1e-2 level
        tol = 1e-7 if prec == gev.FP64 else 2e-5
        assert np.max(np.abs(dref)) > 1e-4
        assert rel_err(dgpu, dref) < tol
        assert rel_err(gq, q) < tol
        tol_f = 1e-7 if prec == gev.FP64 else 1e-4
        assert rel_err(c.get_field(gev.FIELD_PHI), phi) < tol_f
        assert rel_err(c.get_field(gev.FIELD_CHI), chi) < tol_f
        g = c.get_field(gev.FIELD_BI)
        for comp in range(3):
            assert rel_err(g[comp], Bi[comp * N ** 3:(comp + 1) * N ** 3]) < tol_f, comp


@pytest.mark.gpu
def test_ics_basic_arguments():
    """Template, table and capacity checks (the reference aborts on these)."""
    N = 32
    k, pk = pk_table()
    tmpl = template_4x4x4()
    with gev.Context(N, precision=gev.MIXED, capacity=N ** 3, boxsize=160.0) as c:
        with pytest.raises(gev.GevError):
            c.ics_basic(160.0, 0.01, 1e-3, 0.32, 0.68, k, pk, tmpl, 9)            # 64 * 9^3 > capacity
        with pytest.raises(gev.GevError):
            c.ics_basic(160.0, 0.01, 1e-3, 0.32, 0.68, k[200:300], pk[200:300], tmpl, 8)   # table too narrow
        with pytest.raises(gev.GevError):
            c.ics_basic(160.0, 0.01, 1e-3, 0.32, 0.68, k, pk, tmpl * 2.0, 8)      # template outside [0, 1]

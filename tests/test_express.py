"""Express particle files (gev_express_write / gev_express_read) against the
reference's own saveExpress / loadExpress (Particles_gevolution.hpp:98-143,
:2641-2902), compiled into oracle/_ref: files written by either are read by
the other with the same particles, IDs and Gadget-2 header."""
import ctypes
import os

import numpy as np
import pytest

from _fixtures import particles
from _libs import ptr, ref

gev = pytest.importorskip("gevb200")
from gevb200 import gadget2  # noqa: E402

pytestmark = pytest.mark.gpu

MASS = 0.32 / 32768


def _ref():
    r = ref()
    if r is None or not hasattr(r, "express_write"):
        pytest.skip("the reference build (oracle/_ref) is not present")
    return r


def _hdr():
    return gadget2.header(0.25, 320.0, 0.32, 0.68, 0.67, 32 ** 3)


@pytest.mark.parametrize("prec", [gev.FP64, gev.MIXED])
def test_library_file_read_by_reference(tmp_path, prec):
    r = _ref()
    N = 32
    pos, q, ids = particles(N, n=20000, seed=41, qscale=0.01)
    with gev.Context(N, precision=prec, capacity=len(pos)) as c:
        c.set_particles(pos, q, ids, MASS)
        gp, gq, gi = c.get_particles()
        gadget2.express_write(c, tmp_path / "snap.17", _hdr(), real_bytes=8)
    assert os.path.exists(tmp_path / "snap.0") and not os.path.exists(tmp_path / "snap.17")
    cap = len(pos)
    rp, rq, ri = np.zeros((cap, 3)), np.zeros((cap, 3)), np.zeros(cap, dtype=np.int64)
    n = np.zeros(1, dtype=np.int64)
    h = gadget2.Gadget2Header()
    assert r.express_read(str(tmp_path / "snap").encode(), N, cap, ptr(rp), ptr(rq), ptr(ri), ptr(n),
                          ctypes.addressof(h)) == 0
    assert n[0] == len(pos)
    assert np.array_equal(ri, gi) and np.array_equal(rp, gp) and np.array_equal(rq, gq)
    assert h.npart[1] == len(pos) and h.npartTotal[1] == len(pos) and h.num_files == 1 and h.time == 0.25


def test_reference_file_read_by_library(tmp_path):
    r = _ref()
    N = 32
    pos, q, ids = particles(N, n=20000, seed=42, qscale=0.01)
    h = _hdr()
    h.num_files = 1
    assert r.express_write(str(tmp_path / "dump").encode(), N, len(pos), ptr(pos), ptr(q), ptr(ids),
                           ctypes.addressof(h)) == 0
    with gev.Context(N, precision=gev.FP64, capacity=len(pos)) as c:
        got = gadget2.express_read(c, tmp_path / "dump", MASS)
        gp, gq, gi = c.get_particles()
    o = np.argsort(gi)
    assert np.array_equal(gi[o], ids)
    assert np.abs(gp[o] - pos).max() < 1e-15 and np.array_equal(gq[o], q)
    assert got.npartTotal[1] == len(pos) and got.time == 0.25


def test_float_files_and_layout_checks(tmp_path):
    """Real = float round trip (a single-precision build's files), and the
    reader rejects a file of another lattice."""
    N = 32
    pos, q, ids = particles(N, n=5000, seed=43, qscale=0.01)
    with gev.Context(N, precision=gev.MIXED, capacity=len(pos)) as c:
        c.set_particles(pos, q, ids, MASS)
        gadget2.express_write(c, tmp_path / "f", _hdr(), real_bytes=4)
    assert os.path.getsize(tmp_path / "f.0") == 120 + len(pos) * (24 + 8) + 256
    with gev.Context(N, precision=gev.FP64, capacity=len(pos)) as c:
        gadget2.express_read(c, tmp_path / "f", MASS)
        gp, gq, gi = c.get_particles()
    o = np.argsort(gi)
    assert np.array_equal(gi[o], ids)
    assert np.abs(gp[o] - pos.astype(np.float32)).max() < 1e-15
    assert np.array_equal(gq[o], q.astype(np.float32).astype(np.float64))
    with gev.Context(16, precision=gev.FP64, capacity=len(pos)) as c:
        with pytest.raises(gev.GevError):
            gadget2.express_read(c, tmp_path / "f", MASS)

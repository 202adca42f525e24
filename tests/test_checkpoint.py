"""Checkpoint and restart: a run continued from a checkpoint gives the
particles and fields of the uninterrupted run -- to FP64 rounding, since
positions round-trip through box-unit doubles as in the reference's particle
files; a checkpoint restored into a context of the other precision continues
within that precision's tolerance; mismatched contexts and corrupt files are
rejected."""
import ctypes

import numpy as np
import pytest

from _fixtures import particles, rel_err

gev = pytest.importorskip("gevb200")
from gevb200.ics import hconf  # noqa: E402

pytestmark = pytest.mark.gpu


def _setup(N, prec, vector_method=gev.VECTOR_ELLIPTIC, tensor=False):
    import torch
    from gevb200.ics import zeldovich
    box = 5.0 * N
    pos, q, ids, phi, mass, a0, fourpiG = zeldovich(N, box, 100.0, 3, device="cuda")
    pos, q, ids, phi = pos.cpu().numpy(), q.cpu().numpy(), ids.cpu().numpy(), phi.cpu().numpy()
    cosmo = gev.Cosmo(0.32, 0.68, 0.0, fourpiG, 48.0, 0.04, 100.0, box)
    H = gev.hconf(a0, fourpiG, ctypes.byref(cosmo))
    tau0 = gev.particle_horizon(a0, fourpiG, ctypes.byref(cosmo))
    st = gev.State(a0, tau0, min(48.0 / N, 0.04 / H), 0.0, 0, 0.0, 0.0, 0.0)

    def make(p=prec):
        c = gev.Context(N, precision=p, capacity=len(pos), boxsize=box, vector_method=vector_method, tensor=tensor)
        c.set_particles(pos, q, ids, mass)
        c.set_field(gev.FIELD_PHI, phi)
        return c
    return make, cosmo, st


def _snapshot(c):
    p, q, i = c.get_particles()
    o = np.argsort(i)
    return p[o], q[o], c.get_field(gev.FIELD_PHI), c.get_field(gev.FIELD_CHI)


@pytest.mark.parametrize("vector_method,tensor", [(gev.VECTOR_ELLIPTIC, False), (gev.VECTOR_PARABOLIC, True)])
def test_restart_continues_the_run(tmp_path, vector_method, tensor):
    make, cosmo, st = _setup(32, gev.FP64, vector_method, tensor)
    with make() as c:
        for _ in range(3):
            c.step(cosmo, st)
        c.checkpoint_write(tmp_path / "ck", st)
        for _ in range(2):
            c.step(cosmo, st)
        ref = _snapshot(c)
        a_ref = st.a
    with gev.Context(32, precision=gev.FP64, capacity=32 ** 3, boxsize=160.0, vector_method=vector_method,
                     tensor=tensor) as c2:
        st2 = c2.checkpoint_read(tmp_path / "ck")
        for _ in range(2):
            c2.step(cosmo, st2)
        got = _snapshot(c2)
        assert st2.a == a_ref
    d = got[0] - ref[0]
    d -= np.round(d)                                  # periodic positions
    assert np.abs(d).max() < 1e-12
    for x, y in zip(ref[1:], got[1:]):
        assert rel_err(y, x) < 1e-10


def test_restore_into_mixed_context(tmp_path):
    make, cosmo, st = _setup(32, gev.FP64)
    with make() as c:
        for _ in range(2):
            c.step(cosmo, st)
        c.checkpoint_write(tmp_path / "ck", st)
        c.step(cosmo, st)
        ref = _snapshot(c)
    with gev.Context(32, precision=gev.MIXED, capacity=32 ** 3, boxsize=160.0) as c2:
        st2 = c2.checkpoint_read(tmp_path / "ck")
        c2.step(cosmo, st2)
        got = _snapshot(c2)
    assert rel_err(got[1], ref[1]) < 1e-4          # momenta
    assert rel_err(got[2], ref[2]) < 1e-4          # phi


def test_rejects_mismatch_and_garbage(tmp_path):
    make, cosmo, st = _setup(32, gev.MIXED)
    with make() as c:
        c.checkpoint_write(tmp_path / "ck", st)
    with gev.Context(16, precision=gev.MIXED, capacity=32 ** 3, boxsize=160.0) as c16:
        with pytest.raises(gev.GevError):
            c16.checkpoint_read(tmp_path / "ck")
    (tmp_path / "bad").write_bytes(b"not a checkpoint at all")
    with gev.Context(32, precision=gev.MIXED, capacity=32 ** 3, boxsize=160.0) as c32:
        with pytest.raises(gev.GevError):
            c32.checkpoint_read(tmp_path / "bad")
        raw = (tmp_path / "ck").read_bytes()
        # a truncated file is refused and leaves the context as it was
        pos, q, ids = particles(32, n=500, seed=99)
        c32.set_particles(pos, q, ids, 1e-3)
        before = c32.get_particles()
        (tmp_path / "short").write_bytes(raw[: len(raw) - 1000])
        with pytest.raises(gev.GevError):
            c32.checkpoint_read(tmp_path / "short")
        for x, y in zip(c32.get_particles(), before):
            assert np.array_equal(x, y)
    # a different box size is refused
    with gev.Context(32, precision=gev.MIXED, capacity=32 ** 3, boxsize=320.0) as cbox:
        with pytest.raises(gev.GevError, match="box size"):
            cbox.checkpoint_read(tmp_path / "ck")

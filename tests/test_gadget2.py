"""Gadget-2 output: the file layout of the reference's saveGadget2 (header,
POS, VEL, ID blocks with 32-bit record lengths) written by the C ABI and read
back; the snapshot of a context's particles on the GPU."""
import ctypes
import struct

import numpy as np
import pytest

gev = pytest.importorskip("gevb200")
from gevb200 import gadget2  # noqa: E402


def test_write_and_read_back(tmp_path):
    rng = np.random.default_rng(1)
    n = 1000
    pos = rng.random((n, 3)).astype(np.float32) * 1e5
    vel = rng.standard_normal((n, 3)).astype(np.float32)
    ids = rng.permutation(10 * n)[:n].astype(np.int64)
    hdr = gadget2.header(0.5, 2560.0, 0.32, 0.68, 0.67, 512 ** 3)
    path = tmp_path / "lc_0001_cdm"
    gadget2.write(path, hdr, pos, vel, ids)
    raw = open(path, "rb").read()
    # record lengths exactly as the reference writes them
    assert struct.unpack_from("<I", raw, 0)[0] == 256
    assert struct.unpack_from("<I", raw, 4 + 256)[0] == 256
    assert struct.unpack_from("<I", raw, 264)[0] == 12 * n
    assert len(raw) == 4 * 8 + 256 + 24 * n + 8 * n
    h2, p2, v2, i2 = gadget2.read(path)
    assert h2.npart[1] == n and h2.npartTotal[1] == n and h2.npartTotalHW[1] == 0
    assert h2.BoxSize == 2560.0 / 0.001 and h2.time == 0.5 and h2.redshift == 1.0
    assert abs(h2.mass[1] - 2.77459457e11 * 0.32 * 2560.0 ** 3 / 512 ** 3 / 1e10) < 1e-9
    assert np.array_equal(p2, pos) and np.array_equal(v2, vel) and np.array_equal(i2, ids)


def test_empty_file(tmp_path):
    hdr = gadget2.header(1.0, 100.0, 0.3, 0.7, 0.7, 64 ** 3)
    gadget2.write(tmp_path / "empty", hdr, np.zeros((0, 3)), np.zeros((0, 3)), np.zeros(0, np.int64))
    h, p, v, i = gadget2.read(tmp_path / "empty")
    assert h.npart[1] == 0 and len(p) == 0 and len(i) == 0


@pytest.mark.gpu
def test_snapshot_of_context_particles(tmp_path):
    from _fixtures import particles
    N = 32
    pos, q, ids = particles(N, n=20000, seed=9)
    a = 0.25
    with gev.Context(N, precision=gev.FP64, capacity=len(pos), boxsize=320.0) as c:
        c.set_particles(pos, q, ids, 1e-5)
        hdr = gadget2.header(a, 320.0, 0.32, 0.68, 0.67, len(pos), tracer_factor=2)
        gadget2.snapshot(c, tmp_path / "snap", hdr, tracer_factor=2)
    h, p, v, i = gadget2.read(tmp_path / "snap")
    sel = ids % 2 == 0
    order = np.argsort(i)
    ref_order = np.argsort(ids[sel])
    assert np.array_equal(i[order], ids[sel][ref_order])
    box = 320.0 / 0.001
    np.testing.assert_allclose(p[order], (pos[sel][ref_order] * box).astype(np.float32), rtol=1e-6, atol=1e-3)
    vscale = 1.0 / np.sqrt(a) / 3.335640952e-6 / a
    np.testing.assert_allclose(v[order], (q[sel][ref_order] * vscale).astype(np.float32), rtol=1e-6)


def test_c_reader_matches_python_reader_and_rejects_bad_files(tmp_path):
    """gev_gadget2_read against the independent Python parse, plus its
    refusals: too small a capacity, a truncated file, a second species."""
    rng = np.random.default_rng(3)
    n = 777
    pos = rng.random((n, 3)).astype(np.float32) * 1e5
    vel = rng.standard_normal((n, 3)).astype(np.float32)
    ids = rng.permutation(10 * n)[:n].astype(np.int64)
    hdr = gadget2.header(0.25, 320.0, 0.32, 0.68, 0.67, 64 ** 3)
    path = tmp_path / "snap"
    gadget2.write(path, hdr, pos, vel, ids)
    h, p, v, i = gadget2.read_c(path)
    hp, pp, vp, ip = gadget2.read(path)
    assert bytes(h) == bytes(hp)
    assert np.array_equal(p, pp) and np.array_equal(v, vp) and np.array_equal(i, ip)
    assert np.array_equal(p, pos) and np.array_equal(i, ids)
    small = np.empty((10, 3), np.float32)
    nn = ctypes.c_int64()
    rc = gadget2._read(str(path).encode(), ctypes.byref(gadget2.Gadget2Header()), small.ctypes.data_as(ctypes.c_void_p),
                       small.ctypes.data_as(ctypes.c_void_p), np.empty(10, np.int64).ctypes.data_as(ctypes.c_void_p), 10,
                       ctypes.byref(nn))
    assert rc == gev.GEV_ERR_CAPACITY and nn.value == n
    raw = open(path, "rb").read()
    (tmp_path / "short").write_bytes(raw[:-100])
    with pytest.raises(gev.GevError):
        gadget2.read_c(tmp_path / "short")
    bad = gadget2.header(0.25, 320.0, 0.32, 0.68, 0.67, 64 ** 3)
    gadget2.write(tmp_path / "two", bad, pos, vel, ids)
    raw = bytearray(open(tmp_path / "two", "rb").read())
    struct.pack_into("<I", raw, 4, 5)          # npart[0] = 5: a second species
    (tmp_path / "two").write_bytes(bytes(raw))
    with pytest.raises(gev.GevError):
        gadget2.read_c(tmp_path / "two")


@pytest.mark.gpu
def test_load_particle_file_inverts_the_snapshot(tmp_path):
    """A snapshot read back into a context (the reference's particle-file
    ICs): positions and momenta to FP32 rounding of the file, IDs exact."""
    from _fixtures import particles
    N = 32
    pos, q, ids = particles(N, n=20000, seed=19)
    a, box = 0.3, 320.0
    with gev.Context(N, precision=gev.FP64, capacity=len(pos), boxsize=box) as c:
        c.set_particles(pos, q, ids, 1e-5)
        gadget2.snapshot(c, tmp_path / "snap", gadget2.header(a, box, 0.32, 0.68, 0.67, len(pos)), tracer_factor=1)
    with gev.Context(N, precision=gev.FP64, capacity=len(pos), boxsize=box) as c2:
        h = gadget2.load(c2, tmp_path / "snap", 1e-5)
        assert h.time == a
        p2, q2, i2 = c2.get_particles()
    o, r = np.argsort(i2), np.argsort(ids)
    assert np.array_equal(i2[o], ids[r])
    d = p2[o] - pos[r]
    d -= np.round(d)
    assert np.abs(d).max() < 1e-6
    np.testing.assert_allclose(q2[o], q[r], rtol=1e-6, atol=1e-12)

"""Zel'dovich initial conditions on the GPU (gev_ics_zeldovich):
- the white noise is the Philox4x32-10 stream restated in numpy below (its
  implementation is checked against the published known-answer vectors first);
- with a given noise field and a power-law P(k), the particle positions are
  the numpy Zel'dovich displacement of the cell-centre lattice;
- phi and the momenta follow the reference's mPk branch, recomputed with the
  oracle from the GPU's own particle positions."""
import ctypes

import numpy as np
import pytest

from _fixtures import rel_err
from _libs import kshape, oracle, ptr

gev = pytest.importorskip("gevb200")

M0, M1, W0, W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85


def philox(ctr, key):
    """Philox4x32-10 on numpy uint64 arrays (one counter per element)."""
    c = [np.asarray(x, dtype=np.uint64) for x in ctr]
    k0, k1 = np.uint64(key[0]), np.uint64(key[1])
    mask = np.uint64(0xffffffff)
    for r in range(10):
        if r > 0:
            k0 = (k0 + np.uint64(W0)) & mask
            k1 = (k1 + np.uint64(W1)) & mask
        p0 = np.uint64(M0) * c[0]
        p1 = np.uint64(M1) * c[2]
        c = [(p1 >> np.uint64(32)) ^ c[1] ^ k0, p1 & mask, (p0 >> np.uint64(32)) ^ c[3] ^ k1, p0 & mask]
    return c


def test_philox_known_answers():
    # Salmon et al. (2011) / Random123 known-answer vectors for philox4x32-10
    for ctr, key, out in [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
                          ((0xffffffff,) * 4, (0xffffffff,) * 2, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
                          ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
                           (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]:
        got = philox([np.array([v], dtype=np.uint64) for v in ctr], key)
        assert tuple(int(x[0]) for x in got) == out


def noise_stream(N, seed):
    i = np.arange(N ** 3, dtype=np.uint64)
    c = philox([i & np.uint64(0xffffffff), i >> np.uint64(32), np.zeros_like(i), np.zeros_like(i)],
               (seed & 0xffffffff, seed >> 32))
    u1 = (c[0].astype(np.float64) + 0.5) / 4294967296.0
    u2 = c[1].astype(np.float64) / 4294967296.0
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


BOX, A, OM, OL = 160.0, 1.0 / 51.0, 0.32, 0.68


def _pk_table():
    k = np.logspace(-3, 2, 64)
    return k, 1e3 * (k / 0.1) ** -1.5          # a power law: exact under ln-ln interpolation


def _fourpiG():
    return 1.5 * BOX ** 2 / 2997.92458 ** 2


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [0, 12345678901])
def test_device_noise_is_the_philox_stream(seed):
    N = 16
    k, pk = _pk_table()
    with gev.Context(N, precision=gev.FP64, capacity=N ** 3, boxsize=BOX) as c:
        w = c.ics_zeldovich(BOX, A, _fourpiG(), OM, OL, k, pk, seed=seed, return_noise=True)
    ref = noise_stream(N, seed)
    assert np.max(np.abs(w - ref)) < 1e-12
    assert abs(w.mean()) < 0.1 and abs(w.std() - 1.0) < 0.1


def _zeldovich_numpy(N, w, k_tab, p_tab):
    W = np.fft.rfftn(w.reshape(N, N, N))
    kf = np.fft.fftfreq(N, 1.0 / N)
    kh = np.fft.rfftfreq(N, 1.0 / N)
    kz, ky, kx = np.meshgrid(kf, kf, kh, indexing="ij")
    kk = kx * kx + ky * ky + kz * kz
    kphys = 2 * np.pi * np.sqrt(kk) / BOX
    with np.errstate(divide="ignore"):
        lp = np.interp(np.log(np.where(kk > 0, kphys, 1.0)), np.log(k_tab), np.log(p_tab))
    amp = np.sqrt(np.exp(lp) * N ** 3 / BOX ** 3)
    amp[0, 0, 0] = 0
    inv = np.where(kk > 0, 1.0 / np.where(kk > 0, kk, 1.0), 0.0)
    psi = [np.fft.irfftn(1j * kc / (2 * np.pi) * inv * amp * W, s=(N, N, N)).ravel() for kc in (kx, ky, kz)]
    i = np.arange(N ** 3)
    cells = np.stack([i % N, (i // N) % N, i // (N * N)], axis=1)
    return np.remainder((cells + 0.5) / N + np.stack(psi, axis=1), 1.0)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [gev.FP64, gev.MIXED])
def test_positions_phi_and_momenta(prec):
    N = 32
    k, pk = _pk_table()
    w = np.random.default_rng(4).standard_normal(N ** 3)
    fourpiG = _fourpiG()
    with gev.Context(N, precision=prec, capacity=N ** 3, boxsize=BOX) as c:
        c.ics_zeldovich(BOX, A, fourpiG, OM, OL, k, pk, noise=w)
        pos, q, ids = c.get_particles()
        phi = c.get_field(gev.FIELD_PHI).ravel()
    order = np.argsort(ids)
    pos, q, ids = pos[order], q[order], ids[order]
    assert np.array_equal(ids, np.arange(N ** 3))
    ref = _zeldovich_numpy(N, w, k, pk)
    d = pos - ref
    d -= np.round(d)
    tol = 1e-12 if prec == gev.FP64 else 2e-6
    assert np.abs(d).max() < tol, np.abs(d).max()
    # phi: CIC density of the GPU's particles, k = 0 removed, modified Poisson (ic_basic.hpp:2404-2427)
    o = oracle()
    rho = np.zeros(N ** 3)
    o.project_cic(N, len(pos), ptr(pos), OM / N ** 3, ptr(rho))
    FT = np.zeros(kshape(N), dtype=np.complex128)
    o.r2c(N, ptr(rho), ptr(FT))
    FT[0, 0, 0] = 0
    H = np.sqrt((2 * fourpiG / 3) * (OM / A + OL * A * A))
    o.solve_poisson(N, ptr(FT), ptr(FT), fourpiG / A, 3 * (H * H + fourpiG * OM / A))
    phi_ref = np.zeros(N ** 3)
    o.c2r(N, ptr(FT), ptr(phi_ref))
    assert rel_err(phi, phi_ref) < (1e-10 if prec == gev.FP64 else 1e-4)
    # momenta: initialize_q_ic_basic with rescale = a / H / (1.5 Omega_m(a))
    om_a = OM / (OM + OL * A ** 3)
    q_ref = np.zeros_like(pos)
    o.initialize_q(N, len(pos), ptr(np.ascontiguousarray(pos)), ptr(q_ref), ptr(phi_ref), A / H / (1.5 * om_a))
    assert rel_err(q, q_ref) < (1e-9 if prec == gev.FP64 else 1e-4)

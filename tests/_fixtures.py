"""Seeded synthetic inputs shared by the tests (small enough for the oracle)."""
import numpy as np


def particles(N, n=None, seed=1, qscale=0.02, lattice=False, disp=0.3):
    """Seeded particles in box units with momenta q.  lattice=True places one
    particle per cell (the sc1 lattice of the configs) displaced by up to
    `disp` cells; otherwise positions are uniform like unit_tests.cu:28-73."""
    rng = np.random.default_rng(seed)
    if lattice:
        g = (np.arange(N) + 0.125) / N
        x, y, z = np.meshgrid(g, g, g, indexing="ij")
        pos = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
        pos = pos + rng.uniform(-disp, disp, pos.shape) / N
        pos -= np.floor(pos)
        n = pos.shape[0]
    else:
        n = n if n is not None else 4 * N ** 3
        pos = rng.random((n, 3))
    q = rng.uniform(-qscale, qscale, (n, 3))
    ids = np.arange(n, dtype=np.int64) * 7 + 3
    return np.ascontiguousarray(pos), np.ascontiguousarray(q), ids


def trough_phi(N, amp=0.005):
    """unit_tests.cu:222-234: phi = -amp*(cos(pi r/N) - 1) for r < N/2 around the box centre."""
    i = np.arange(N)
    z, y, x = np.meshgrid(i, i, i, indexing="ij")
    r = np.sqrt((x - N / 2) ** 2 + (y - N / 2) ** 2 + (z - N / 2) ** 2)
    phi = np.where(r < N / 2, -amp * (np.cos(np.pi * r / N) - 1.0), 0.0)
    return np.ascontiguousarray(phi.ravel())


def smooth_field(N, seed, amp=1e-3, kmax=4):
    """Seeded smooth random field (a few low modes), flat N^3 array."""
    rng = np.random.default_rng(seed)
    i = np.arange(N) / N
    z, y, x = np.meshgrid(i, i, i, indexing="ij")
    f = np.zeros((N, N, N))
    for _ in range(6):
        k = rng.integers(-kmax, kmax + 1, 3)
        ph = rng.random() * 2 * np.pi
        f += rng.normal() * np.cos(2 * np.pi * (k[0] * x + k[1] * y + k[2] * z) + ph)
    f += 0.1 * rng.normal(size=f.shape)
    return np.ascontiguousarray((amp * f).ravel())


def rfft3(f, N):
    """Unnormalised forward R2C of a flat N^3 field (index x + N(y + Nz)) into
    the half spectrum [kz][ky][kx] with kx <= N/2 -- the library's and the
    oracle's convention, exp(-2 pi i k.x/N).  pocketfft through scipy.fft with
    all host threads."""
    import scipy.fft
    return scipy.fft.rfftn(np.asarray(f, dtype=np.float64).reshape(N, N, N), workers=-1)


def irfft3(F, N):
    """Unnormalised C2R of a half spectrum [kz][ky][kx] into a flat N^3 field."""
    import scipy.fft
    return scipy.fft.irfftn(F, s=(N, N, N), norm="forward", workers=-1).ravel()


def rel_err(a, b):
    """max |a - b| / max |b|; complex arrays are compared by the modulus of
    the complex difference (real and imaginary parts both count)."""
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    dt = np.complex128 if (np.iscomplexobj(a) or np.iscomplexobj(b)) else np.float64
    a = a.astype(dt, copy=False)
    b = b.astype(dt, copy=False)
    scale = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() / scale

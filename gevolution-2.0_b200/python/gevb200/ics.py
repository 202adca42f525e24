"""Seeded synthetic initial conditions for the benchmark boxes.

A Gaussian random field with the linear matter power spectrum at z_in
(primordial A_s, n_s, k_pivot; Eisenstein & Hu 1998 no-wiggle transfer
function; growth D = a in matter domination) displaces one particle per cell
from the cell centres (the sc1 template of gevolution's settings.ini tiled
N/4 times puts particles at (i + 1/2)/N) by the Zel'dovich approximation.
Momenta follow linear theory, q = a f H_conf psi.  The potential phi solves the
same modified Poisson equation as the reference's IC generator
(ic_basic.hpp:2404-2425): (k^2 + 3 (H^2 + 4 pi G Omega_m / a)) phi = -(4 pi G / a) delta rho.

This is input synthesis, not part of the timed cycle; it runs on torch.
"""
import math

import numpy as np

C_LIGHT = 2997.92458          # c in units of 100 km/s (metadata.hpp)


def eh_nowiggle_T(k_hmpc, h=0.67, omega_m=0.32, fb=0.15, tcmb=2.7255):
    """Eisenstein & Hu (1998) zero-baryon-oscillation transfer function; k in h/Mpc."""
    om_h2 = omega_m * h * h
    ob_h2 = fb * om_h2
    theta = tcmb / 2.7
    s = 44.5 * math.log(9.83 / om_h2) / math.sqrt(1.0 + 10.0 * ob_h2 ** 0.75)
    alpha = 1.0 - 0.328 * math.log(431.0 * om_h2) * fb + 0.38 * math.log(22.3 * om_h2) * fb * fb
    k = np.asarray(k_hmpc, dtype=np.float64) * h            # 1/Mpc
    gamma_eff = omega_m * h * (alpha + (1.0 - alpha) / (1.0 + (0.43 * k * s) ** 4))
    q = np.asarray(k_hmpc) * theta * theta / gamma_eff
    L0 = np.log(2.0 * math.e + 1.8 * q)
    C0 = 14.2 + 731.0 / (1.0 + 62.5 * q)
    return L0 / (L0 + C0 * q * q)


def linear_pk(k_hmpc, a, h=0.67, omega_m=0.32, A_s=2.1e-9, n_s=0.965, k_pivot=0.05):
    """Matter P(k) [(Mpc/h)^3] at scale factor a (early times, D = a)."""
    k = np.asarray(k_hmpc, dtype=np.float64)
    ks = np.maximum(k, 1e-30)                               # the k = 0 mode is set to zero below
    H0 = 1.0 / C_LIGHT                                      # h/Mpc
    T = eh_nowiggle_T(ks, h, omega_m)
    delta2 = (4.0 / 25.0) * (ks / H0) ** 4 / omega_m ** 2 * T * T * a * a * A_s * (ks * h / k_pivot) ** (n_s - 1.0)
    return np.where(k > 0, 2.0 * math.pi ** 2 * delta2 / ks ** 3, 0.0)


def sc1_template():
    """The 64-particle simple-cubic template of gevolution's sc1 crystal
    (settings.ini's particle file): one particle at the centre of each cell
    of a 4^3 grid, (i + 1/2) / 4 per axis, x fastest.  Tiled N/4 times per
    axis it puts one particle at every cell centre.  (The reference's file
    lists the same 64 positions in another order, which permutes the IDs
    within each tile.)"""
    g = (np.arange(4, dtype=np.float32) + np.float32(0.5)) / np.float32(4.0)
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    return np.ascontiguousarray(np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1), dtype=np.float32)


def hconf(a, fourpiG, om, ol):
    return math.sqrt((2.0 * fourpiG / 3.0) * (om / a + ol * a * a))


def zeldovich(N, boxsize, z_in, seed, device="cuda", omega_m=0.32, omega_l=0.68, h=0.67):
    """Returns (pos [n,3] float64 box units, q [n,3] float64, ids int64, phi [N^3] float64,
    mass) as torch tensors on `device` (phi as a flat array in x-fastest order)."""
    import torch

    a = 1.0 / (1.0 + z_in)
    fourpiG = 1.5 * boxsize * boxsize / C_LIGHT ** 2
    H = hconf(a, fourpiG, omega_m, omega_l)
    om_a = omega_m / (omega_m + omega_l * a ** 3)
    f = om_a ** 0.55
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    w = torch.randn((N, N, N), generator=g, device=device, dtype=torch.float32).to(torch.float64)
    W = torch.fft.rfftn(w)                                   # [kz, ky, kx]
    del w
    kf = torch.fft.fftfreq(N, d=1.0 / N, device=device, dtype=torch.float64)   # integer wavenumbers
    kh = torch.fft.rfftfreq(N, d=1.0 / N, device=device, dtype=torch.float64)
    kz, ky, kx = torch.meshgrid(kf, kf, kh, indexing="ij")
    k2 = (kx * kx + ky * ky + kz * kz) * (2 * math.pi) ** 2            # box units
    kmag = torch.sqrt(k2) / boxsize                                      # h/Mpc
    pk = torch.as_tensor(linear_pk(kmag.cpu().numpy(), a, h, omega_m), device=device)
    amp = torch.sqrt(pk * N ** 3 / boxsize ** 3)
    delta_k = W * amp
    delta_k[0, 0, 0] = 0
    del W, pk, amp, kmag
    inv = torch.where(k2 > 0, 1.0 / k2, torch.zeros_like(k2))
    psi = []
    for kc in (kx, ky, kz):
        psi.append(torch.fft.irfftn(1j * 2 * math.pi * kc * inv * delta_k, s=(N, N, N)).reshape(-1))
    # potential: finite-difference k^2 and the modified Poisson equation of ic_basic.hpp:2425
    gk2 = sum((2.0 * N * torch.sin(math.pi * kc / N)) ** 2 for kc in (kx, ky, kz))
    modif = 3.0 * (H * H + fourpiG * omega_m / a)
    phi_k = -(fourpiG / a) * omega_m * delta_k / (gk2 + modif)
    phi = torch.fft.irfftn(phi_k, s=(N, N, N)).reshape(-1)
    del delta_k, phi_k, inv, gk2, k2, kx, ky, kz
    i = (torch.arange(N, device=device, dtype=torch.float64) + 0.5) / N
    zz, yy, xx = torch.meshgrid(i, i, i, indexing="ij")
    lattice = torch.stack([xx.reshape(-1), yy.reshape(-1), zz.reshape(-1)], dim=1)
    del xx, yy, zz
    disp = torch.stack(psi, dim=1)
    pos = torch.remainder(lattice + disp, 1.0)
    q = a * f * H * disp
    ids = torch.arange(N ** 3, device=device, dtype=torch.int64)
    mass = omega_m / N ** 3
    return pos, q, ids, phi, mass, a, fourpiG

"""Differentiable Newtonian PM run through the C ABI (gev_pm_*), its
hand-written adjoint, and a thin torch.autograd.Function used for gradient
checks.

The run is main.cu's gr_flag == 0 branch for CDM: CIC projection, Poisson
solve with coefficient fourpiG / a, update_q_Newton (GRADIENT_ORDER 2) and
update_pos_Newton, on a fixed schedule of `nsteps` steps uniform in conformal
time.  Particles are in ID order with unwrapped box-unit positions.
"""
import ctypes
import math

import numpy as np

from . import Cosmo, GevError, _sig, particle_horizon, rungekutta4bg

_d, _i, _l, _p = ctypes.c_double, ctypes.c_int32, ctypes.c_int64, ctypes.c_void_p


class PmConfig(ctypes.Structure):
    _fields_ = [("N", _i), ("precision", _i), ("np", _l), ("mass", _d), ("checkpoint_every", _i), ("device", _i)]


_create = _sig("gev_pm_create", [ctypes.POINTER(PmConfig), ctypes.POINTER(_p)])
_destroy = _sig("gev_pm_destroy", [_p])
_err = _sig("gev_pm_last_error", [_p], ctypes.c_char_p)
_forward = _sig("gev_pm_forward", [_p, _i, _p, _p, _p, _p, _p, _p])
_adjoint = _sig("gev_pm_adjoint", [_p, _p, _p, _p])
_stream = _sig("gev_pm_stream", [_p], _p)


def schedule(N, fourpiG, omega_m, omega_l, a_in, a_out, nsteps):
    """Per-step coefficients (kq, kx, pc) of main.cu's Newtonian cycle with a
    fixed step dtau uniform in conformal time from a_in to a_out: the first kick
    uses (dtau + dtau_old)/2 with dtau_old = 0, the drift the scale factor after
    the first background half step (main.cu:1225-1283)."""
    c = Cosmo(omega_m, omega_l, 0.0, fourpiG, 48.0, 0.04, 0.0, 1.0)
    tau0 = particle_horizon(a_in, fourpiG, ctypes.byref(c))
    tau1 = particle_horizon(a_out, fourpiG, ctypes.byref(c))
    dtau = (tau1 - tau0) / nsteps
    coef = np.empty(3 * nsteps)
    a = a_in
    dtau_old = 0.0
    for n in range(nsteps):
        kick = 0.5 * (dtau + dtau_old)
        coef[3 * n] = kick * a * N                     # update_q_Newton: dtau * a / dx
        coef[3 * n + 2] = fourpiG / a                  # solveModifiedPoissonFT(..., fourpiG / a)
        ah = rungekutta4bg(a, fourpiG, c, 0.5 * dtau)
        coef[3 * n + 1] = dtau / ah                    # update_pos_Newton: dtau / a
        a = rungekutta4bg(ah, fourpiG, c, 0.5 * dtau)
        dtau_old = dtau
    return coef, a


class PM:
    """One differentiable run configuration on the current CUDA device."""

    def __init__(self, N, np_, mass, precision, checkpoint_every=8, device=0):
        self.N, self.np = int(N), int(np_)
        cfg = PmConfig(self.N, int(precision), self.np, float(mass), int(checkpoint_every), int(device))
        h = _p()
        rc = _create(ctypes.byref(cfg), ctypes.byref(h))
        if rc != 0:
            raise GevError(rc, _err(None).decode())
        self._h = h
        self._destroy = _destroy   # held by the object: module globals may be gone when it is collected at exit

    def close(self):
        if getattr(self, "_h", None):
            self._destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def _ck(self, rc):
        if rc != 0:
            raise GevError(rc, _err(self._h).decode())

    def stream(self):
        return _stream(self._h)

    def forward(self, coef, x0, q0, delta, x_out=None, q_out=None):
        """Device tensors: x0, q0 (np, 3) float64, delta N^3 float64 (written)."""
        coef = np.ascontiguousarray(coef, dtype=np.float64)
        self._ck(_forward(self._h, len(coef) // 3, coef.ctypes.data_as(_p), _p(x0.data_ptr()), _p(q0.data_ptr()),
                          _p(delta.data_ptr()), _p(x_out.data_ptr()) if x_out is not None else None,
                          _p(q_out.data_ptr()) if q_out is not None else None))

    def adjoint(self, ddelta, gx0, gq0):
        self._ck(_adjoint(self._h, _p(ddelta.data_ptr()), _p(gx0.data_ptr()), _p(gq0.data_ptr())))


def run_function():
    """torch.autograd.Function: (x0, q0) -> final CIC density contrast, with
    backward through gev_pm_adjoint."""
    import torch

    class PMRun(torch.autograd.Function):
        @staticmethod
        def forward(ctx, x0, q0, pm, coef):
            torch.cuda.synchronize()
            delta = torch.empty(pm.N ** 3, dtype=torch.float64, device=x0.device)
            pm.forward(coef, x0.detach().contiguous(), q0.detach().contiguous(), delta)
            ctx.pm = pm
            return delta

        @staticmethod
        def backward(ctx, gdelta):
            pm = ctx.pm
            torch.cuda.synchronize()
            gd = gdelta.detach().contiguous().to(torch.float64)
            gx = torch.empty((pm.np, 3), dtype=torch.float64, device=gd.device)
            gq = torch.empty((pm.np, 3), dtype=torch.float64, device=gd.device)
            pm.adjoint(gd, gx, gq)
            return gx, gq, None, None

    return PMRun


def zeldovich_map(noise, N, boxsize, a, fourpiG, omega_m=0.32, omega_l=0.68, h=0.67):
    """Differentiable (torch) map from white-noise modes (N^3 real, unit
    variance) to Zel'dovich initial conditions: unwrapped positions (np, 3) in
    box units from the cell-centre lattice, momenta q = a f H_conf psi."""
    import torch

    from .ics import linear_pk

    dev = noise.device
    H = math.sqrt((2.0 * fourpiG / 3.0) * (omega_m / a + omega_l * a * a))
    om_a = omega_m / (omega_m + omega_l * a ** 3)
    f = om_a ** 0.55
    W = torch.fft.rfftn(noise.reshape(N, N, N))
    kf = torch.fft.fftfreq(N, d=1.0 / N, device=dev, dtype=torch.float64)
    kh = torch.fft.rfftfreq(N, d=1.0 / N, device=dev, dtype=torch.float64)
    kz, ky, kx = torch.meshgrid(kf, kf, kh, indexing="ij")
    k2 = (kx * kx + ky * ky + kz * kz) * (2 * math.pi) ** 2
    kmag = torch.sqrt(k2) / boxsize
    pk = torch.as_tensor(linear_pk(kmag.cpu().numpy(), a, h, omega_m), device=dev)
    amp = torch.sqrt(pk * N ** 3 / boxsize ** 3)
    amp[0, 0, 0] = 0
    delta_k = W * amp
    inv = torch.where(k2 > 0, 1.0 / k2, torch.zeros_like(k2))
    psi = [torch.fft.irfftn(1j * 2 * math.pi * kc * inv * delta_k, s=(N, N, N)).reshape(-1) for kc in (kx, ky, kz)]
    i = (torch.arange(N, device=dev, dtype=torch.float64) + 0.5) / N
    zz, yy, xx = torch.meshgrid(i, i, i, indexing="ij")
    lattice = torch.stack([xx.reshape(-1), yy.reshape(-1), zz.reshape(-1)], dim=1)
    disp = torch.stack(psi, dim=1)
    return lattice + disp, a * f * H * disp

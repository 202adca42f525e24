"""Differentiable Newtonian PM run (gev_pm_*) and its hand-written adjoint.

- forward: one and several steps against the oracle's composition of the
  reference's Newtonian cycle (CIC projection, Poisson, update_q_Newton,
  update_pos_Newton; the kick/drift pinned to the reference in
  test_oracle_pin.py);
- adjoint: directional and per-mode central finite differences of the loss
  sum (delta - target)^2 with respect to the white-noise initial modes, the
  FP64 adjoint against the mixed-precision one, and repeatability."""
import math

import numpy as np
import pytest

from _fixtures import rel_err
from _libs import oracle, ptr

gev = pytest.importorskip("gevb200")
torch = pytest.importorskip("torch")
from gevb200 import pm as gpm  # noqa: E402

pytestmark = pytest.mark.gpu

OM, OL = 0.32, 0.68


def setup_run(N, nsteps, boxsize, z_in=50.0, seed=5):
    fourpiG = 1.5 * boxsize ** 2 / 2997.92458 ** 2
    a_in = 1.0 / (1.0 + z_in)
    coef, a_end = gpm.schedule(N, fourpiG, OM, OL, a_in, 1.0, nsteps)
    g = torch.Generator(device="cpu").manual_seed(seed)
    noise = torch.randn(N ** 3, generator=g, dtype=torch.float64).cuda()
    target = 0.5 * torch.randn(N ** 3, generator=g, dtype=torch.float64).cuda()
    return dict(N=N, fourpiG=fourpiG, a_in=a_in, coef=coef, noise=noise, target=target, boxsize=boxsize,
                mass=OM / N ** 3)


def ics(run, noise):
    return gpm.zeldovich_map(noise, run["N"], run["boxsize"], run["a_in"], run["fourpiG"], OM, OL)


def oracle_run(run, x0, q0, nsteps):
    """The same steps on the CPU oracle."""
    o = oracle()
    N = run["N"]
    x = np.ascontiguousarray(x0.cpu().numpy())
    q = np.ascontiguousarray(q0.cpu().numpy())
    np_ = len(x)
    for n in range(nsteps):
        kq, kx, pc = run["coef"][3 * n:3 * n + 3]
        rho = np.zeros(N ** 3)
        o.project_cic(N, np_, ptr(np.remainder(x, 1.0)), run["mass"], ptr(rho))
        src = np.zeros((N, N, N // 2 + 1), dtype=np.complex128)
        o.r2c(N, ptr(rho), ptr(src))
        pot = np.zeros_like(src)
        o.solve_poisson(N, ptr(src), ptr(pot), pc, 0.0)
        psi = np.zeros(N ** 3)
        o.c2r(N, ptr(pot), ptr(psi))
        # q -= dtau a N grad psi with dtau a N = kq; x += dtau q / a with dtau / a = kx
        o.update_q_newton(N, np_, ptr(np.remainder(x, 1.0)), ptr(q), ptr(psi), kq / N, 1.0)
        o.lib.orc_update_pos_newton(np_, ptr(x), ptr(q), kx, 1.0)
    rho = np.zeros(N ** 3)
    o.project_cic(N, np_, ptr(np.remainder(x, 1.0)), 1.0 / np_, ptr(rho))
    return x, q, rho - 1.0


@pytest.mark.parametrize("nsteps", [1, 3])
def test_forward_matches_oracle(nsteps):
    N = 32
    run = setup_run(N, 8, 160.0)
    x0, q0 = ics(run, run["noise"])
    p = gpm.PM(N, N ** 3, run["mass"], gev.FP64, checkpoint_every=2)
    delta = torch.empty(N ** 3, dtype=torch.float64, device="cuda")
    xo = torch.empty_like(x0)
    qo = torch.empty_like(q0)
    p.forward(run["coef"][:3 * nsteps], x0, q0, delta, xo, qo)
    xr, qr, dr = oracle_run(run, x0, q0, nsteps)
    assert rel_err(qo.cpu().numpy(), qr) < 1e-10
    assert np.abs(xo.cpu().numpy() - xr).max() < 1e-12
    assert rel_err(delta.cpu().numpy(), dr) < 1e-10


def loss_and_grad(run, noise, precision, every=8, nsteps=None):
    N = run["N"]
    coef = run["coef"] if nsteps is None else run["coef"][:3 * nsteps]
    p = gpm.PM(N, N ** 3, run["mass"], precision, checkpoint_every=every)
    PMRun = gpm.run_function()
    w = noise.clone().requires_grad_(True)
    x0, q0 = ics(run, w)
    delta = PMRun.apply(x0, q0, p, coef)
    loss = ((delta - run["target"]) ** 2).sum()
    loss.backward()
    return loss.item(), w.grad.detach().clone()


def loss_only(run, noise, precision=None, nsteps=None):
    N = run["N"]
    coef = run["coef"] if nsteps is None else run["coef"][:3 * nsteps]
    p = gpm.PM(N, N ** 3, run["mass"], gev.FP64 if precision is None else precision, checkpoint_every=8)
    x0, q0 = ics(run, noise)
    delta = torch.empty(N ** 3, dtype=torch.float64, device="cuda")
    p.forward(coef, x0.contiguous(), q0.contiguous(), delta)
    return ((delta - run["target"]) ** 2).sum().item()


def test_adjoint_directional_derivative():
    """<grad, v> against a central difference along a random direction v."""
    run = setup_run(32, 16, 160.0)
    L, g = loss_and_grad(run, run["noise"], gev.FP64, every=4)
    v = torch.randn(run["N"] ** 3, generator=torch.Generator().manual_seed(9), dtype=torch.float64).cuda()
    eps = 1e-5
    fd = (loss_only(run, run["noise"] + eps * v) - loss_only(run, run["noise"] - eps * v)) / (2 * eps)
    ad = float((g * v).sum())
    assert abs(fd - ad) / abs(ad) < 1e-3, (fd, ad)


def test_adjoint_modes_fd_and_fp64_vs_mixed():
    """The differentiable configuration on a reduced grid: per-mode central
    differences on 16 random modes, and the mixed-precision adjoint against FP64."""
    run = setup_run(64, 32, 320.0)
    L, g64 = loss_and_grad(run, run["noise"], gev.FP64, every=8)
    rng = np.random.default_rng(3)
    modes = rng.choice(run["N"] ** 3, size=16, replace=False)
    eps = 1e-4
    fd = []
    for m in modes:
        e = torch.zeros_like(run["noise"])
        e[int(m)] = eps
        fd.append((loss_only(run, run["noise"] + e) - loss_only(run, run["noise"] - e)) / (2 * eps))
    fd = np.array(fd)
    ad = g64.cpu().numpy()[modes]
    assert np.linalg.norm(fd - ad) / np.linalg.norm(ad) < 1e-3, (fd, ad)
    _, g32 = loss_and_grad(run, run["noise"], gev.MIXED, every=8)
    assert float(torch.linalg.norm(g32 - g64) / torch.linalg.norm(g64)) < 1e-3


def test_adjoint_checkpoint_interval_and_repeat():
    run = setup_run(32, 12, 160.0)
    L1, g1 = loss_and_grad(run, run["noise"], gev.FP64, every=12)
    L2, g2 = loss_and_grad(run, run["noise"], gev.FP64, every=5)
    assert abs(L1 / L2 - 1) < 1e-12
    assert float(torch.linalg.norm(g1 - g2) / torch.linalg.norm(g1)) < 1e-10

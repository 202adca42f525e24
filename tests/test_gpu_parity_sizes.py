"""GPU parity of the Fourier solves at production grid sizes.

The kernels that the 512^3 cycle runs are specialised per N: the y and z
passes load their pencils as one bulk tensor box up to N = 256 and as several
boxes beyond (N = 384: three boxes of 128; N = 512: two of 256; N = 768: three
of 256), and every N has its own twiddle tables and radix sequence.  These
tests compare each solve with an independent FP64 reference at those sizes:
pocketfft (scipy.fft, the same transform numpy uses, pinned to the oracle's
FFT in test_oracle_pin.py) for the transforms and the oracle's C restatements
for the pointwise physics (prepareFTsource, solveModifiedPoissonFT,
projectFTscalar, projectFTtensor, evolveFTtensor, projectFTvector), which are
themselves pinned to the reference's own code.

Inputs are seeded white noise, which puts weight on every mode and so on every
twiddle factor and box offset.  Tolerances: FP64 1e-10 and mixed precision
(FP32 fields and transforms, FP64 solver arithmetic) 1e-4, relative to the
largest magnitude of the compared array, as for the small-N solver tests.
Complex spectra are compared by the modulus of the complex difference.

Each test computes its reference once and checks both precisions against it."""
import numpy as np
import pytest

from _fixtures import irfft3, rel_err, rfft3
from _libs import oracle, ptr

gev = pytest.importorskip("gevb200")

pytestmark = pytest.mark.gpu

TOL = {gev.FP64: 1e-10, gev.MIXED: 1e-4}
PRECS = (gev.FP64, gev.MIXED)
FOURPIG = 1.5 * 2560.0 ** 2 / 2997.92458 ** 2
SIZES = [128, 256, 384, 512]


def noise(N, seed, amp=1.0, ncomp=1):
    rng = np.random.default_rng(seed)
    return amp * rng.standard_normal(ncomp * N ** 3)


def ctx(N, prec, **kw):
    c = gev.Context(N, precision=prec, capacity=8, **kw)
    c.set_particles(np.zeros((1, 3)), np.zeros((1, 3)))
    return c


@pytest.mark.parametrize("N", SIZES)
def test_solve_phi_sizes(N):
    """prepareFTsource (T00 form) + R2C + solveModifiedPoissonFT + C2R
    (main.cu:719-809) and the k = 0 mode, at N = 128 ... 512."""
    o = oracle()
    dx = 1.0 / N
    source = 0.32 * (1.0 + 0.5 * noise(N, 101))
    phi = noise(N, 102, 1e-5)
    chi = noise(N, 103, 1e-6)
    H, dtau_old, a = 0.8, 0.01, 0.3
    args = (0.32, 3 * H * dx * dx / dtau_old, FOURPIG * dx * dx / a, 3 * H * H * dx * dx)
    res = np.zeros(N ** 3)
    s_ref = o.prepare_T00(N, ptr(phi), ptr(chi), ptr(source), *args, ptr(res))
    FT = rfft3(res, N)
    del res
    o.solve_poisson(N, ptr(FT), ptr(FT), 1 / (dx * dx), 3 * H / dtau_old)
    phom_ref = FT[0, 0, 0].real
    scale_ft = np.abs(FT).max()
    ph_ref = irfft3(FT, N)
    del FT
    for prec in PRECS:
        with ctx(N, prec) as c:
            c.set_field(gev.FIELD_SOURCE, source)
            c.set_field(gev.FIELD_PHI, phi)
            c.set_field(gev.FIELD_CHI, chi)
            s, phom = c.solve_phi(True, *args, 1 / (dx * dx), 3 * H / dtau_old)
            assert abs(s / s_ref - 1) < (1e-12 if prec == gev.FP64 else 1e-6), prec
            assert abs(phom - phom_ref) <= TOL[prec] * scale_ft, prec
            assert rel_err(c.get_field(gev.FIELD_PHI), ph_ref) < TOL[prec], prec


def test_solve_phi_768_mixed():
    """The 768^3 z and y passes (three bulk tensor boxes of 256 per pencil) in
    mixed precision, without prepareFTsource: R2C, solveModifiedPoissonFT with
    a screening term, C2R."""
    N = 768
    o = oracle()
    dx = 1.0 / N
    source = noise(N, 111)
    FT = rfft3(source, N)
    o.solve_poisson(N, ptr(FT), ptr(FT), 1 / (dx * dx), 40.0)
    ph_ref = irfft3(FT, N)
    del FT
    with ctx(N, gev.MIXED) as c:
        c.set_field(gev.FIELD_SOURCE, source)
        c.solve_phi(False, 0.0, 0.0, 0.0, 0.0, 1 / (dx * dx), 40.0)
        assert rel_err(c.get_field(gev.FIELD_PHI), ph_ref) < TOL[gev.MIXED]


@pytest.mark.parametrize("N", SIZES)
def test_solve_chi_tensor_sizes(N):
    """prepareFTsource (Tij form) + 6 R2C + projectFTscalar + C2R (main.cu:811-903)
    with the tensor state on: projectFTtensor on the first cycle, then one
    evolveFTtensor step (main.cu:961-965); h_ij and h_ij' compared as complex
    spectra, chi in real space."""
    o = oracle()
    dx = 1.0 / N
    n3 = N ** 3
    Tij = noise(N, 120, 1e-3, 6)
    phi = noise(N, 121, 1e-5)
    coeff = 2 * FOURPIG * dx * dx / 0.4
    S = np.zeros(6 * n3)
    o.prepare_Tij(N, ptr(phi), ptr(Tij), coeff, ptr(S))
    SFT = np.empty((6, N, N, N // 2 + 1), dtype=np.complex128)
    for k in range(6):
        SFT[k] = rfft3(S[k * n3:(k + 1) * n3], N)
    del S
    chiFT = np.zeros((N, N, N // 2 + 1), dtype=np.complex128)
    o.project_scalar(N, ptr(SFT), ptr(chiFT), 0)
    chi_ref = irfft3(chiFT, N)
    del chiFT
    hFT = np.zeros_like(SFT)
    o.project_tensor(N, ptr(SFT), ptr(hFT))
    hubble, dtau, dtau_old = 0.9, 0.01, 0.012
    h1, hp1 = hFT.copy(), np.zeros_like(hFT)
    o.evolve_tensor(N, ptr(SFT), ptr(h1), ptr(hp1), hubble, dtau, dtau_old)   # modifies SFT's trace at k = 0
    del SFT
    for prec in PRECS:
        with ctx(N, prec, tensor=True) as c:
            c.set_field(gev.FIELD_SIJ, Tij)
            c.set_field(gev.FIELD_PHI, phi)
            c.solve_chi(coeff, cycle0=True)
            assert rel_err(c.get_field(gev.FIELD_CHI), chi_ref) < TOL[prec], prec
            assert rel_err(c.get_field(gev.FIELD_HIJ_FT), hFT) < TOL[prec], prec
            c.solve_chi(coeff, cycle0=False, hubble=hubble, dtau=dtau, dtau_old=dtau_old)
            assert rel_err(c.get_field(gev.FIELD_CHI), chi_ref) < TOL[prec], prec
            assert rel_err(c.get_field(gev.FIELD_HIJ_FT), h1) < TOL[prec], prec
            assert rel_err(c.get_field(gev.FIELD_HIJP_FT), hp1) < TOL[prec], prec


@pytest.mark.parametrize("N", SIZES)
def test_solve_B_sizes(N):
    """3 R2C + projectFTvector + 3 C2R (main.cu:905-955)."""
    o = oracle()
    dx = 1.0 / N
    n3 = N ** 3
    T0i = noise(N, 130, 1e-4, 3)
    FT = np.empty((3, N, N, N // 2 + 1), dtype=np.complex128)
    for k in range(3):
        FT[k] = rfft3(T0i[k * n3:(k + 1) * n3], N)
    coeff = FOURPIG * dx * dx
    o.project_vector(N, ptr(FT), ptr(FT), coeff, 0.0)
    B_ref = np.concatenate([irfft3(FT[k], N) for k in range(3)])
    del FT
    for prec in PRECS:
        with ctx(N, prec) as c:
            c.set_field(gev.FIELD_BI, T0i)
            c.solve_B(coeff)
            assert rel_err(c.get_field(gev.FIELD_BI).ravel(), B_ref) < TOL[prec], prec
